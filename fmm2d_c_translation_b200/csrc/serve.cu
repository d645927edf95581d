// serve.cu -- the request loop for many independent evaluations on one GPU.
//
// A server owns `slots` worker threads.  Each worker has its own CUDA
// stream (the per-thread stream of the library), so the evaluations it runs
// overlap on the device with those of the other workers.  Requests enter a
// queue; a free worker takes the first queued request whose estimated
// device footprint fits into what the HBM budget has left (a request that
// does not fit yet does not hold back the smaller ones behind it, within a
// look-ahead window), runs it through the same engine as the drop-in entry
// points, and releases its share of the budget when it finishes.  Workspace
// comes from the device's stream-ordered pool, so a finished request's
// blocks are reused by the next ones without returning to the driver.
//
// Continuous batching: a worker that takes a small lfmm2d request also
// takes the queued requests of the same kind (arithmetic -- mixed, FP64 or
// split --, strengths, output flags) that fit the budget, up to kBatchMax
// requests and kBatchPoints points, and evaluates them together as one
// forest (run_laplace_batch) at the smallest eps among them: one launch per
// level and pass for all of them.  Their trees (and, for the looser eps,
// their orders) differ from the ones they would get alone, so their results
// agree with the alone ones to the requested eps.  FMM2D_B200_SERVE_BATCH=0, read
// when the server is made, turns batching off.
//
// The reference has no counterpart (its entry points are single calls).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>
#include <stdlib.h>
#include <string.h>

#include "engine.cuh"
#include "helmholtz.cuh"
#include "runtime.cuh"

namespace fmm2d {
namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Upper estimate of the device bytes one evaluation holds at its peak:
// inputs and their tree-order copies, outputs in both orders, the tree
// (boxes <= 4 (ns + nt) / ndiv + levels), lists and expansions, and the
// sort buffers.
double footprint_bytes(const FmmCall &c) {
    const double ns = c.ns, nt = c.nt, nd = c.nd;
    const int ndiv = std::max(1, c.ndiv >= 0 ? c.ndiv : leaf_capacity(c.eps, c.ns, c.nt));
    const double nb = 4.0 * (ns + nt) / ndiv + 64.0;
    const double ndc = c.kernel == kLaplace ? 2.0 * nd : nd;
    double coeffs;
    if (c.kernel == kHelmholtz) {
        // the finest levels dominate; the coarse ones add at most a factor
        // of two for the orders reached at |zk| <= 2 pi * 16 per box
        const double zk = std::hypot(c.zk[0], c.zk[1]);
        const double p = 40.0 + 2.0 * zk;
        coeffs = 2.0 * nb * (2.0 * p + 1.0) * nd * 2.0;
    } else {
        coeffs = 2.0 * nb * (laplace_nterms(c.eps) + 1.0) * ndc;
    }
    const int comps = c.kernel == kCauchy ? 1 : 3;
    const double pts = 16.0 * (ns + nt) * 3.0;
    const double strengths = 16.0 * ns * ndc * (c.ifcharge + c.ifdipole) * 2.0 + 32.0 * ns * nd;
    const double outs = 16.0 * ndc * comps * 2.0 * (ns * (c.ifpgh > 0) + nt * (c.ifpghtarg > 0));
    const double tree = 400.0 * nb + 40.0 * (ns + nt);
    return 1.25 * (pts + strengths + outs + tree + 16.0 * coeffs) + (1 << 20);
}

constexpr int kBatchMax = 64;
constexpr int kBatchPoints = 200000;   // points of one batch
constexpr int kBatchRequest = 50000;   // largest request that is batched

// A request may join a batch only if it would also pass the batch driver's
// own argument checks (at least one source, a charge or a dipole, valid
// output flags), so one malformed request cannot fail its neighbours.
bool batchable(const FmmCall &c) {
    return c.kernel == kLaplace && c.nd == 1 && c.ndiv < 0 && c.ifnear == 1 && !c.timeinfo &&
           c.ns >= 1 && c.nt >= 0 && (c.ifcharge || c.ifdipole) && c.ifpgh >= 0 &&
           c.ifpgh <= 3 && c.ifpghtarg >= 0 && c.ifpghtarg <= 3 &&
           (int64_t)c.ns + c.nt <= kBatchRequest;
}

// The arithmetic a call runs in: 2 mixed (explicit, or auto at eps >= 0.5e-6),
// else its precision code (all-FP64 or split).
int arith_class(const FmmCall &c) {
    const bool mixed = c.precision == kPrecMixed || (c.precision == kPrecAuto && c.eps >= 0.5e-6);
    return mixed ? kPrecMixed : (c.precision == kPrecAuto ? kPrecFP64 : c.precision);
}

// Requests of one arithmetic and output layout batch together; the batch
// runs at the smallest eps among them, which meets every member's eps.
bool same_kind(const FmmCall &a, const FmmCall &b) {
    return arith_class(a) == arith_class(b) && a.ifcharge == b.ifcharge &&
           a.ifdipole == b.ifdipole && a.ifpgh == b.ifpgh && (a.nt > 0) == (b.nt > 0) &&
           (a.nt == 0 || a.ifpghtarg == b.ifpghtarg);
}

struct Request {
    FmmCall call;
    double bytes = 0;
    double t_submit = 0, t_start = 0, t_end = 0;
    int ier = 0;
    bool done = false;
};

class Server {
  public:
    Server(int slots, double budget, int device)
        : budget_(budget), device_(device) {
        const char *e = getenv("FMM2D_B200_SERVE_BATCH");
        batch_ = !(e && !strcmp(e, "0"));
        for (int i = 0; i < slots; i++) workers_.emplace_back([this] { loop(); });
    }
    ~Server() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_work_.notify_all();
        for (auto &t : workers_) t.join();
        for (auto &kv : reqs_) delete kv.second;
    }

    long long submit(const FmmCall &c) {
        Request *r = new Request;
        r->call = c;
        r->bytes = footprint_bytes(c);
        r->t_submit = now_ms();
        std::lock_guard<std::mutex> g(mu_);
        const long long id = next_id_++;
        reqs_[id] = r;
        if (r->bytes > budget_) {
            // can never be admitted
            r->ier = 4;
            r->done = true;
            r->t_start = r->t_end = r->t_submit;
            rejected_++;
        } else {
            queue_.push_back(id);
            cv_work_.notify_one();
        }
        return id;
    }

    // Blocks until request `id` has finished; fills queue, run and total
    // milliseconds and forgets the request.
    int wait(long long id, double *times) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end()) return -1;
        Request *r = it->second;
        cv_done_.wait(lk, [&] { return r->done; });
        if (times) {
            times[0] = r->t_start - r->t_submit;
            times[1] = r->t_end - r->t_start;
            times[2] = r->t_end - r->t_submit;
        }
        const int ier = r->ier;
        reqs_.erase(it);
        delete r;
        return ier;
    }

    // in-use bytes now, the largest in-use seen, requests queued, running,
    // rejected
    void stats(double *out) {
        std::lock_guard<std::mutex> g(mu_);
        out[0] = in_use_;
        out[1] = peak_in_use_;
        out[2] = (double)queue_.size();
        out[3] = running_;
        out[4] = rejected_;
        out[5] = peak_running_;
    }

    // requests that ran in batches of two or more
    long long batched() {
        std::lock_guard<std::mutex> g(mu_);
        return batched_;
    }

  private:
    static constexpr size_t kWindow = 64;

    // first queued request (within the window) that fits the budget left
    bool pick(long long &id) {
        const size_t n = std::min(queue_.size(), kWindow);
        for (size_t i = 0; i < n; i++) {
            Request *r = reqs_[queue_[i]];
            if (in_use_ + r->bytes <= budget_) {
                id = queue_[i];
                queue_.erase(queue_.begin() + (long)i);
                return true;
            }
        }
        return false;
    }

    // Queued requests of r's kind that fit the budget (mu_ held).
    void gather_batch(Request *r, std::vector<Request *> &batch) {
        int64_t pts = (int64_t)r->call.ns + r->call.nt;
        size_t i = 0;
        while (i < std::min(queue_.size(), kWindow) && (int)batch.size() < kBatchMax) {
            Request *q = reqs_[queue_[i]];
            const int64_t n = (int64_t)q->call.ns + q->call.nt;
            if (batchable(q->call) && same_kind(r->call, q->call) && pts + n <= kBatchPoints &&
                in_use_ + q->bytes <= budget_) {
                batch.push_back(q);
                in_use_ += q->bytes;
                pts += n;
                queue_.erase(queue_.begin() + (long)i);
            } else {
                i++;
            }
        }
    }

    int run_batch(const std::vector<Request *> &batch) {
        const size_t n = batch.size();
        std::vector<int> ns(n), nt(n);
        std::vector<const double *> src(n), trg(n), q(n), d(n), v(n);
        std::vector<double *> o[6];
        for (auto &x : o) x.resize(n);
        for (size_t k = 0; k < n; k++) {
            const FmmCall &c = batch[k]->call;
            ns[k] = c.ns;
            nt[k] = c.nt;
            src[k] = c.sources;
            trg[k] = c.targ;
            q[k] = c.charge;
            d[k] = c.dipstr;
            v[k] = c.dipvec;
            o[0][k] = c.pot;
            o[1][k] = c.grad;
            o[2][k] = c.hess;
            o[3][k] = c.pottarg;
            o[4][k] = c.gradtarg;
            o[5][k] = c.hesstarg;
        }
        const FmmCall &c0 = batch[0]->call;
        BatchCall b;
        b.kernel = c0.kernel;
        b.eps = c0.eps;
        for (const Request *r : batch) b.eps = std::min(b.eps, r->call.eps);
        b.nprob = (int)n;
        b.ns = ns.data();
        b.nt = nt.data();
        b.sources = src.data();
        b.targ = trg.data();
        b.charge = c0.ifcharge ? q.data() : nullptr;
        b.dipstr = c0.ifdipole ? d.data() : nullptr;
        b.dipvec = c0.ifdipole ? v.data() : nullptr;
        b.ifpgh = c0.ifpgh;
        b.ifpghtarg = c0.ifpghtarg;
        b.pot = o[0].data();
        b.grad = o[1].data();
        b.hess = o[2].data();
        b.pottarg = o[3].data();
        b.gradtarg = o[4].data();
        b.hesstarg = o[5].data();
        // (the class's arithmetic at the batch's eps)
        b.precision = arith_class(c0) == kPrecMixed ? kPrecMixed : c0.precision;
        return run_laplace_batch(b);
    }

    void loop() {
        cudaSetDevice(device_);
        for (;;) {
            long long id = -1;
            std::vector<Request *> batch;
            {
                std::unique_lock<std::mutex> lk(mu_);
                // queued work is drained before a stopping server exits
                cv_work_.wait(lk, [&] { return pick(id) || (stop_ && queue_.empty()); });
                if (id < 0) return;
                Request *r = reqs_[id];
                batch.push_back(r);
                in_use_ += r->bytes;
                if (batch_ && batchable(r->call)) gather_batch(r, batch);
                peak_in_use_ = std::max(peak_in_use_, in_use_);
                running_ += (int)batch.size();
                peak_running_ = std::max(peak_running_, running_);
                if (batch.size() > 1) batched_ += (long long)batch.size();
            }
            const double t0 = now_ms();
            for (Request *r : batch) r->t_start = t0;
            std::vector<int> iers(batch.size(), 0);
            if (batch.size() == 1) {
                iers[0] = run_fmm(batch[0]->call);
            } else if (run_batch(batch) != 0) {
                // a failed batch is rerun one request at a time, so each
                // request gets the status it would have had alone
                for (size_t i = 0; i < batch.size(); i++) iers[i] = run_fmm(batch[i]->call);
            }
            const double t_end = now_ms();
            {
                std::lock_guard<std::mutex> g(mu_);
                for (size_t i = 0; i < batch.size(); i++) {
                    Request *r = batch[i];
                    r->ier = iers[i];
                    r->t_end = t_end;
                    r->done = true;
                    in_use_ -= r->bytes;
                }
                running_ -= (int)batch.size();
            }
            cv_done_.notify_all();
            cv_work_.notify_all();
        }
    }

    double budget_;
    int device_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::deque<long long> queue_;
    std::unordered_map<long long, Request *> reqs_;
    std::vector<std::thread> workers_;
    long long next_id_ = 0;
    double in_use_ = 0, peak_in_use_ = 0;
    int running_ = 0, peak_running_ = 0, rejected_ = 0;
    long long batched_ = 0;
    bool stop_ = false, batch_ = true;
};

}  // namespace
}  // namespace fmm2d

using namespace fmm2d;

// One request (host or device arrays, the guru drivers' arguments).
struct fmm2d_b200_request {
    int kernel;  // 0 lfmm2d, 1 cfmm2d, 2 hfmm2d
    int nd;
    double eps;
    double zk[2];
    int ns;
    const double *sources;
    int ifcharge;
    const double *charge;
    int ifdipole;
    const double *dipstr;
    const double *dipvec;
    int ifpgh;
    double *pot, *grad, *hess;
    int nt;
    const double *targ;
    int ifpghtarg;
    double *pottarg, *gradtarg, *hesstarg;
    int precision;  // 0 auto, 1 all-FP64, 2 mixed
};

FMM_EXPORT void *fmm2d_b200_server_create(int slots, double hbm_budget_bytes) {
    if (slots < 1 || hbm_budget_bytes <= 0) return nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = 0;
    }
    return new Server(slots, hbm_budget_bytes, dev);
}

FMM_EXPORT long long fmm2d_b200_server_submit(void *srv, const fmm2d_b200_request *q) {
    if (!srv || !q || q->kernel < 0 || q->kernel > 2) return -1;
    FmmCall c;
    c.kernel = (Kernel)q->kernel;
    c.nd = q->nd;
    c.eps = q->eps;
    c.zk[0] = q->zk[0];
    c.zk[1] = q->zk[1];
    c.ns = q->ns;
    c.sources = q->sources;
    c.ifcharge = q->ifcharge;
    c.charge = q->charge;
    c.ifdipole = q->ifdipole;
    c.dipstr = q->dipstr;
    c.dipvec = q->dipvec;
    c.ifpgh = q->ifpgh;
    c.pot = q->pot;
    c.grad = q->grad;
    c.hess = q->hess;
    c.nt = q->nt;
    c.targ = q->targ;
    c.ifpghtarg = q->ifpghtarg;
    c.pottarg = q->pottarg;
    c.gradtarg = q->gradtarg;
    c.hesstarg = q->hesstarg;
    c.precision = q->precision;
    return static_cast<Server *>(srv)->submit(c);
}

FMM_EXPORT int fmm2d_b200_server_wait(void *srv, long long ticket, double *times_ms) {
    if (!srv) return -1;
    return static_cast<Server *>(srv)->wait(ticket, times_ms);
}

FMM_EXPORT void fmm2d_b200_server_stats(void *srv, double *out6) {
    if (srv) static_cast<Server *>(srv)->stats(out6);
}

FMM_EXPORT double fmm2d_b200_request_bytes(const fmm2d_b200_request *q) {
    FmmCall c;
    c.kernel = (Kernel)q->kernel;
    c.nd = q->nd;
    c.eps = q->eps;
    c.zk[0] = q->zk[0];
    c.zk[1] = q->zk[1];
    c.ns = q->ns;
    c.nt = q->nt;
    c.ifcharge = q->ifcharge;
    c.ifdipole = q->ifdipole;
    c.ifpgh = q->ifpgh;
    c.ifpghtarg = q->ifpghtarg;
    return footprint_bytes(c);
}

FMM_EXPORT void fmm2d_b200_server_destroy(void *srv) { delete static_cast<Server *>(srv); }

// Requests of the server that ran in batches of two or more so far.
FMM_EXPORT long long fmm2d_b200_server_batched(void *srv) {
    return srv ? static_cast<Server *>(srv)->batched() : 0;
}
