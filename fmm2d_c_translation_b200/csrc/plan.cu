// plan.cu -- resident geometry for repeated Laplace / Cauchy evaluations.
//
// A plan keeps on the device what a call derives from the points alone:
// the adaptive tree, its interaction lists, the points in tree order and
// the M2L planning (work lists, window runs).  Each evaluation then only
// gathers the new strengths, runs the FMM passes and scatters the outputs
// -- the pattern of an iterative solver that applies the same
// boundary-integral operator to a new density every step.
//
// The first evaluation runs eagerly and fills the planning cache.  From the
// second one on, the whole evaluation -- gathers, the level sweeps of every
// pass, scatters -- is captured once into a CUDA graph over plan-owned
// staging buffers and replayed: the caller's arrays are copied in, the
// graph is launched, the outputs are copied out.  The M2L's bounded-wait
// error flag is then read after the launch.  FMM2D_B200_PLAN_GRAPH=0 keeps
// every evaluation eager; a capture that fails falls back to eager
// evaluations for the plan.
//
// The plan owns a stream for its buffers and graph launches, so it may be
// destroyed from any thread; evaluations of one plan are serialised.
#include "engine.cuh"
#include "laplace.cuh"
#include "runtime.cuh"

#include <mutex>

namespace fmm2d {
namespace {

struct Plan {
    int dev = 0;
    cudaStream_t s = nullptr;
    FmmCall shape;
    LapGeometry G;
    std::mutex mu;
    M2LCache cache;
    bool warm = false;  // the first (eager) evaluation filled the cache
    // graph replay
    bool graph_failed = false;
    cudaGraphExec_t exec = nullptr;
    DevBuf<int> err;
    DevBuf<double> in[3];   // charge, dipstr, dipvec (the caller's layouts)
    size_t in_n[3] = {0, 0, 0};
    DevBuf<double> out[6];  // pot, grad, hess, pottarg, gradtarg, hesstarg
    size_t out_n[6] = {0, 0, 0, 0, 0, 0};
    ~Plan() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

bool on_device(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool graphs_enabled() {
    const char *e = getenv("FMM2D_B200_PLAN_GRAPH");
    return !(e && !strcmp(e, "0"));
}

// Sizes (in doubles) of the caller's strength and output arrays.
void array_sizes(Plan &pl) {
    const FmmCall &c = pl.shape;
    const bool lap = c.kernel == kLaplace;
    const size_t nd = c.nd, ns = c.ns, nt = c.nt;
    const size_t gc = lap ? 2 : 1, hc = lap ? 3 : 1;
    pl.in_n[0] = c.ifcharge ? 2 * nd * ns : 0;
    pl.in_n[1] = c.ifdipole ? 2 * nd * ns : 0;
    pl.in_n[2] = (c.ifdipole && lap) ? 2 * nd * ns : 0;
    pl.out_n[0] = c.ifpgh >= 1 ? 2 * nd * ns : 0;
    pl.out_n[1] = c.ifpgh >= 2 ? 2 * nd * gc * ns : 0;
    pl.out_n[2] = c.ifpgh >= 3 ? 2 * nd * hc * ns : 0;
    pl.out_n[3] = c.ifpghtarg >= 1 ? 2 * nd * nt : 0;
    pl.out_n[4] = c.ifpghtarg >= 2 ? 2 * nd * gc * nt : 0;
    pl.out_n[5] = c.ifpghtarg >= 3 ? 2 * nd * hc * nt : 0;
}

// Captures one evaluation over the staging buffers into pl.exec.
void build_graph(Plan &pl) {
    cudaStream_t s = pl.s;
    array_sizes(pl);
    for (int k = 0; k < 3; k++)
        if (pl.in_n[k]) pl.in[k].alloc(pl.in_n[k], s);
    for (int k = 0; k < 6; k++)
        if (pl.out_n[k]) pl.out[k].alloc(pl.out_n[k], s);
    pl.err.alloc(1, s);
    pl.err.zero(s);
    FMM_CUDA(cudaStreamSynchronize(s));
    FmmCall g = pl.shape;
    g.charge = pl.in[0].get();
    g.dipstr = pl.in[1].get();
    g.dipvec = pl.in[2].get();
    double *o[6];
    for (int k = 0; k < 6; k++) o[k] = pl.out[k].get();
    g.pot = o[0];
    g.grad = o[1];
    g.hess = o[2];
    g.pottarg = o[3];
    g.gradtarg = o[4];
    g.hesstarg = o[5];
    pl.cache.err = pl.err.get();
    pl.cache.deferred = true;
    cudaGraph_t graph = nullptr;
    FMM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
        laplace_evaluate(g, pl.G, true, s, &pl.cache, false);
    } catch (...) {
        cudaStreamEndCapture(s, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        pl.cache.deferred = false;
        throw;
    }
    pl.cache.deferred = false;
    FMM_CUDA(cudaStreamEndCapture(s, &graph));
    const cudaError_t e = cudaGraphInstantiate(&pl.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        pl.exec = nullptr;
        FMM_CUDA(e);
    }
}

// One replay: the caller's strengths in, the graph, the outputs out.
void replay(Plan &pl, const double *const in[3], double *const out[6]) {
    cudaStream_t s = pl.s;
    for (int k = 0; k < 3; k++)
        if (pl.in_n[k])
            FMM_CUDA(cudaMemcpyAsync(pl.in[k].get(), in[k], pl.in_n[k] * sizeof(double),
                                     cudaMemcpyDefault, s));
    FMM_CUDA(cudaGraphLaunch(pl.exec, s));
    for (int k = 0; k < 6; k++)
        if (pl.out_n[k] && out[k])
            FMM_CUDA(cudaMemcpyAsync(out[k], pl.out[k].get(), pl.out_n[k] * sizeof(double),
                                     cudaMemcpyDefault, s));
    if (read_scalar(pl.err.get(), s) != 0)
        throw FmmError(4, "tensor-core M2L: a wait for an MMA or operand barrier timed out");
}

}  // namespace
}  // namespace fmm2d

using namespace fmm2d;

FMM_EXPORT int fmm2d_b200_plan_create(int kernel, int nd, double eps, int ns,
                                      const double *sources, int ifcharge, int ifdipole,
                                      int ifpgh, int nt, const double *targ, int ifpghtarg,
                                      void **plan) {
    if (plan) *plan = nullptr;
    return guarded([&] {
        if (!plan) throw FmmError(4, "plan: null handle pointer");
        if (kernel != kLaplace && kernel != kCauchy)
            throw FmmError(4, "plan: kernel must be 0 (lfmm2d) or 1 (cfmm2d)");
        if (ns < 1 || nt < 0 || nd < 1 || (!ifcharge && !ifdipole) || !sources ||
            (nt > 0 && !targ) || ifpgh < 0 || ifpgh > 3 || ifpghtarg < 0 || ifpghtarg > 3)
            throw FmmError(4, "plan: invalid arguments");
        CallCtx ctx;  // device and memory-pool set-up
        Plan *pl = new Plan;
        try {
            pl->dev = ctx.device();
            FMM_CUDA(cudaStreamCreateWithFlags(&pl->s, cudaStreamNonBlocking));
            FmmCall &c = pl->shape;
            c.kernel = (Kernel)kernel;
            c.nd = nd;
            c.eps = eps;
            c.ns = ns;
            c.sources = sources;
            c.ifcharge = ifcharge;
            c.ifdipole = ifdipole;
            c.ifpgh = ifpgh;
            c.nt = nt;
            c.targ = targ;
            c.ifpghtarg = nt > 0 ? ifpghtarg : 0;
            c.precision = current_precision();
            laplace_geometry(c, on_device(sources), pl->s, pl->G);
            FMM_CUDA(cudaStreamSynchronize(pl->s));
            c.sources = nullptr;  // not kept: the plan holds its own copy
            c.targ = nullptr;
        } catch (...) {
            cudaStream_t st = pl->s;
            if (st) cudaStreamSynchronize(st);
            delete pl;
            if (st) {
                cudaStreamSynchronize(st);
                cudaStreamDestroy(st);
            }
            throw;
        }
        *plan = pl;
    });
}

FMM_EXPORT int fmm2d_b200_plan_eval(void *plan, const double *charge, const double *dipstr,
                                    const double *dipvec, double *pot, double *grad,
                                    double *hess, double *pottarg, double *gradtarg,
                                    double *hesstarg) {
    return guarded([&] {
        Plan *pl = static_cast<Plan *>(plan);
        if (!pl) throw FmmError(4, "plan: null handle");
        FmmCall c = pl->shape;
        if ((c.ifcharge && !charge) || (c.ifdipole && !dipstr) ||
            (c.ifdipole && c.kernel == kLaplace && !dipvec))
            throw FmmError(4, "plan: a strength array the plan was made for is missing");
        std::lock_guard<std::mutex> lock(pl->mu);
        CallCtx ctx;
        if (ctx.device() != pl->dev)
            throw FmmError(4, "plan: evaluated on another device than it was made on");
        c.charge = charge;
        c.dipstr = dipstr;
        c.dipvec = dipvec;
        c.pot = pot;
        c.grad = grad;
        c.hess = hess;
        c.pottarg = pottarg;
        c.gradtarg = gradtarg;
        c.hesstarg = hesstarg;
        const void *any = charge ? (const void *)charge : (const void *)dipstr;
        if (pl->warm && !pl->exec && !pl->graph_failed && graphs_enabled()) {
            // (the plan's stream follows the caller's: arrays the caller wrote
            // on its own stream are complete before the copies in)
            FMM_CUDA(cudaStreamSynchronize(ctx.stream()));
            try {
                build_graph(*pl);
            } catch (const FmmError &) {
                pl->graph_failed = true;  // eager evaluations from here on
                if (pl->exec) cudaGraphExecDestroy(pl->exec);
                pl->exec = nullptr;
            }
        }
        if (pl->exec && graphs_enabled()) {
            FMM_CUDA(cudaStreamSynchronize(ctx.stream()));
            const double *in[3] = {charge, dipstr, dipvec};
            double *out[6] = {pot, grad, hess, pottarg, gradtarg, hesstarg};
            replay(*pl, in, out);
            return;
        }
        laplace_evaluate(c, pl->G, on_device(any), ctx.stream(), &pl->cache, true);
        pl->warm = true;
    });
}

FMM_EXPORT int fmm2d_b200_plan_destroy(void *plan) {
    return guarded([&] {
        Plan *pl = static_cast<Plan *>(plan);
        if (!pl) return;
        cudaStream_t st = pl->s;
        FMM_CUDA(cudaStreamSynchronize(st));
        delete pl;  // buffers free on the plan's stream
        FMM_CUDA(cudaStreamSynchronize(st));
        FMM_CUDA(cudaStreamDestroy(st));
    });
}

// 1 when the plan's evaluations replay a captured CUDA graph, 0 when they
// run eagerly (first evaluation, graphs off, or a capture that failed).
FMM_EXPORT int fmm2d_b200_plan_uses_graph(void *plan) {
    Plan *pl = static_cast<Plan *>(plan);
    return (pl && pl->exec && graphs_enabled()) ? 1 : 0;
}
