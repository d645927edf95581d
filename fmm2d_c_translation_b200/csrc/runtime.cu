// runtime.cu -- call context, device pool set-up and the library-level
// C entry points that are not FMM evaluations (version, errors, memory,
// tree inspection).
#include "runtime.cuh"
#include "tree.cuh"

#include <mutex>
#include <string.h>

namespace fmm2d {

namespace {
std::mutex g_pool_mu;
bool g_pool_ready[64];

void ensure_pool(int dev) {
    std::lock_guard<std::mutex> g(g_pool_mu);
    if (dev < 0 || dev >= 64 || g_pool_ready[dev]) return;
    cudaMemPool_t pool;
    FMM_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t thr = UINT64_MAX;
    FMM_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    g_pool_ready[dev] = true;
}
}  // namespace

// One non-blocking stream per (host thread, device), created on first use and
// kept for the life of the thread, so that buffers owned by long-lived
// objects (tree handles) always free on a live stream.
namespace {
thread_local cudaStream_t g_user_stream = nullptr;
thread_local bool g_user_stream_set = false;
}  // namespace

CallCtx::CallCtx() : dev_(0), s_(nullptr) {
    static thread_local cudaStream_t streams[64];
    FMM_CUDA(cudaGetDevice(&dev_));
    if (dev_ < 0 || dev_ >= 64) throw FmmError(4, "device index out of range");
    ensure_pool(dev_);
    if (g_user_stream_set) {
        s_ = g_user_stream;
        return;
    }
    if (!streams[dev_])
        FMM_CUDA(cudaStreamCreateWithFlags(&streams[dev_], cudaStreamNonBlocking));
    s_ = streams[dev_];
}

cudaStream_t CallCtx::copy_stream() const {
    static thread_local cudaStream_t streams[64];
    if (!streams[dev_])
        FMM_CUDA(cudaStreamCreateWithFlags(&streams[dev_], cudaStreamNonBlocking));
    return streams[dev_];
}

void set_user_stream(cudaStream_t s, bool on) {
    g_user_stream = s;
    g_user_stream_set = on;
}

CallCtx::~CallCtx() {
    if (s_) cudaStreamSynchronize(s_);
}

}  // namespace fmm2d

using namespace fmm2d;

// ---------------------------------------------------------------------------
// Library information and housekeeping.
// ---------------------------------------------------------------------------
FMM_EXPORT const char *fmm2d_b200_version(void) { return "fmm2d-b200 0.1"; }

// Copies the message of the last failed call (any thread) into buf.
FMM_EXPORT int fmm2d_b200_last_error(char *buf, int len) {
    std::string m = get_last_error();
    if (buf && len > 0) {
        strncpy(buf, m.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return (int)m.size();
}

// Makes the calling thread's subsequent calls run on `stream` (a
// cudaStream_t of the current device; 0 = legacy default stream).  Calls
// still return only after their work on that stream has completed.
FMM_EXPORT int fmm2d_b200_set_stream(void *stream) {
    set_user_stream((cudaStream_t)stream, true);
    return 0;
}

// Back to the library's own per-thread stream.
FMM_EXPORT int fmm2d_b200_reset_stream(void) {
    set_user_stream(nullptr, false);
    return 0;
}

// Number of kernels the library has launched in this process.
FMM_EXPORT unsigned long long fmm2d_b200_launch_count(void) { return launch_count(); }

// Phase profiling of subsequent calls (CUDA events on the call's stream).
FMM_EXPORT int fmm2d_b200_set_profiling(int on) {
    set_profiling(on);
    return 0;
}

// "phase=ms;...;#count=value;" of the last profiled call on this thread.
FMM_EXPORT int fmm2d_b200_last_profile(char *buf, int len) {
    std::string m = prof_report();
    if (buf && len > 0) {
        strncpy(buf, m.c_str(), (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return (int)m.size();
}

// Failure injection for the failure tests (host side only; no GPU fault):
// the nth device allocation from now fails as out of memory (0: off).
FMM_EXPORT int fmm2d_b200_inject_alloc_failure(long long nth) {
    inject_alloc_failure(nth);
    return 0;
}

// Failure injection: the tensor-core M2L kernels issue no MMAs and their
// bounded waits give up after wait_ms (on = 0 restores the normal 2 s limit),
// so the evaluation returns ier = 4.
FMM_EXPORT int fmm2d_b200_inject_tc_stall(int on, double wait_ms) {
    const double ns = wait_ms > 0 ? wait_ms * 1e6 : 1e6;
    inject_tc_stall(on, (unsigned long long)ns);
    return 0;
}

// Bytes of the current device's memory pool held by live allocations of
// this process (cudaMemPoolAttrUsedMemCurrent): the same before and after a
// call, failed or not, when the call released everything it allocated.
FMM_EXPORT int fmm2d_b200_device_bytes_in_use(unsigned long long *bytes) {
    return guarded([&] {
        int dev;
        FMM_CUDA(cudaGetDevice(&dev));
        cudaMemPool_t pool;
        FMM_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
        uint64_t v = 0;
        FMM_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &v));
        *bytes = (unsigned long long)v;
    });
}

// Returns cached device workspace of the current device to the driver.
FMM_EXPORT int fmm2d_b200_release_memory(void) {
    return guarded([&] {
        int dev;
        FMM_CUDA(cudaGetDevice(&dev));
        FMM_CUDA(cudaDeviceSynchronize());
        cudaMemPool_t pool;
        FMM_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
        FMM_CUDA(cudaMemPoolTrimTo(pool, 0));
    });
}

// ---------------------------------------------------------------------------
// Tree inspection: builds the quadtree of a point set on the device and
// exposes it in the reference's layout (pts_tree_mem / pts_tree_build /
// pts_tree_sort, src/common/pts_tree2d.f:34,406,1222) plus the lists of
// computelists (src/common/tree_routs2d.f:486).
// ---------------------------------------------------------------------------
struct TreeHandle {
    Tree T;
    int ns = 0, nt = 0;
    bool lists = false;
};

FMM_EXPORT int fmm2d_b200_tree_build(const double *sources, int ns,
                                     const double *targ, int nt, int ndiv,
                                     int idivflag, void **handle) {
    *handle = nullptr;
    return guarded([&] {
        if (ns < 0 || nt < 0 || ns + nt < 1)
            throw FmmError(4, "tree needs at least one point");
        CallCtx ctx;
        cudaStream_t s = ctx.stream();
        DevBuf<double2> ds(std::max(ns, 1), s), dt(std::max(nt, 1), s);
        if (ns)
            FMM_CUDA(cudaMemcpyAsync(ds.get(), sources, sizeof(double2) * ns,
                                     cudaMemcpyHostToDevice, s));
        if (nt)
            FMM_CUDA(cudaMemcpyAsync(dt.get(), targ, sizeof(double2) * nt,
                                     cudaMemcpyHostToDevice, s));
        TreeHandle *h = new TreeHandle();
        try {
            build_tree(ds.get(), ns, dt.get(), nt, ndiv, idivflag, kMaxLevels,
                       s, h->T);
            compute_lists(h->T, s);
            h->lists = true;
            h->ns = ns;
            h->nt = nt;
            FMM_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            delete h;
            throw;
        }
        *handle = h;
    });
}

FMM_EXPORT int fmm2d_b200_tree_sizes(void *handle, int *nlevels, int *nboxes,
                                     int *ltree) {
    TreeHandle *h = (TreeHandle *)handle;
    *nlevels = h->T.nlevels;
    *nboxes = h->T.nboxes;
    *ltree = 17 * h->T.nboxes + 2 * (h->T.nlevels + 1);
    return 0;
}

FMM_EXPORT int fmm2d_b200_tree_export(void *handle, int *itree, int *iptr,
                                      double *centers, double *boxsize,
                                      int *isrc, int *isrcse, int *itarg,
                                      int *itargse) {
    TreeHandle *h = (TreeHandle *)handle;
    return guarded([&] {
        CallCtx ctx;
        export_reference_tree(h->T, h->ns, h->nt, itree, iptr, centers,
                              boxsize, isrc, isrcse, itarg, itargse,
                              ctx.stream());
    });
}

// Lists in the reference's layout: nlist_k(nboxes), list_k(mnlist_k, nboxes),
// 1-based box numbers, mnlist = 13 / 27 / 20 / 5.
FMM_EXPORT int fmm2d_b200_tree_lists(void *handle, int *nlist1, int *list1,
                                     int *nlist2, int *list2, int *nlist3,
                                     int *list3, int *nlist4, int *list4) {
    TreeHandle *h = (TreeHandle *)handle;
    return guarded([&] {
        CallCtx ctx;
        cudaStream_t s = ctx.stream();
        const Tree &T = h->T;
        const int nb = T.nboxes;
        struct L {
            const DevBuf<int> *n, *l;
            int *hn, *hl, m;
        } ls[4] = {{&T.nlist1, &T.list1, nlist1, list1, kMaxList1},
                   {&T.nlist2, &T.list2, nlist2, list2, kMaxList2},
                   {&T.nlist3, &T.list3, nlist3, list3, kMaxList3},
                   {&T.nlist4, &T.list4, nlist4, list4, kMaxList4}};
        for (auto &x : ls) {
            FMM_CUDA(cudaMemcpyAsync(x.hn, x.n->get(), sizeof(int) * nb,
                                     cudaMemcpyDeviceToHost, s));
            FMM_CUDA(cudaMemcpyAsync(x.hl, x.l->get(), sizeof(int) * nb * x.m,
                                     cudaMemcpyDeviceToHost, s));
        }
        FMM_CUDA(cudaStreamSynchronize(s));
        for (auto &x : ls)
            for (int b = 0; b < nb; b++)
                for (int k = 0; k < x.m; k++) {
                    int &v = x.hl[(size_t)b * x.m + k];
                    v = k < x.hn[b] ? v + 1 : 0;
                }
    });
}

FMM_EXPORT void fmm2d_b200_tree_free(void *handle) {
    TreeHandle *h = (TreeHandle *)handle;
    if (!h) return;
    try {
        CallCtx ctx;
        delete h;
    } catch (...) {
    }
}
