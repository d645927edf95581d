// noalloc.cu -- the complex-Laplace direct sum in a form that allocates no
// device memory.
//
// Some callers cannot allocate device memory themselves or let a library
// do it: a host application whose GPU memory is owned by another allocator
// or by a fixed budget reserved up front (so an extra cudaMalloc either
// fails or breaks the budget), or a latency-critical caller for which an
// allocation call, which may synchronize the device, is not acceptable.
// fmm2d_b200_l2d_direct allocates scratch for its per-chunk partial sums;
// fmm2d_b200_l2d_direct_noalloc computes the same sums with that scratch in
// the file-scope device array below instead.
//
// Limits and rules of the no-allocation form:
//  * The scratch holds 262144 complex values (4 MiB).  A call needs
//    nd * nt * k values per source chunk, k = 1 (pot), 3 (+grad) or
//    6 (+hess); a call whose nd * nt * k exceeds the capacity is rejected
//    with ier = 4 and a message, and otherwise the number of source chunks
//    is reduced to fit.
//  * Every GPU that loads this library holds the 4 MiB array until the
//    process exits.
//  * The first call on a device looks up the array's device address (with
//    that device current) and keeps it; make that first call before any
//    stream capture begins.
//  * All arrays must be device memory of the current device; host arrays,
//    arrays of another device and NULL arrays that the flags require are
//    rejected with ier = 4 before any GPU work (copying host arrays would
//    need device memory).
//  * The scratch address is looked up once per device and kept for the life
//    of the process: do not call this entry point on a device after
//    cudaDeviceReset (or any other teardown of its primary context) in the
//    same process, since the kept address then no longer names the array.
//  * Every call on a device shares the one array.  A call first writes every
//    scratch value it later reads, so what a previous call left behind is
//    never read; but calls whose work overlaps on the GPU (for example from
//    two host threads, or on two streams) race on the array and must not
//    be issued.
//  * The call runs on `stream` (a cudaStream_t, 0 for the legacy default
//    stream) and returns after that stream has finished it.
#include "direct.cuh"
#include "runtime.cuh"

#include <mutex>

namespace fmm2d {
namespace {

constexpr size_t kNoAllocScratchValues = (size_t)1 << 18;  // 4 MiB of double2

static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocScratchValues];

std::mutex g_noalloc_mu;
double2 *g_noalloc_addr[64];

// Device address of g_noalloc_scratch on `dev` (the current device), looked
// up once per device.  In host code the array's name is only a host-side
// handle, never a device address.
double2 *noalloc_scratch(int dev) {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            throw FmmError(4, std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                                  cudaGetErrorString(e));
        }
        g_noalloc_addr[dev] = static_cast<double2 *>(p);
    }
    return g_noalloc_addr[dev];
}

// True when p is device (or managed) memory that device `dev` owns.
bool on_device(const void *p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace
}  // namespace fmm2d

using namespace fmm2d;

// Same arguments and results as fmm2d_b200_l2d_direct, plus the stream to run
// on; allocates no device memory (see the rules at the top of this file).
FMM_EXPORT int fmm2d_b200_l2d_direct_noalloc(
    int nd, int ns, const double *sources, int ifcharge, const double *charge,
    int ifdipole, const double *dipstr, const double *dipvec, int nt,
    const double *targ, int ifpgh, double *pot, double *grad, double *hess,
    double thresh, void *stream) {
    return guarded([&] {
        if (nd < 1 || ns < 0 || nt < 0 || ifpgh < 1 || ifpgh > 3 ||
            (!ifcharge && !ifdipole))
            throw FmmError(4, "invalid direct-sum arguments");
        if (nt == 0 || ns == 0) return;
        check_direct_arrays(kFormLaplace, sources, ifcharge, charge, ifdipole,
                            dipstr, dipvec, targ, ifpgh, pot, grad, hess);
        const int nout = direct_outputs(kFormLaplace, ifpgh);
        const size_t per_chunk = (size_t)nd * nt * nout;
        if (per_chunk > kNoAllocScratchValues)
            throw FmmError(4, "nd * nt * outputs = " + std::to_string(per_chunk) +
                                  " exceeds the no-allocation scratch of " +
                                  std::to_string(kNoAllocScratchValues) +
                                  " complex values");
        const void *arrays[] = {sources, targ, pot, ifcharge ? charge : nullptr,
                                ifdipole ? dipstr : nullptr,
                                ifdipole ? dipvec : nullptr,
                                ifpgh >= 2 ? grad : nullptr,
                                ifpgh >= 3 ? hess : nullptr};
        int dev = 0;
        FMM_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64) throw FmmError(4, "device index out of range");
        for (const void *p : arrays)
            if (p && !on_device(p, dev))
                throw FmmError(4, "the no-allocation entry point takes device arrays "
                                  "of the current device only");
        double2 *scratch = noalloc_scratch(dev);
        int nchunk = direct_chunks(ns, nt, nd);
        const int cap = (int)(kNoAllocScratchValues / per_chunk);
        if (nchunk > cap) nchunk = cap;
        DirectArgs a;
        a.form = kFormLaplace;
        a.nd = nd;
        a.ns = ns;
        a.src = (const double2 *)sources;
        a.ifcharge = ifcharge;
        a.chg = (const double2 *)charge;
        a.ifdipole = ifdipole;
        a.dip = (const double2 *)dipstr;
        a.dv = dipvec;
        a.nt = nt;
        a.trg = (const double2 *)targ;
        a.pgh = ifpgh;
        a.pot = (double2 *)pot;
        a.grad = (double2 *)grad;
        a.hess = (double2 *)hess;
        a.thresh = thresh;
        a.strict = direct_strict(kFormLaplace, ifcharge, ifdipole, ifpgh);
        cudaStream_t s = (cudaStream_t)stream;
        direct_sum(a, scratch, nchunk, s);
        FMM_CUDA(cudaStreamSynchronize(s));
    });
}
