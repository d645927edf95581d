// plan.cu -- resident geometry for repeated Laplace / Cauchy evaluations.
//
// A plan keeps on the device what a call derives from the points alone:
// the adaptive tree, its interaction lists and the points in tree order.
// Each evaluation then only gathers the new strengths, runs the FMM passes
// and scatters the outputs -- the pattern of an iterative solver that
// applies the same boundary-integral operator to a new density every step.
// The plan owns a stream of its own for its buffers, so it may be
// destroyed from any thread; evaluations run on the calling thread's
// stream (or the one set with fmm2d_b200_set_stream).
#include "engine.cuh"
#include "runtime.cuh"

namespace fmm2d {
namespace {

struct Plan {
    int dev = 0;
    cudaStream_t s = nullptr;
    FmmCall shape;
    LapGeometry G;
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
            if (pl->s) {
                cudaStream_t st = pl->s;
                cudaStreamSynchronize(st);
                delete pl;
                cudaStreamSynchronize(st);
                cudaStreamDestroy(st);
            } else {
                delete pl;
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
        laplace_evaluate(c, pl->G, on_device(any), ctx.stream());
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
