// direct.cu -- FP64 direct sums on the device: every target against every
// source, the reference's public direct kernels l2d_direct{c,d,cd}{p,g,h}
// (complex-Laplace form, src/laplace/lapkernels2d.f) and
// c2d_direct{c,d,cd}{p,g,h} (Cauchy form, src/laplace/cauchykernels2d.f).
// Used to measure the FMM's error on sampled targets at full problem size.
//
// Work split: a grid of (target blocks) x (source chunks) x (densities).
// Each CTA stages its chunk's sources through shared memory in tiles and
// each thread owns one target; per-chunk partial sums go to a scratch
// array that a second kernel reduces in chunk order (deterministic) and
// adds into the outputs.  Splitting the sources keeps all 148 SMs busy
// when there are few targets (10^4 sampled targets against 10^7 sources).
#include "direct.cuh"
#include "runtime.cuh"

#include <algorithm>

namespace fmm2d {

namespace {

constexpr int kDThreads = 128;
constexpr int kDTile = 256;

// outputs per target and density: Laplace form pot, grad(2), hess(3);
// Cauchy form pot, grad, hess.
__host__ __device__ constexpr int nouts(int form, int pgh) {
    return form == kFormLaplace ? (pgh >= 3 ? 6 : (pgh >= 2 ? 3 : 1))
                                : (pgh >= 3 ? 3 : (pgh >= 2 ? 2 : 1));
}

template <int FORM, int PGH, bool IFC, bool IFD>
__global__ void __launch_bounds__(kDThreads) direct_partial_kernel(
    int ns, const double2 *__restrict__ src, const double2 *__restrict__ chg,
    const double2 *__restrict__ dip, const double *__restrict__ dv, int nd,
    int nt, const double2 *__restrict__ trg, int chunk, double th2, int strict,
    double2 *__restrict__ part) {
    __shared__ double2 s_pos[kDTile];
    __shared__ double2 s_q[kDTile];
    __shared__ double2 s_d[kDTile];
    __shared__ double2 s_v[kDTile];
    constexpr int NO = nouts(FORM, PGH);
    const int t = blockIdx.x * kDThreads + threadIdx.x;
    const int c = blockIdx.y, j = blockIdx.z;
    const int s0 = c * chunk, s1 = min(ns, s0 + chunk);
    const double2 x = t < nt ? trg[t] : make_double2(0.0, 0.0);
    double2 acc[NO];
#pragma unroll
    for (int o = 0; o < NO; o++) acc[o] = make_double2(0.0, 0.0);
    for (int b0 = s0; b0 < s1; b0 += kDTile) {
        const int nb = min(kDTile, s1 - b0);
        __syncthreads();
        for (int k = threadIdx.x; k < nb; k += kDThreads) {
            const size_t i = (size_t)(b0 + k);
            s_pos[k] = src[i];
            if (IFC) s_q[k] = chg[i * nd + j];
            if (IFD) {
                s_d[k] = dip[i * nd + j];
                if (FORM == kFormLaplace)
                    s_v[k] = make_double2(dv[(i * 2 + 0) * nd + j], dv[(i * 2 + 1) * nd + j]);
            }
        }
        __syncthreads();
        if (t >= nt) continue;
        for (int k = 0; k < nb; k++) {
            const double dx = x.x - s_pos[k].x, dy = x.y - s_pos[k].y;
            const double rr = dx * dx + dy * dy;
            if (strict ? (rr < th2) : (rr <= th2)) continue;
            const double ri = 1.0 / rr;
            if (FORM == kFormLaplace) {
                if (IFC) {
                    const double2 q = s_q[k];
                    const double lr = 0.5 * log(rr);
                    cfma(acc[0], q, make_double2(lr, 0.0));
                    if (PGH >= 2) {
                        cfma(acc[1], q, make_double2(dx * ri, 0.0));
                        cfma(acc[2], q, make_double2(dy * ri, 0.0));
                    }
                    if (PGH >= 3) {
                        const double r4 = ri * ri;
                        cfma(acc[3], q, make_double2((rr - 2 * dx * dx) * r4, 0.0));
                        cfma(acc[4], q, make_double2(-2 * dx * dy * r4, 0.0));
                        cfma(acc[5], q, make_double2((rr - 2 * dy * dy) * r4, 0.0));
                    }
                }
                if (IFD) {
                    const double2 d = s_d[k];
                    const double v1 = s_v[k].x, v2 = s_v[k].y;
                    const double sv = v1 * dx + v2 * dy;
                    cfma(acc[0], d, make_double2(-sv * ri, 0.0));
                    if (PGH >= 2) {
                        const double r4 = ri * ri;
                        cfma(acc[1], d, make_double2(-v1 * ri + 2 * dx * sv * r4, 0.0));
                        cfma(acc[2], d, make_double2(-v2 * ri + 2 * dy * sv * r4, 0.0));
                        if (PGH >= 3) {
                            const double r6 = r4 * ri;
                            cfma(acc[3], d, make_double2((4 * v1 * dx + 2 * sv) * r4 - 8 * dx * dx * sv * r6, 0.0));
                            cfma(acc[4], d, make_double2((2 * v1 * dy + 2 * v2 * dx) * r4 - 8 * dx * dy * sv * r6, 0.0));
                            cfma(acc[5], d, make_double2((4 * v2 * dy + 2 * sv) * r4 - 8 * dy * dy * sv * r6, 0.0));
                        }
                    }
                }
            } else {
                const double2 zi = make_double2(dx * ri, -dy * ri);
                const double2 zi2 = cmul(zi, zi);
                if (IFC) {
                    const double2 q = s_q[k];
                    cfma(acc[0], q, make_double2(0.5 * log(rr), 0.0));
                    if (PGH >= 2) cfma(acc[1], q, zi);
                    if (PGH >= 3) cfma(acc[2], q, cscal(zi2, -1.0));
                }
                if (IFD) {
                    const double2 d = s_d[k];
                    cfma(acc[0], d, zi);
                    if (PGH >= 2) cfma(acc[1], d, cscal(zi2, -1.0));
                    if (PGH >= 3) cfma(acc[2], d, cscal(cmul(zi2, zi), 2.0));
                }
            }
        }
    }
    if (t < nt) {
        double2 *p = part + (((size_t)c * nd + j) * nt + t) * NO;
#pragma unroll
        for (int o = 0; o < NO; o++) p[o] = acc[o];
    }
}

// Sums the chunk partials in chunk order and adds them into the outputs
// (pot(nd,nt); grad(nd,2,nt) / hess(nd,3,nt) in the Laplace form,
// grad(nd,nt) / hess(nd,nt) in the Cauchy form).
__global__ void direct_reduce_kernel(int form, int pgh, int nd, int nt,
                                     int nchunk,
                                     const double2 *__restrict__ part,
                                     double2 *pot, double2 *grad,
                                     double2 *hess) {
    const int no = nouts(form, pgh);
    const int64_t n = (int64_t)nt * nd;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(e / nd), j = (int)(e % nd);
        double2 acc[6];
        for (int o = 0; o < no; o++) acc[o] = make_double2(0.0, 0.0);
        for (int c = 0; c < nchunk; c++) {
            const double2 *p = part + (((size_t)c * nd + j) * nt + t) * no;
            for (int o = 0; o < no; o++) acc[o] = cadd(acc[o], p[o]);
        }
        pot[(size_t)t * nd + j] = cadd(pot[(size_t)t * nd + j], acc[0]);
        if (form == kFormLaplace) {
            if (pgh >= 2)
                for (int q = 0; q < 2; q++) {
                    double2 &g = grad[((size_t)t * 2 + q) * nd + j];
                    g = cadd(g, acc[1 + q]);
                }
            if (pgh >= 3)
                for (int q = 0; q < 3; q++) {
                    double2 &h = hess[((size_t)t * 3 + q) * nd + j];
                    h = cadd(h, acc[3 + q]);
                }
        } else {
            if (pgh >= 2) grad[(size_t)t * nd + j] = cadd(grad[(size_t)t * nd + j], acc[1]);
            if (pgh >= 3) hess[(size_t)t * nd + j] = cadd(hess[(size_t)t * nd + j], acc[2]);
        }
    }
}

template <int FORM, int PGH>
void launch_partial(const DirectArgs &a, int chunk, int nchunk, double2 *part,
                    cudaStream_t s) {
    dim3 grid((a.nt + kDThreads - 1) / kDThreads, nchunk, a.nd);
    const double th2 = a.thresh * a.thresh;
#define FMM_DIRECT_CASE(IFC, IFD)                                              \
    direct_partial_kernel<FORM, PGH, IFC, IFD><<<grid, kDThreads, 0, s>>>(     \
        a.ns, a.src, a.chg, a.dip, a.dv, a.nd, a.nt, a.trg, chunk, th2,       \
        a.strict, part)
    if (a.ifcharge && a.ifdipole)
        FMM_DIRECT_CASE(true, true);
    else if (a.ifcharge)
        FMM_DIRECT_CASE(true, false);
    else
        FMM_DIRECT_CASE(false, true);
#undef FMM_DIRECT_CASE
    FMM_CHECK_LAUNCH();
}

}  // namespace

int direct_outputs(int form, int pgh) { return nouts(form, pgh); }

void check_direct_arrays(int form, const void *sources, int ifcharge,
                         const void *charge, int ifdipole, const void *dipstr,
                         const void *dipvec, const void *targ, int ifpgh,
                         const void *pot, const void *grad, const void *hess) {
    const char *missing = nullptr;
    if (!sources) missing = "sources";
    else if (!targ) missing = "targ";
    else if (!pot) missing = "pot";
    else if (ifcharge && !charge) missing = "charge";
    else if (ifdipole && !dipstr) missing = "dipstr";
    else if (ifdipole && form == kFormLaplace && !dipvec) missing = "dipvec";
    else if (ifpgh >= 2 && !grad) missing = "grad";
    else if (ifpgh >= 3 && !hess) missing = "hess";
    if (missing)
        throw FmmError(4, std::string("direct sum: ") + missing +
                              " is NULL but the flags require it");
}

int direct_chunks(int ns, int nt, int nd) {
    const int tblocks = (nt + kDThreads - 1) / kDThreads;
    int want = (4 * kNumSM + tblocks * nd - 1) / std::max(1, tblocks * nd);
    int maxc = std::max(1, ns / 1024);
    return std::max(1, std::min(want, maxc));
}

void direct_sum(const DirectArgs &a, double2 *part, int nchunk,
                cudaStream_t s) {
    if (a.nt <= 0 || a.ns <= 0) return;
    const int chunk = (a.ns + nchunk - 1) / nchunk;
    if (a.form == kFormLaplace) {
        if (a.pgh == 1) launch_partial<kFormLaplace, 1>(a, chunk, nchunk, part, s);
        if (a.pgh == 2) launch_partial<kFormLaplace, 2>(a, chunk, nchunk, part, s);
        if (a.pgh == 3) launch_partial<kFormLaplace, 3>(a, chunk, nchunk, part, s);
    } else {
        if (a.pgh == 1) launch_partial<kFormCauchy, 1>(a, chunk, nchunk, part, s);
        if (a.pgh == 2) launch_partial<kFormCauchy, 2>(a, chunk, nchunk, part, s);
        if (a.pgh == 3) launch_partial<kFormCauchy, 3>(a, chunk, nchunk, part, s);
    }
    const int64_t n = (int64_t)a.nt * a.nd;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, kNumSM * 8);
    direct_reduce_kernel<<<blocks, 256, 0, s>>>(a.form, a.pgh, a.nd, a.nt,
                                                nchunk, part, a.pot, a.grad,
                                                a.hess);
    FMM_CHECK_LAUNCH();
}

namespace {

bool dev_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// Host-or-device staging for the allocating entry points.
struct Staged {
    DevBuf<double2> own;
    double2 *ptr = nullptr;
    void in(const void *u, size_t n, bool on_dev, cudaStream_t s) {
        if (!u || !n) return;
        if (on_dev) {
            ptr = (double2 *)u;
            return;
        }
        own.alloc(n, s);
        FMM_CUDA(cudaMemcpyAsync(own.get(), u, n * sizeof(double2),
                                 cudaMemcpyHostToDevice, s));
        ptr = own.get();
    }
    void out(void *u, size_t n, bool on_dev, cudaStream_t s) {
        if (u && n && !on_dev)
            FMM_CUDA(cudaMemcpyAsync(u, ptr, n * sizeof(double2),
                                     cudaMemcpyDeviceToHost, s));
    }
};

int run_direct(int form, int nd, int ns, const double *sources, int ifcharge,
               const double *charge, int ifdipole, const double *dipstr,
               const double *dipvec, int nt, const double *targ, int ifpgh,
               double *pot, double *grad, double *hess, double thresh) {
    return guarded([&] {
        if (nd < 1 || ns < 0 || nt < 0 || ifpgh < 1 || ifpgh > 3 ||
            (!ifcharge && !ifdipole))
            throw FmmError(4, "invalid direct-sum arguments");
        if (nt == 0 || ns == 0) return;
        check_direct_arrays(form, sources, ifcharge, charge, ifdipole, dipstr,
                            dipvec, targ, ifpgh, pot, grad, hess);
        CallCtx ctx;
        cudaStream_t s = ctx.stream();
        const bool od = dev_ptr(sources);
        {
            // Every array the flags use must live where `sources` lives: a
            // device kernel given a host pointer, or a host copy given a
            // device pointer, would fault.
            const void *used[] = {targ, pot, ifcharge ? charge : nullptr,
                                  ifdipole ? dipstr : nullptr,
                                  (ifdipole && form == kFormLaplace) ? dipvec : nullptr,
                                  ifpgh >= 2 ? grad : nullptr,
                                  ifpgh >= 3 ? hess : nullptr};
            for (const void *p : used)
                if (p && dev_ptr(p) != od)
                    throw FmmError(4, "direct sum: arrays mix host and device memory");
        }
        const int gc = form == kFormLaplace ? 2 : 1, hc = form == kFormLaplace ? 3 : 1;
        Staged S, T, Q, D, V, Po, G, H;
        S.in(sources, ns, od, s);
        T.in(targ, nt, od, s);
        if (ifcharge) Q.in(charge, (size_t)nd * ns, od, s);
        if (ifdipole) {
            D.in(dipstr, (size_t)nd * ns, od, s);
            if (form == kFormLaplace) V.in(dipvec, (size_t)nd * ns, od, s);
        }
        Po.in(pot, (size_t)nd * nt, od, s);
        if (ifpgh >= 2) G.in(grad, (size_t)nd * gc * nt, od, s);
        if (ifpgh >= 3) H.in(hess, (size_t)nd * hc * nt, od, s);
        DirectArgs a;
        a.form = form;
        a.nd = nd;
        a.ns = ns;
        a.src = S.ptr;
        a.ifcharge = ifcharge;
        a.chg = Q.ptr;
        a.ifdipole = ifdipole;
        a.dip = D.ptr;
        a.dv = (const double *)V.ptr;
        a.nt = nt;
        a.trg = T.ptr;
        a.pgh = ifpgh;
        a.pot = Po.ptr;
        a.grad = G.ptr;
        a.hess = H.ptr;
        a.thresh = thresh;
        a.strict = direct_strict(form, ifcharge, ifdipole, ifpgh);
        const int nchunk = direct_chunks(ns, nt, nd);
        DevBuf<double2> part((size_t)nchunk * nd * nt * nouts(form, ifpgh), s);
        direct_sum(a, part.get(), nchunk, s);
        Po.out(pot, (size_t)nd * nt, od, s);
        if (ifpgh >= 2) G.out(grad, (size_t)nd * gc * nt, od, s);
        if (ifpgh >= 3) H.out(hess, (size_t)nd * hc * nt, od, s);
        FMM_CUDA(cudaStreamSynchronize(s));
    });
}

}  // namespace

// Threshold rule of the reference kernels: pairs with |z|^2 < thresh^2 are
// skipped by l2d_directc{g,h}, l2d_directcd{g,h} and every Cauchy g/h kernel;
// all others skip |z|^2 <= thresh^2 (lapkernels2d.c, cauchykernels2d.c).
int direct_strict(int form, int ifcharge, int ifdipole, int pgh) {
    if (form == kFormLaplace) return (ifcharge && pgh >= 2) ? 1 : 0;
    (void)ifdipole;
    return pgh >= 2 ? 1 : 0;
}

}  // namespace fmm2d

using namespace fmm2d;

// Complex-Laplace direct sum (l2d_direct*, src/laplace/lapkernels2d.f):
// increments pot(nd,nt), grad(nd,2,nt), hess(nd,3,nt) at the targets.
// Arrays: sources(2,ns), charge/dipstr(nd,ns) complex, dipvec(nd,2,ns);
// host or device memory.  Returns 0 or 4.
FMM_EXPORT int fmm2d_b200_l2d_direct(int nd, int ns, const double *sources,
                                     int ifcharge, const double *charge,
                                     int ifdipole, const double *dipstr,
                                     const double *dipvec, int nt,
                                     const double *targ, int ifpgh,
                                     double *pot, double *grad, double *hess,
                                     double thresh) {
    return run_direct(kFormLaplace, nd, ns, sources, ifcharge, charge,
                      ifdipole, dipstr, dipvec, nt, targ, ifpgh, pot, grad,
                      hess, thresh);
}

// Cauchy direct sum (c2d_direct*, src/laplace/cauchykernels2d.f):
// increments pot(nd,nt), grad(nd,nt), hess(nd,nt).
FMM_EXPORT int fmm2d_b200_c2d_direct(int nd, int ns, const double *sources,
                                     int ifcharge, const double *charge,
                                     int ifdipole, const double *dipstr, int nt,
                                     const double *targ, int ifpgh, double *pot,
                                     double *grad, double *hess,
                                     double thresh) {
    return run_direct(kFormCauchy, nd, ns, sources, ifcharge, charge, ifdipole,
                      dipstr, nullptr, nt, targ, ifpgh, pot, grad, hess,
                      thresh);
}
