// capi.cu -- the drop-in C ABI: the reference's gfortran-convention entry
// points (lowercase name + '_', every argument by pointer, integer = int32,
// complex*16 = interleaved doubles, column-major arrays) plus the one
// bind(c) Helmholtz entry of include/fmm2d/helmholtz.h.
//
//   lfmm2d_{s,t,st}_{c,d,cd}_{p,g,h}_   src/laplace/lfmm2dwrap.f:31-1704
//   cfmm2d_{s,t,st}_{c,d,cd}_{p,g,h}_   src/laplace/cfmm2dwrap.f:31-1659
//   hfmm2d_{s,t,st}_{c,d,cd}_{p,g,h}_   src/helmholtz/hfmm2dwrap.f:41-1871
//   rfmm2d_{s,t,st}_{c,d,cd}_{p,g,h}_   src/laplace/rfmm2dwrap.f:36-1709
//   {l,c,h,r}fmm2d_*_vec_               the *wrap_vec.f files (leading nd)
//   lfmm2d_ / cfmm2d_ / hfmm2d_ / rfmm2d_   guru drivers (lfmm2d.f:29,
//                                       cfmm2d.f:23, hfmm2d.f:19, rfmm2d.f:27)
//   {l,c,h,r}fmm2d_ndiv_                MATLAB-path drivers
//   hfmm2d_s_c_p                        src/helmholtz_c.f03:5-15
//
// Each wrapper fixes ifcharge / ifdipole / ifpgh / ifpghtarg with nd = 1,
// nt = 0 for the sources-only forms and ifpgh = 0 for the targets-only
// forms, exactly as the Fortran wrappers do, and runs the evaluation on
// the GPU.  Arrays may be host or device memory (see engine.cuh).
#include <stdint.h>

#include "engine.cuh"
#include "hankel.cuh"
#include "helmholtz.cuh"
#include "runtime.cuh"

using namespace fmm2d;

typedef int32_t fint;

namespace {

FmmCall base_call(Kernel k, const double *eps, const double *zk, const fint *ns,
                  const double *src) {
    FmmCall c;
    c.kernel = k;
    c.eps = *eps;
    if (zk) {
        c.zk[0] = zk[0];
        c.zk[1] = zk[1];
    }
    c.ns = *ns;
    c.sources = src;
    c.precision = current_precision();
    return c;
}

void wrap(Kernel k, int nd, const double *eps, const double *zk, const fint *ns,
          const double *src, const double *chg, const double *dip,
          const double *dv, int ifc, int ifd, int pgh, double *pot,
          double *grad, double *hess, int nt, const double *targ, int pght,
          double *pt, double *gt, double *ht, fint *ier) {
    FmmCall c = base_call(k, eps, zk, ns, src);
    c.nd = nd;
    c.ifcharge = ifc;
    c.charge = chg;
    c.ifdipole = ifd;
    c.dipstr = dip;
    c.dipvec = dv;
    c.ifpgh = pgh;
    c.pot = pot;
    c.grad = grad;
    c.hess = hess;
    c.nt = nt;
    c.targ = targ;
    c.ifpghtarg = pght;
    c.pottarg = pt;
    c.gradtarg = gt;
    c.hesstarg = ht;
    *ier = run_fmm(c);
}

}  // namespace

// Complex*16 arrays are passed as interleaved doubles, real*8 arrays as
// doubles: every array argument is a double pointer in the C ABI.
typedef double arr_t;

// source-strength argument lists: c = charge, d = dipole, cd = both
#define SRC_c(V) const arr_t *charge
#define SRC_d(V) const arr_t *dipstr V(const double *dipvec)
#define SRC_cd(V) const arr_t *charge, const arr_t *dipstr V(const double *dipvec)
#define PASS_c charge, nullptr, nullptr, 1, 0
#define PASS_d nullptr, dipstr, DV(dipvec), 0, 1
#define PASS_cd charge, dipstr, DV(dipvec), 1, 1
#define OUT_S_p arr_t *pot
#define OUT_S_g arr_t *pot, arr_t *grad
#define OUT_S_h arr_t *pot, arr_t *grad, arr_t *hess
#define OUT_T_p arr_t *pottarg
#define OUT_T_g arr_t *pottarg, arr_t *gradtarg
#define OUT_T_h arr_t *pottarg, arr_t *gradtarg, arr_t *hesstarg
#define PS_p 1, pot, nullptr, nullptr
#define PS_g 2, pot, grad, nullptr
#define PS_h 3, pot, grad, hess
#define PT_p 1, pottarg, nullptr, nullptr
#define PT_g 2, pottarg, gradtarg, nullptr
#define PT_h 3, pottarg, gradtarg, hesstarg
#define WITH_DV(x) , x
#define NO_DV(x)
#define ND_ARG() const fint *nd,
#define ZK_ARG() const arr_t *zk,
#define NONE()

// The three wrappers (sources only, targets only, both) of one strength
// kind K and output level P of a family: NAME prefix, SUF "_" or "_vec_",
// kernel KERN, NDP/NDA the nd argument (the _vec forms) or nd = 1, ZKP/ZKA
// the wavenumber argument (Helmholtz), DVM whether dipoles carry dipvec.
#define WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, K, P)                        \
    FMM_EXPORT void NAME##_s_##K##_##P##SUF(NDP() const double *eps, ZKP() const fint *ns, \
                                            const double *sources, SRC_##K(DVM),       \
                                            OUT_S_##P, fint *ier) {                    \
        wrap(KERN, NDA, eps, ZKA, ns, sources, PASS_##K, PS_##P, 0, nullptr, 0,      \
             nullptr, nullptr, nullptr, ier);                                        \
    }                                                                                \
    FMM_EXPORT void NAME##_t_##K##_##P##SUF(                                         \
        NDP() const double *eps, ZKP() const fint *ns, const double *sources,        \
        SRC_##K(DVM), const fint *nt, const double *targ, OUT_T_##P, fint *ier) {    \
        wrap(KERN, NDA, eps, ZKA, ns, sources, PASS_##K, 0, nullptr, nullptr,        \
             nullptr, *nt, targ, PT_##P, ier);                                       \
    }                                                                                \
    FMM_EXPORT void NAME##_st_##K##_##P##SUF(                                        \
        NDP() const double *eps, ZKP() const fint *ns, const double *sources,        \
        SRC_##K(DVM), OUT_S_##P, const fint *nt, const double *targ, OUT_T_##P,      \
        fint *ier) {                                                                 \
        wrap(KERN, NDA, eps, ZKA, ns, sources, PASS_##K, PS_##P, *nt, targ, PT_##P,  \
             ier);                                                                   \
    }

// All 27 (strength kind x output level) of a family.
#define WRAP27(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM)                \
    WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, c, p)               \
    WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, c, g)               \
    WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, c, h)               \
    WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, d, p)               \
    WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, d, g)               \
    WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, d, h)               \
    WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, cd, p)              \
    WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, cd, g)              \
    WRAP3(NAME, SUF, KERN, NDP, NDA, ZKP, ZKA, DVM, cd, h)

#define DV(x) x
// lfmm2d_*_ (src/laplace/lfmm2dwrap.f:31-1704), lfmm2d_*_vec_
// (src/laplace/lfmm2dwrap_vec.f:31-1685)
WRAP27(lfmm2d, _, kLaplace, NONE, 1, NONE, nullptr, WITH_DV)
WRAP27(lfmm2d, _vec_, kLaplace, ND_ARG, *nd, NONE, nullptr, WITH_DV)
// rfmm2d_*_ (src/laplace/rfmm2dwrap.f:36-1709), rfmm2d_*_vec_
// (src/laplace/rfmm2dwrap_vec.f:36-1690): real charges, dipole strengths
// and outputs
WRAP27(rfmm2d, _, kReal, NONE, 1, NONE, nullptr, WITH_DV)
WRAP27(rfmm2d, _vec_, kReal, ND_ARG, *nd, NONE, nullptr, WITH_DV)
// hfmm2d_*_ (src/helmholtz/hfmm2dwrap.f:41-1871), hfmm2d_*_vec_
// (src/helmholtz/hfmm2dwrap_vec.f:6-1790)
WRAP27(hfmm2d, _, kHelmholtz, NONE, 1, ZK_ARG, zk, WITH_DV)
WRAP27(hfmm2d, _vec_, kHelmholtz, ND_ARG, *nd, ZK_ARG, zk, WITH_DV)
#undef DV

#define DV(x) nullptr
// cfmm2d_*_ (src/laplace/cfmm2dwrap.f:31-1659), cfmm2d_*_vec_
// (src/laplace/cfmm2dwrap_vec.f:37-1646): no dipole vectors
WRAP27(cfmm2d, _, kCauchy, NONE, 1, NONE, nullptr, NO_DV)
WRAP27(cfmm2d, _vec_, kCauchy, ND_ARG, *nd, NONE, nullptr, NO_DV)
#undef DV

// ---------------------------------------------------------------------------
// Guru drivers.  `iper` is accepted and ignored (set to 0), as in the
// reference (src/laplace/cfmm2d.f:150).
// ---------------------------------------------------------------------------
namespace {
void guru(Kernel k, const fint *nd, const double *eps, const double *zk,
          const fint *ns, const double *sources, const fint *ifcharge,
          const double *charge, const fint *ifdipole, const double *dipstr,
          const double *dipvec, fint *iper, const fint *ifpgh, double *pot,
          double *grad, double *hess, const fint *nt, const double *targ,
          const fint *ifpghtarg, double *pottarg, double *gradtarg,
          double *hesstarg, const fint *ndiv, const fint *idivflag,
          const fint *ifnear, double *timeinfo, fint *ier) {
    FmmCall c = base_call(k, eps, zk, ns, sources);
    c.nd = *nd;
    c.ifcharge = *ifcharge;
    c.charge = charge;
    c.ifdipole = *ifdipole;
    c.dipstr = dipstr;
    c.dipvec = dipvec;
    c.ifpgh = *ifpgh;
    c.pot = pot;
    c.grad = grad;
    c.hess = hess;
    c.nt = *nt;
    c.targ = targ;
    c.ifpghtarg = *ifpghtarg;
    c.pottarg = pottarg;
    c.gradtarg = gradtarg;
    c.hesstarg = hesstarg;
    if (ndiv) {
        c.ndiv = *ndiv;
        c.idivflag = *idivflag;
    }
    if (ifnear) c.ifnear = *ifnear;
    c.timeinfo = timeinfo;
    if (iper) *iper = 0;
    *ier = run_fmm(c);
}
}  // namespace

FMM_EXPORT void lfmm2d_(const fint *nd, const double *eps, const fint *ns,
                        const double *sources, const fint *ifcharge,
                        const arr_t *charge, const fint *ifdipole,
                        const arr_t *dipstr, const double *dipvec, fint *iper,
                        const fint *ifpgh, arr_t *pot, arr_t *grad,
                        arr_t *hess, const fint *nt, const double *targ,
                        const fint *ifpghtarg, arr_t *pottarg,
                        arr_t *gradtarg, arr_t *hesstarg, fint *ier) {
    guru(kLaplace, nd, eps, nullptr, ns, sources, ifcharge, charge, ifdipole,
         dipstr, dipvec, iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
         pottarg, gradtarg, hesstarg, nullptr, nullptr, nullptr, nullptr, ier);
}

FMM_EXPORT void cfmm2d_(const fint *nd, const double *eps, const fint *ns,
                        const double *sources, const fint *ifcharge,
                        const arr_t *charge, const fint *ifdipole,
                        const arr_t *dipstr, fint *iper, const fint *ifpgh,
                        arr_t *pot, arr_t *grad, arr_t *hess, const fint *nt,
                        const double *targ, const fint *ifpghtarg,
                        arr_t *pottarg, arr_t *gradtarg, arr_t *hesstarg,
                        fint *ier) {
    guru(kCauchy, nd, eps, nullptr, ns, sources, ifcharge, charge, ifdipole,
         dipstr, nullptr, iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
         pottarg, gradtarg, hesstarg, nullptr, nullptr, nullptr, nullptr, ier);
}

FMM_EXPORT void hfmm2d_(const fint *nd, const double *eps, const arr_t *zk,
                        const fint *ns, const double *sources,
                        const fint *ifcharge, const arr_t *charge,
                        const fint *ifdipole, const arr_t *dipstr,
                        const double *dipvec, fint *iper, const fint *ifpgh,
                        arr_t *pot, arr_t *grad, arr_t *hess, const fint *nt,
                        const double *targ, const fint *ifpghtarg,
                        arr_t *pottarg, arr_t *gradtarg, arr_t *hesstarg,
                        fint *ier) {
    guru(kHelmholtz, nd, eps, zk, ns, sources, ifcharge, charge, ifdipole,
         dipstr, dipvec, iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
         pottarg, gradtarg, hesstarg, nullptr, nullptr, nullptr, nullptr, ier);
}

FMM_EXPORT void lfmm2d_ndiv_(const fint *nd, const double *eps, const fint *ns,
                             const double *sources, const fint *ifcharge,
                             const arr_t *charge, const fint *ifdipole,
                             const arr_t *dipstr, const double *dipvec,
                             fint *iper, const fint *ifpgh, arr_t *pot,
                             arr_t *grad, arr_t *hess, const fint *nt,
                             const double *targ, const fint *ifpghtarg,
                             arr_t *pottarg, arr_t *gradtarg,
                             arr_t *hesstarg, const fint *ndiv,
                             const fint *idivflag, const fint *ifnear,
                             double *timeinfo, fint *ier) {
    guru(kLaplace, nd, eps, nullptr, ns, sources, ifcharge, charge, ifdipole,
         dipstr, dipvec, iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
         pottarg, gradtarg, hesstarg, ndiv, idivflag, ifnear, timeinfo, ier);
}

FMM_EXPORT void cfmm2d_ndiv_(const fint *nd, const double *eps, const fint *ns,
                             const double *sources, const fint *ifcharge,
                             const arr_t *charge, const fint *ifdipole,
                             const arr_t *dipstr, fint *iper,
                             const fint *ifpgh, arr_t *pot, arr_t *grad,
                             arr_t *hess, const fint *nt, const double *targ,
                             const fint *ifpghtarg, arr_t *pottarg,
                             arr_t *gradtarg, arr_t *hesstarg,
                             const fint *ndiv, const fint *idivflag,
                             const fint *ifnear, double *timeinfo, fint *ier) {
    guru(kCauchy, nd, eps, nullptr, ns, sources, ifcharge, charge, ifdipole,
         dipstr, nullptr, iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
         pottarg, gradtarg, hesstarg, ndiv, idivflag, ifnear, timeinfo, ier);
}

FMM_EXPORT void hfmm2d_ndiv_(const fint *nd, const double *eps,
                             const arr_t *zk, const fint *ns,
                             const double *sources, const fint *ifcharge,
                             const arr_t *charge, const fint *ifdipole,
                             const arr_t *dipstr, const double *dipvec,
                             fint *iper, const fint *ifpgh, arr_t *pot,
                             arr_t *grad, arr_t *hess, const fint *nt,
                             const double *targ, const fint *ifpghtarg,
                             arr_t *pottarg, arr_t *gradtarg,
                             arr_t *hesstarg, const fint *ndiv,
                             const fint *idivflag, const fint *ifnear,
                             double *timeinfo, fint *ier) {
    guru(kHelmholtz, nd, eps, zk, ns, sources, ifcharge, charge, ifdipole,
         dipstr, dipvec, iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
         pottarg, gradtarg, hesstarg, ndiv, idivflag, ifnear, timeinfo, ier);
}

// Real-valued Laplace FMM (src/laplace/rfmm2d.f:27; the ndiv form
// src/laplace/rfmm2d_ndiv.f:27, c_translation/src/rfmm2d_ndiv.c:51): real
// charge(nd,ns), dipstr(nd,ns), dipvec(nd,2,ns), pot(nd,*), grad(nd,2,*),
// hess(nd,3,*).
FMM_EXPORT void rfmm2d_(const fint *nd, const double *eps, const fint *ns,
                        const double *sources, const fint *ifcharge,
                        const double *charge, const fint *ifdipole,
                        const double *dipstr, const double *dipvec, fint *iper,
                        const fint *ifpgh, double *pot, double *grad, double *hess,
                        const fint *nt, const double *targ, const fint *ifpghtarg,
                        double *pottarg, double *gradtarg, double *hesstarg, fint *ier) {
    guru(kReal, nd, eps, nullptr, ns, sources, ifcharge, charge, ifdipole, dipstr, dipvec,
         iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg,
         nullptr, nullptr, nullptr, nullptr, ier);
}

FMM_EXPORT void rfmm2d_ndiv_(const fint *nd, const double *eps, const fint *ns,
                             const double *sources, const fint *ifcharge,
                             const double *charge, const fint *ifdipole,
                             const double *dipstr, const double *dipvec, fint *iper,
                             const fint *ifpgh, double *pot, double *grad, double *hess,
                             const fint *nt, const double *targ, const fint *ifpghtarg,
                             double *pottarg, double *gradtarg, double *hesstarg,
                             const fint *ndiv, const fint *idivflag, const fint *ifnear,
                             double *timeinfo, fint *ier) {
    guru(kReal, nd, eps, nullptr, ns, sources, ifcharge, charge, ifdipole, dipstr, dipvec,
         iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg, ndiv,
         idivflag, ifnear, timeinfo, ier);
}

// ---------------------------------------------------------------------------
// Library knobs with no counterpart in the reference.
// ---------------------------------------------------------------------------
// Precision policy: 0 auto (mixed for eps >= 1e-6), 1 all-FP64, 2 mixed.
// A batch of independent lfmm2d (kernel 0) / cfmm2d (kernel 1) problems,
// nd = 1, same eps and output flags, evaluated as one forest.
FMM_EXPORT int fmm2d_b200_fmm2d_batch(int kernel, int nprob, double eps, const int *ns,
                                      const double *const *sources, const double *const *charge,
                                      const double *const *dipstr, const double *const *dipvec,
                                      int ifpgh, double *const *pot, double *const *grad,
                                      double *const *hess, const int *nt,
                                      const double *const *targ, int ifpghtarg,
                                      double *const *pottarg, double *const *gradtarg,
                                      double *const *hesstarg) {
    BatchCall b;
    b.kernel = (Kernel)kernel;
    b.eps = eps;
    b.nprob = nprob;
    b.ns = ns;
    b.nt = nt;
    b.sources = sources;
    b.targ = targ;
    b.charge = charge;
    b.dipstr = dipstr;
    b.dipvec = dipvec;
    b.ifpgh = ifpgh;
    b.ifpghtarg = ifpghtarg;
    b.pot = pot;
    b.grad = grad;
    b.hess = hess;
    b.pottarg = pottarg;
    b.gradtarg = gradtarg;
    b.hesstarg = hesstarg;
    b.precision = current_precision();
    if (!ns || !sources || (ifpgh >= 1 && !pot) || (ifpgh >= 2 && !grad) ||
        (ifpgh >= 3 && !hess) || (ifpghtarg >= 1 && nt && !pottarg) ||
        (ifpghtarg >= 2 && nt && !gradtarg) || (ifpghtarg >= 3 && nt && !hesstarg) ||
        (nt && !targ)) {
        set_last_error("batch: an array list the flags ask for is missing");
        return 4;
    }
    return run_laplace_batch(b);
}

FMM_EXPORT int fmm2d_b200_set_precision(int mode) {
    if (mode < 0 || mode > 3) return 4;
    set_precision(mode);
    return 0;
}

// Host-only helpers (no device needed): the eps -> order and eps -> leaf
// capacity rules the drivers use.
FMM_EXPORT int fmm2d_b200_laplace_nterms(double eps) { return laplace_nterms(eps); }
FMM_EXPORT int fmm2d_b200_leaf_capacity(double eps, int ns, int nt) {
    return leaf_capacity(eps, ns, nt);
}

// ---------------------------------------------------------------------------
// bind(c) Helmholtz entry, src/helmholtz_c.f03:5-15: eps, zk and ns by
// value, ns and ier 64-bit.  A complex double passed by value has the
// calling convention of a struct of two doubles.
// ---------------------------------------------------------------------------
struct cplx_by_value {
    double re, im;
};

FMM_EXPORT void hfmm2d_s_c_p(double eps, cplx_by_value zk, int64_t ns, const double *sources,
                             const arr_t *charge, arr_t *pot, int64_t *ier) {
    if (ns < 1 || ns > INT32_MAX) {
        set_last_error("ns out of range for the 32-bit drivers");
        *ier = 4;
        return;
    }
    const double zkv[2] = {zk.re, zk.im};
    const fint ns32 = (fint)ns;
    fint ier32 = 0;
    wrap(kHelmholtz, 1, &eps, zkv, &ns32, sources, charge, nullptr, nullptr, 1, 0, 1, pot, nullptr,
         nullptr, 0, nullptr, 0, nullptr, nullptr, nullptr, &ier32);
    *ier = ier32;
}

// Helmholtz direct sum (h2d_direct*, c_translation/src/helmkernels2d.c):
// increments pot(nd,nt), grad(nd,2,nt), hess(nd,3,nt); zk = (re, im).
FMM_EXPORT int fmm2d_b200_h2d_direct(int nd, const double *zk, int ns, const double *sources,
                                     int ifcharge, const double *charge, int ifdipole,
                                     const double *dipstr, const double *dipvec, int nt,
                                     const double *targ, int ifpgh, double *pot, double *grad,
                                     double *hess, double thresh) {
    return run_helm_direct(nd, zk, ns, sources, ifcharge, charge, ifdipole, dipstr, dipvec, nt,
                           targ, ifpgh, pot, grad, hess, thresh);
}

// Host-only: the Helmholtz expansion order of h2dterms for a box size, and
// H0, H1 of the library's own Hankel routine at n complex points
// (z[2k], z[2k+1]) -> out[4k .. 4k+3] = (H0 re, im, H1 re, im).
FMM_EXPORT int fmm2d_b200_helm_nterms(double bsize, double zk_re, double zk_im, double eps) {
    return helm_nterms(bsize, make_double2(zk_re, zk_im), eps);
}
FMM_EXPORT void fmm2d_b200_hankel01(int n, const double *z, double *out) {
    for (int k = 0; k < n; k++) {
        double2 h0, h1;
        hk::hankel01(make_double2(z[2 * k], z[2 * k + 1]), h0, h1);
        out[4 * k] = h0.x;
        out[4 * k + 1] = h0.y;
        out[4 * k + 2] = h1.x;
        out[4 * k + 3] = h1.y;
    }
}
// Host-only: the scaled sequences the Helmholtz translations are built
// from, out[0..n] complex (interleaved): H_k(z) rscale^k (h2dall) and
// J_k(z) / rscale^k (jbessel2d).
FMM_EXPORT void fmm2d_b200_helm_hvec(int n, double z_re, double z_im, double rscale, double *out) {
    helm_hvec(n, make_double2(z_re, z_im), rscale, reinterpret_cast<double2 *>(out));
}
FMM_EXPORT void fmm2d_b200_helm_jvec(int n, double z_re, double z_im, double rscale, double *out) {
    helm_jvec(n, make_double2(z_re, z_im), rscale, reinterpret_cast<double2 *>(out));
}

// Leaf capacity of the mixed-precision Laplace / Cauchy mode for order
// nterms (ndiv <= 0: back to the reference's rule); the current choice.
FMM_EXPORT int fmm2d_b200_set_leaf_capacity(int nterms, int ndiv) {
    if (nterms < 0 || nterms >= 128) return 4;
    set_mixed_leaf_capacity(nterms, ndiv);
    return 0;
}
FMM_EXPORT int fmm2d_b200_mixed_leaf_capacity(double eps, int ns, int nt) {
    return mixed_leaf_capacity(laplace_nterms(eps), leaf_capacity(eps, ns, nt));
}
