/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 * The reference's C translation (c_translation/src/*.c) covers the Cauchy and
 * Helmholtz engines but three pieces of the user-facing path exist only in
 * Fortran.  This file restates them in C so that the reference's own C code
 * can be driven through exactly the entry points the GPU library replaces:
 *
 *   lndiv2d_      src/laplace/lndiv2d.f:1-39      eps -> (ndiv, idivflag)
 *   lfmm2d_       src/laplace/lfmm2d.f:29-225     complex-Laplace driver; the
 *                 reference C port provides the identical channel packing in
 *                 lfmm2d_ndiv_ (c_translation/src/lfmm2d_ndiv.c), so lfmm2d_
 *                 is lndiv2d_ followed by lfmm2d_ndiv_ with ifnear = 1,
 *                 which is what src/laplace/lfmm2d.f:160-164 -> cfmm2d does.
 *   81 wrappers   src/laplace/lfmm2dwrap.f:31-1704, cfmm2dwrap.f:31-1659,
 *                 src/helmholtz/hfmm2dwrap.f:41-1871: each sets
 *                 ifcharge/ifdipole/ifpgh/ifpghtarg, nd = 1, nt = 0 for the
 *                 sources-only forms and ifpgh = 0 for the targets-only
 *                 forms, then calls the guru driver.
 *   hfmm2d_s_c_p  src/helmholtz_c.f03:5-15 (bind(c), by-value eps/zk/ns).
 *
 * Built together with the reference sources into oracle/_ref/ by
 * oracle/Makefile.  It is the checker the GPU path is compared against.
 */
#include <complex.h>
#include <stdint.h>
#include <stddef.h>

typedef int32_t fint;
typedef double _Complex fcomplex;

/* reference C port entry points (exported under their gfortran names) */
extern void lfmm2d_ndiv_(const fint *nd, const double *eps, const fint *ns,
                         const double *sources, const fint *ifcharge,
                         const fcomplex *charge, const fint *ifdipole,
                         const fcomplex *dipstr, const double *dipvec,
                         fint *iper, const fint *ifpgh, fcomplex *pot,
                         fcomplex *grad, fcomplex *hess, const fint *nt,
                         const double *targ, const fint *ifpghtarg,
                         fcomplex *pottarg, fcomplex *gradtarg,
                         fcomplex *hesstarg, const fint *ndiv,
                         const fint *idivflag, const fint *ifnear,
                         double *timeinfo, fint *ier);
extern void cfmm2d_(const fint *nd, const double *eps, const fint *ns,
                    const double *sources, const fint *ifcharge,
                    const fcomplex *charge, const fint *ifdipole,
                    const fcomplex *dipstr, fint *iper, const fint *ifpgh,
                    fcomplex *pot, fcomplex *grad, fcomplex *hess,
                    const fint *nt, const double *targ, const fint *ifpghtarg,
                    fcomplex *pottarg, fcomplex *gradtarg, fcomplex *hesstarg,
                    fint *ier);
extern void hfmm2d_(const fint *nd, const double *eps, const fcomplex *zk,
                    const fint *ns, const double *sources,
                    const fint *ifcharge, const fcomplex *charge,
                    const fint *ifdipole, const fcomplex *dipstr,
                    const double *dipvec, fint *iper, const fint *ifpgh,
                    fcomplex *pot, fcomplex *grad, fcomplex *hess,
                    const fint *nt, const double *targ, const fint *ifpghtarg,
                    fcomplex *pottarg, fcomplex *gradtarg, fcomplex *hesstarg,
                    fint *ier);

/* src/laplace/lndiv2d.f:1-39: leaf capacity from the requested precision. */
void lndiv2d_(const double *eps, const fint *ns, const fint *nt,
              const fint *ifcharge, const fint *ifdipole, const fint *ifpgh,
              const fint *ifpghtarg, fint *ndiv, fint *idivflag)
{
    static const double cut[8] = {0.5, 0.5e-1, 0.5e-2, 0.5e-3,
                                  0.5e-6, 0.5e-9, 0.5e-12, 0.5e-15};
    static const fint val[8] = {3, 5, 8, 10, 15, 20, 25, 45};
    (void)ifcharge; (void)ifdipole; (void)ifpgh; (void)ifpghtarg;
    *idivflag = 0;
    for (int k = 0; k < 8; k++) {
        if (*eps >= cut[k]) { *ndiv = val[k]; return; }
    }
    *ndiv = *ns + *nt;
}

/* src/laplace/lfmm2d.f:29-225 (guru complex-Laplace driver). */
void lfmm2d_(const fint *nd, const double *eps, const fint *ns,
             const double *sources, const fint *ifcharge,
             const fcomplex *charge, const fint *ifdipole,
             const fcomplex *dipstr, const double *dipvec, fint *iper,
             const fint *ifpgh, fcomplex *pot, fcomplex *grad, fcomplex *hess,
             const fint *nt, const double *targ, const fint *ifpghtarg,
             fcomplex *pottarg, fcomplex *gradtarg, fcomplex *hesstarg,
             fint *ier)
{
    fint ndiv, idivflag, ifnear = 1;
    double timeinfo[8];
    lndiv2d_(eps, ns, nt, ifcharge, ifdipole, ifpgh, ifpghtarg, &ndiv,
             &idivflag);
    *iper = 0;
    lfmm2d_ndiv_(nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                 dipvec, iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
                 pottarg, gradtarg, hesstarg, &ndiv, &idivflag, &ifnear,
                 timeinfo, ier);
}

/* ------------------------------------------------------------------ */
/* The 81 flag wrappers.  One generic call per family; each exported   */
/* wrapper only fixes the flags and forwards its own arguments.        */
/* ------------------------------------------------------------------ */
static fcomplex zdum[8];
static double ddum[8];

static void lcall(const double *eps, const fint *ns, const double *src,
                  const fcomplex *chg, const fcomplex *dip, const double *dv,
                  fint ifc, fint ifd, fint ifpgh, fcomplex *pot, fcomplex *grad,
                  fcomplex *hess, fint nt, const double *targ, fint ifpt,
                  fcomplex *pt, fcomplex *gt, fcomplex *ht, fint *ier)
{
    fint nd = 1, iper = 0;
    lfmm2d_(&nd, eps, ns, src, &ifc, chg ? chg : zdum, &ifd, dip ? dip : zdum,
            dv ? dv : ddum, &iper, &ifpgh, pot ? pot : zdum,
            grad ? grad : zdum, hess ? hess : zdum, &nt, targ ? targ : ddum,
            &ifpt, pt ? pt : zdum, gt ? gt : zdum, ht ? ht : zdum, ier);
}

static void ccall(const double *eps, const fint *ns, const double *src,
                  const fcomplex *chg, const fcomplex *dip, const double *dv,
                  fint ifc, fint ifd, fint ifpgh, fcomplex *pot, fcomplex *grad,
                  fcomplex *hess, fint nt, const double *targ, fint ifpt,
                  fcomplex *pt, fcomplex *gt, fcomplex *ht, fint *ier)
{
    fint nd = 1, iper = 0;
    (void)dv;
    cfmm2d_(&nd, eps, ns, src, &ifc, chg ? chg : zdum, &ifd, dip ? dip : zdum,
            &iper, &ifpgh, pot ? pot : zdum, grad ? grad : zdum,
            hess ? hess : zdum, &nt, targ ? targ : ddum, &ifpt,
            pt ? pt : zdum, gt ? gt : zdum, ht ? ht : zdum, ier);
}

static void hcall(const fcomplex *hzk, const double *eps, const fint *ns, const double *src,
                  const fcomplex *chg, const fcomplex *dip, const double *dv,
                  fint ifc, fint ifd, fint ifpgh, fcomplex *pot, fcomplex *grad,
                  fcomplex *hess, fint nt, const double *targ, fint ifpt,
                  fcomplex *pt, fcomplex *gt, fcomplex *ht, fint *ier)
{
    fint nd = 1, iper = 0;
    hfmm2d_(&nd, eps, hzk, ns, src, &ifc, chg ? chg : zdum, &ifd,
            dip ? dip : zdum, dv ? dv : ddum, &iper, &ifpgh,
            pot ? pot : zdum, grad ? grad : zdum, hess ? hess : zdum, &nt,
            targ ? targ : ddum, &ifpt, pt ? pt : zdum, gt ? gt : zdum,
            ht ? ht : zdum, ier);
}

/* source-strength argument lists: c = charge, d = dipole, cd = both */
#define SRC_c(V) const fcomplex *charge
#define SRC_d(V) const fcomplex *dipstr V(const double *dipvec)
#define SRC_cd(V) const fcomplex *charge, const fcomplex *dipstr V(const double *dipvec)
#define PASS_c charge, NULL, NULL, 1, 0
#define PASS_d NULL, dipstr, DV(dipvec), 0, 1
#define PASS_cd charge, dipstr, DV(dipvec), 1, 1
/* output argument lists at sources (s) and targets (t) */
#define OUT_S_p fcomplex *pot
#define OUT_S_g fcomplex *pot, fcomplex *grad
#define OUT_S_h fcomplex *pot, fcomplex *grad, fcomplex *hess
#define OUT_T_p fcomplex *pottarg
#define OUT_T_g fcomplex *pottarg, fcomplex *gradtarg
#define OUT_T_h fcomplex *pottarg, fcomplex *gradtarg, fcomplex *hesstarg
#define PS_p 1, pot, NULL, NULL
#define PS_g 2, pot, grad, NULL
#define PS_h 3, pot, grad, hess
#define PT_p 1, pottarg, NULL, NULL
#define PT_g 2, pottarg, gradtarg, NULL
#define PT_h 3, pottarg, gradtarg, hesstarg

#define WITH_DV(x) , x
#define NO_DV(x)

/* lfmm2d_* and hfmm2d_* carry dipvec; cfmm2d_* do not */
#define DV(x) x
#define LWRAP(K, P)                                                         \
    void lfmm2d_s_##K##_##P##_(const double *eps, const fint *ns,           \
                               const double *sources, SRC_##K(WITH_DV),     \
                               OUT_S_##P, fint *ier)                        \
    { lcall(eps, ns, sources, PASS_##K, PS_##P, 0, NULL, 0, NULL, NULL,     \
            NULL, ier); }                                                   \
    void lfmm2d_t_##K##_##P##_(const double *eps, const fint *ns,           \
                               const double *sources, SRC_##K(WITH_DV),     \
                               const fint *nt, const double *targ,          \
                               OUT_T_##P, fint *ier)                        \
    { lcall(eps, ns, sources, PASS_##K, 0, NULL, NULL, NULL, *nt, targ,     \
            PT_##P, ier); }                                                 \
    void lfmm2d_st_##K##_##P##_(const double *eps, const fint *ns,          \
                                const double *sources, SRC_##K(WITH_DV),    \
                                OUT_S_##P, const fint *nt,                  \
                                const double *targ, OUT_T_##P, fint *ier)   \
    { lcall(eps, ns, sources, PASS_##K, PS_##P, *nt, targ, PT_##P, ier); }

#define HWRAP(K, P)                                                         \
    void hfmm2d_s_##K##_##P##_(const double *eps, const fcomplex *zk,       \
                               const fint *ns, const double *sources,       \
                               SRC_##K(WITH_DV), OUT_S_##P, fint *ier)      \
    { hcall(zk, eps, ns, sources, PASS_##K, PS_##P, 0, NULL, 0,       \
                      NULL, NULL, NULL, ier); }                             \
    void hfmm2d_t_##K##_##P##_(const double *eps, const fcomplex *zk,       \
                               const fint *ns, const double *sources,       \
                               SRC_##K(WITH_DV), const fint *nt,            \
                               const double *targ, OUT_T_##P, fint *ier)    \
    { hcall(zk, eps, ns, sources, PASS_##K, 0, NULL, NULL, NULL, *nt, \
                      targ, PT_##P, ier); }                                 \
    void hfmm2d_st_##K##_##P##_(const double *eps, const fcomplex *zk,      \
                                const fint *ns, const double *sources,      \
                                SRC_##K(WITH_DV), OUT_S_##P,                \
                                const fint *nt, const double *targ,         \
                                OUT_T_##P, fint *ier)                       \
    { hcall(zk, eps, ns, sources, PASS_##K, PS_##P, *nt, targ,        \
                      PT_##P, ier); }

LWRAP(c, p) LWRAP(c, g) LWRAP(c, h)
LWRAP(d, p) LWRAP(d, g) LWRAP(d, h)
LWRAP(cd, p) LWRAP(cd, g) LWRAP(cd, h)
HWRAP(c, p) HWRAP(c, g) HWRAP(c, h)
HWRAP(d, p) HWRAP(d, g) HWRAP(d, h)
HWRAP(cd, p) HWRAP(cd, g) HWRAP(cd, h)
#undef DV

#define DV(x) NULL
#define CWRAP(K, P)                                                         \
    void cfmm2d_s_##K##_##P##_(const double *eps, const fint *ns,           \
                               const double *sources, SRC_##K(NO_DV),       \
                               OUT_S_##P, fint *ier)                        \
    { ccall(eps, ns, sources, PASS_##K, PS_##P, 0, NULL, 0, NULL, NULL,     \
            NULL, ier); }                                                   \
    void cfmm2d_t_##K##_##P##_(const double *eps, const fint *ns,           \
                               const double *sources, SRC_##K(NO_DV),       \
                               const fint *nt, const double *targ,          \
                               OUT_T_##P, fint *ier)                        \
    { ccall(eps, ns, sources, PASS_##K, 0, NULL, NULL, NULL, *nt, targ,     \
            PT_##P, ier); }                                                 \
    void cfmm2d_st_##K##_##P##_(const double *eps, const fint *ns,          \
                                const double *sources, SRC_##K(NO_DV),      \
                                OUT_S_##P, const fint *nt,                  \
                                const double *targ, OUT_T_##P, fint *ier)   \
    { ccall(eps, ns, sources, PASS_##K, PS_##P, *nt, targ, PT_##P, ier); }

CWRAP(c, p) CWRAP(c, g) CWRAP(c, h)
CWRAP(d, p) CWRAP(d, g) CWRAP(d, h)
CWRAP(cd, p) CWRAP(cd, g) CWRAP(cd, h)
#undef DV

/* src/helmholtz_c.f03:5-15: bind(c) form with by-value scalars. */
void hfmm2d_s_c_p(double eps, fcomplex zk, int64_t ns, const double *sources,
                  const fcomplex *charge, fcomplex *pot, int64_t *ier)
{
    fint ns32 = (fint)ns, ier32 = 0;
    hfmm2d_s_c_p_(&eps, &zk, &ns32, sources, charge, pot, &ier32);
    *ier = ier32;
}
