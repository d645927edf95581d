/*
 * fmm2d_b200.h -- C ABI of libfmm2d_b200.so, the B200 evaluation path of
 * fmm2d (complex-Laplace, Cauchy and Helmholtz FMMs in two dimensions).
 *
 * The first group of entry points replaces the reference library's own
 * symbols one for one: same names (gfortran convention: lowercase + '_'),
 * same arguments in the same order, every argument by pointer, Fortran
 * integer = int32_t, complex*16 = double _Complex (interleaved re, im),
 * arrays column-major exactly as the reference documents them.  A program
 * linked against the reference library links against this one unchanged.
 * Each declaration cites the reference interface it replaces.
 *
 * Semantics follow the reference: outputs are overwritten (not
 * accumulated) in input order; ier = 0 on success, 4 on failure (the only
 * code the reference reports, src/helmholtz/hfmm2d.f:374-381); the message
 * of a failure is available from fmm2d_b200_last_error().  Arrays may be
 * host memory (pageable or pinned) or device memory of the calling
 * thread's current CUDA device; all arrays of one call must be of the same
 * kind.  Calls are synchronous and may be made concurrently from several
 * host threads.
 *
 * The second group (fmm2d_b200_*) has no counterpart in the reference:
 * library-specific controls, inspection and measurement helpers.
 */
#ifndef FMM2D_B200_H
#define FMM2D_B200_H

#include <stdint.h>
#ifdef __cplusplus
/* C++ callers pass complex arrays as double * (interleaved re, im) */
#define _Complex
extern "C" {
#endif

/* ===================================================================== */
/* Flag wrappers: {l,c,h}fmm2d_{s,t,st}_{c,d,cd}_{p,g,h}_ (rfmm2d and    */
/* the _vec forms follow below)                                          */
/*   s / t / st : evaluate at sources, at targets, at both               */
/*   c / d / cd : charges, dipoles, both                                 */
/*   p / g / h  : potential, + gradient, + Hessian                       */
/* lfmm2d: grad(2,n), hess(3,n); cfmm2d: grad(n), hess(n) (d/dz, d2/dz2);  */
/* hfmm2d: grad(2,n), hess(3,n) and the Helmholtz parameter zk.          */
/* ===================================================================== */
/* src/laplace/lfmm2dwrap.f:31 */
void lfmm2d_s_c_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   double _Complex *pot, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:93 */
void lfmm2d_s_c_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   double _Complex *pot, double _Complex *grad, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:156 */
void lfmm2d_s_c_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   double _Complex *pot, double _Complex *grad,
                   double _Complex *hess, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:217 */
void lfmm2d_s_d_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   const double *dipvec, double _Complex *pot, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:280 */
void lfmm2d_s_d_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   const double *dipvec, double _Complex *pot,
                   double _Complex *grad, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:344 */
void lfmm2d_s_d_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   const double *dipvec, double _Complex *pot,
                   double _Complex *grad, double _Complex *hess,
                   int32_t *ier);
/* src/laplace/lfmm2dwrap.f:406 */
void lfmm2d_s_cd_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    double _Complex *pot, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:468 */
void lfmm2d_s_cd_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    double _Complex *pot, double _Complex *grad,
                    int32_t *ier);
/* src/laplace/lfmm2dwrap.f:531 */
void lfmm2d_s_cd_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    double _Complex *pot, double _Complex *grad,
                    double _Complex *hess, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:594 */
void lfmm2d_t_c_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:654 */
void lfmm2d_t_c_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, double _Complex *gradtarg,
                   int32_t *ier);
/* src/laplace/lfmm2dwrap.f:715 */
void lfmm2d_t_c_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, double _Complex *gradtarg,
                   double _Complex *hesstarg, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:775 */
void lfmm2d_t_d_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   const double *dipvec, const int32_t *nt,
                   const double *targ, double _Complex *pottarg,
                   int32_t *ier);
/* src/laplace/lfmm2dwrap.f:836 */
void lfmm2d_t_d_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   const double *dipvec, const int32_t *nt,
                   const double *targ, double _Complex *pottarg,
                   double _Complex *gradtarg, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:898 */
void lfmm2d_t_d_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   const double *dipvec, const int32_t *nt,
                   const double *targ, double _Complex *pottarg,
                   double _Complex *gradtarg, double _Complex *hesstarg,
                   int32_t *ier);
/* src/laplace/lfmm2dwrap.f:959 */
void lfmm2d_t_cd_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1019 */
void lfmm2d_t_cd_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1080 */
void lfmm2d_t_cd_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    double _Complex *hesstarg, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1143 */
void lfmm2d_st_c_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    double _Complex *pot, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1204 */
void lfmm2d_st_c_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    double _Complex *pot, double _Complex *grad,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1267 */
void lfmm2d_st_c_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    double _Complex *pot, double _Complex *grad,
                    double _Complex *hess, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    double _Complex *gradtarg, double _Complex *hesstarg,
                    int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1330 */
void lfmm2d_st_d_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *dipstr,
                    const double *dipvec, double _Complex *pot,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1392 */
void lfmm2d_st_d_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *dipstr,
                    const double *dipvec, double _Complex *pot,
                    double _Complex *grad, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    double _Complex *gradtarg, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1456 */
void lfmm2d_st_d_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *dipstr,
                    const double *dipvec, double _Complex *pot,
                    double _Complex *grad, double _Complex *hess,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    double _Complex *hesstarg, int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1520 */
void lfmm2d_st_cd_p_(const double *eps, const int32_t *ns,
                     const double *sources, const double _Complex *charge,
                     const double _Complex *dipstr, const double *dipvec,
                     double _Complex *pot, const int32_t *nt,
                     const double *targ, double _Complex *pottarg,
                     int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1581 */
void lfmm2d_st_cd_g_(const double *eps, const int32_t *ns,
                     const double *sources, const double _Complex *charge,
                     const double _Complex *dipstr, const double *dipvec,
                     double _Complex *pot, double _Complex *grad,
                     const int32_t *nt, const double *targ,
                     double _Complex *pottarg, double _Complex *gradtarg,
                     int32_t *ier);
/* src/laplace/lfmm2dwrap.f:1644 */
void lfmm2d_st_cd_h_(const double *eps, const int32_t *ns,
                     const double *sources, const double _Complex *charge,
                     const double _Complex *dipstr, const double *dipvec,
                     double _Complex *pot, double _Complex *grad,
                     double _Complex *hess, const int32_t *nt,
                     const double *targ, double _Complex *pottarg,
                     double _Complex *gradtarg, double _Complex *hesstarg,
                     int32_t *ier);
/* src/laplace/cfmm2dwrap.f:31 */
void cfmm2d_s_c_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   double _Complex *pot, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:92 */
void cfmm2d_s_c_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   double _Complex *pot, double _Complex *grad, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:154 */
void cfmm2d_s_c_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   double _Complex *pot, double _Complex *grad,
                   double _Complex *hess, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:214 */
void cfmm2d_s_d_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   double _Complex *pot, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:275 */
void cfmm2d_s_d_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   double _Complex *pot, double _Complex *grad, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:337 */
void cfmm2d_s_d_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   double _Complex *pot, double _Complex *grad,
                   double _Complex *hess, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:397 */
void cfmm2d_s_cd_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, double _Complex *pot,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:457 */
void cfmm2d_s_cd_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, double _Complex *pot,
                    double _Complex *grad, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:518 */
void cfmm2d_s_cd_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, double _Complex *pot,
                    double _Complex *grad, double _Complex *hess,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:579 */
void cfmm2d_t_c_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:638 */
void cfmm2d_t_c_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, double _Complex *gradtarg,
                   int32_t *ier);
/* src/laplace/cfmm2dwrap.f:698 */
void cfmm2d_t_c_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *charge,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, double _Complex *gradtarg,
                   double _Complex *hesstarg, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:757 */
void cfmm2d_t_d_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:816 */
void cfmm2d_t_d_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, double _Complex *gradtarg,
                   int32_t *ier);
/* src/laplace/cfmm2dwrap.f:876 */
void cfmm2d_t_d_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double _Complex *dipstr,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, double _Complex *gradtarg,
                   double _Complex *hesstarg, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:935 */
void cfmm2d_t_cd_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:993 */
void cfmm2d_t_cd_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    double _Complex *gradtarg, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1052 */
void cfmm2d_t_cd_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    const double _Complex *dipstr, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    double _Complex *gradtarg, double _Complex *hesstarg,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1113 */
void cfmm2d_st_c_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    double _Complex *pot, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1173 */
void cfmm2d_st_c_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    double _Complex *pot, double _Complex *grad,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1235 */
void cfmm2d_st_c_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *charge,
                    double _Complex *pot, double _Complex *grad,
                    double _Complex *hess, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    double _Complex *gradtarg, double _Complex *hesstarg,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1297 */
void cfmm2d_st_d_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *dipstr,
                    double _Complex *pot, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1357 */
void cfmm2d_st_d_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *dipstr,
                    double _Complex *pot, double _Complex *grad,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1419 */
void cfmm2d_st_d_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double _Complex *dipstr,
                    double _Complex *pot, double _Complex *grad,
                    double _Complex *hess, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    double _Complex *gradtarg, double _Complex *hesstarg,
                    int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1481 */
void cfmm2d_st_cd_p_(const double *eps, const int32_t *ns,
                     const double *sources, const double _Complex *charge,
                     const double _Complex *dipstr, double _Complex *pot,
                     const int32_t *nt, const double *targ,
                     double _Complex *pottarg, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1540 */
void cfmm2d_st_cd_g_(const double *eps, const int32_t *ns,
                     const double *sources, const double _Complex *charge,
                     const double _Complex *dipstr, double _Complex *pot,
                     double _Complex *grad, const int32_t *nt,
                     const double *targ, double _Complex *pottarg,
                     double _Complex *gradtarg, int32_t *ier);
/* src/laplace/cfmm2dwrap.f:1601 */
void cfmm2d_st_cd_h_(const double *eps, const int32_t *ns,
                     const double *sources, const double _Complex *charge,
                     const double _Complex *dipstr, double _Complex *pot,
                     double _Complex *grad, double _Complex *hess,
                     const int32_t *nt, const double *targ,
                     double _Complex *pottarg, double _Complex *gradtarg,
                     double _Complex *hesstarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:41 */
void hfmm2d_s_c_p_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *charge, double _Complex *pot,
                   int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:108 */
void hfmm2d_s_c_g_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *charge, double _Complex *pot,
                   double _Complex *grad, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:177 */
void hfmm2d_s_c_h_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *charge, double _Complex *pot,
                   double _Complex *grad, double _Complex *hess,
                   int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:245 */
void hfmm2d_s_d_p_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *dipstr, const double *dipvec,
                   double _Complex *pot, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:312 */
void hfmm2d_s_d_g_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *dipstr, const double *dipvec,
                   double _Complex *pot, double _Complex *grad, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:382 */
void hfmm2d_s_d_h_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *dipstr, const double *dipvec,
                   double _Complex *pot, double _Complex *grad,
                   double _Complex *hess, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:451 */
void hfmm2d_s_cd_p_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    double _Complex *pot, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:521 */
void hfmm2d_s_cd_g_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    double _Complex *pot, double _Complex *grad,
                    int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:590 */
void hfmm2d_s_cd_h_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    double _Complex *pot, double _Complex *grad,
                    double _Complex *hess, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:657 */
void hfmm2d_t_c_p_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *charge, const int32_t *nt,
                   const double *targ, double _Complex *pottarg,
                   int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:721 */
void hfmm2d_t_c_g_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *charge, const int32_t *nt,
                   const double *targ, double _Complex *pottarg,
                   double _Complex *gradtarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:788 */
void hfmm2d_t_c_h_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *charge, const int32_t *nt,
                   const double *targ, double _Complex *pottarg,
                   double _Complex *gradtarg, double _Complex *hesstarg,
                   int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:855 */
void hfmm2d_t_d_p_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *dipstr, const double *dipvec,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:920 */
void hfmm2d_t_d_g_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *dipstr, const double *dipvec,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, double _Complex *gradtarg,
                   int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:988 */
void hfmm2d_t_d_h_(const double *eps, const double _Complex *zk,
                   const int32_t *ns, const double *sources,
                   const double _Complex *dipstr, const double *dipvec,
                   const int32_t *nt, const double *targ,
                   double _Complex *pottarg, double _Complex *gradtarg,
                   double _Complex *hesstarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1056 */
void hfmm2d_t_cd_p_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1124 */
void hfmm2d_t_cd_g_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1191 */
void hfmm2d_t_cd_h_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *charge,
                    const double _Complex *dipstr, const double *dipvec,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    double _Complex *hesstarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1264 */
void hfmm2d_st_c_p_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *charge, double _Complex *pot,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1329 */
void hfmm2d_st_c_g_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *charge, double _Complex *pot,
                    double _Complex *grad, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    double _Complex *gradtarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1397 */
void hfmm2d_st_c_h_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *charge, double _Complex *pot,
                    double _Complex *grad, double _Complex *hess,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    double _Complex *hesstarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1465 */
void hfmm2d_st_d_p_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *dipstr, const double *dipvec,
                    double _Complex *pot, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1531 */
void hfmm2d_st_d_g_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *dipstr, const double *dipvec,
                    double _Complex *pot, double _Complex *grad,
                    const int32_t *nt, const double *targ,
                    double _Complex *pottarg, double _Complex *gradtarg,
                    int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1600 */
void hfmm2d_st_d_h_(const double *eps, const double _Complex *zk,
                    const int32_t *ns, const double *sources,
                    const double _Complex *dipstr, const double *dipvec,
                    double _Complex *pot, double _Complex *grad,
                    double _Complex *hess, const int32_t *nt,
                    const double *targ, double _Complex *pottarg,
                    double _Complex *gradtarg, double _Complex *hesstarg,
                    int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1669 */
void hfmm2d_st_cd_p_(const double *eps, const double _Complex *zk,
                     const int32_t *ns, const double *sources,
                     const double _Complex *charge,
                     const double _Complex *dipstr, const double *dipvec,
                     double _Complex *pot, const int32_t *nt,
                     const double *targ, double _Complex *pottarg,
                     int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1738 */
void hfmm2d_st_cd_g_(const double *eps, const double _Complex *zk,
                     const int32_t *ns, const double *sources,
                     const double _Complex *charge,
                     const double _Complex *dipstr, const double *dipvec,
                     double _Complex *pot, double _Complex *grad,
                     const int32_t *nt, const double *targ,
                     double _Complex *pottarg, double _Complex *gradtarg,
                     int32_t *ier);
/* src/helmholtz/hfmm2dwrap.f:1806 */
void hfmm2d_st_cd_h_(const double *eps, const double _Complex *zk,
                     const int32_t *ns, const double *sources,
                     const double _Complex *charge,
                     const double _Complex *dipstr, const double *dipvec,
                     double _Complex *pot, double _Complex *grad,
                     double _Complex *hess, const int32_t *nt,
                     const double *targ, double _Complex *pottarg,
                     double _Complex *gradtarg, double _Complex *hesstarg,
                     int32_t *ier);

/* ===================================================================== */
/* rfmm2d_{s,t,st}_{c,d,cd}_{p,g,h}_: the real-valued Laplace FMM        */
/* (src/laplace/rfmm2d.f:27): real charge(n), dipstr(n), dipvec(2,n),    */
/* real pot(n), grad(2,n), hess(3,n).                                    */
/* ===================================================================== */
/* src/laplace/rfmm2dwrap.f:36 */
void rfmm2d_s_c_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double *charge, double *pot,
                   int32_t *ier);
/* src/laplace/rfmm2dwrap.f:98 */
void rfmm2d_s_c_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double *charge, double *pot,
                   double *grad, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:161 */
void rfmm2d_s_c_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double *charge, double *pot,
                   double *grad, double *hess, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:222 */
void rfmm2d_s_d_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double *dipstr,
                   const double *dipvec, double *pot, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:285 */
void rfmm2d_s_d_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double *dipstr,
                   const double *dipvec, double *pot, double *grad,
                   int32_t *ier);
/* src/laplace/rfmm2dwrap.f:349 */
void rfmm2d_s_d_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double *dipstr,
                   const double *dipvec, double *pot, double *grad,
                   double *hess, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:411 */
void rfmm2d_s_cd_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double *charge,
                    const double *dipstr, const double *dipvec, double *pot,
                    int32_t *ier);
/* src/laplace/rfmm2dwrap.f:473 */
void rfmm2d_s_cd_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double *charge,
                    const double *dipstr, const double *dipvec, double *pot,
                    double *grad, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:536 */
void rfmm2d_s_cd_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double *charge,
                    const double *dipstr, const double *dipvec, double *pot,
                    double *grad, double *hess, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:599 */
void rfmm2d_t_c_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double *charge,
                   const int32_t *nt, const double *targ, double *pottarg,
                   int32_t *ier);
/* src/laplace/rfmm2dwrap.f:659 */
void rfmm2d_t_c_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double *charge,
                   const int32_t *nt, const double *targ, double *pottarg,
                   double *gradtarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:720 */
void rfmm2d_t_c_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double *charge,
                   const int32_t *nt, const double *targ, double *pottarg,
                   double *gradtarg, double *hesstarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:780 */
void rfmm2d_t_d_p_(const double *eps, const int32_t *ns,
                   const double *sources, const double *dipstr,
                   const double *dipvec, const int32_t *nt,
                   const double *targ, double *pottarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:841 */
void rfmm2d_t_d_g_(const double *eps, const int32_t *ns,
                   const double *sources, const double *dipstr,
                   const double *dipvec, const int32_t *nt,
                   const double *targ, double *pottarg, double *gradtarg,
                   int32_t *ier);
/* src/laplace/rfmm2dwrap.f:903 */
void rfmm2d_t_d_h_(const double *eps, const int32_t *ns,
                   const double *sources, const double *dipstr,
                   const double *dipvec, const int32_t *nt,
                   const double *targ, double *pottarg, double *gradtarg,
                   double *hesstarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:964 */
void rfmm2d_t_cd_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double *charge,
                    const double *dipstr, const double *dipvec,
                    const int32_t *nt, const double *targ, double *pottarg,
                    int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1024 */
void rfmm2d_t_cd_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double *charge,
                    const double *dipstr, const double *dipvec,
                    const int32_t *nt, const double *targ, double *pottarg,
                    double *gradtarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1085 */
void rfmm2d_t_cd_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double *charge,
                    const double *dipstr, const double *dipvec,
                    const int32_t *nt, const double *targ, double *pottarg,
                    double *gradtarg, double *hesstarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1148 */
void rfmm2d_st_c_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double *charge, double *pot,
                    const int32_t *nt, const double *targ, double *pottarg,
                    int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1209 */
void rfmm2d_st_c_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double *charge, double *pot,
                    double *grad, const int32_t *nt, const double *targ,
                    double *pottarg, double *gradtarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1272 */
void rfmm2d_st_c_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double *charge, double *pot,
                    double *grad, double *hess, const int32_t *nt,
                    const double *targ, double *pottarg, double *gradtarg,
                    double *hesstarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1335 */
void rfmm2d_st_d_p_(const double *eps, const int32_t *ns,
                    const double *sources, const double *dipstr,
                    const double *dipvec, double *pot, const int32_t *nt,
                    const double *targ, double *pottarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1397 */
void rfmm2d_st_d_g_(const double *eps, const int32_t *ns,
                    const double *sources, const double *dipstr,
                    const double *dipvec, double *pot, double *grad,
                    const int32_t *nt, const double *targ, double *pottarg,
                    double *gradtarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1461 */
void rfmm2d_st_d_h_(const double *eps, const int32_t *ns,
                    const double *sources, const double *dipstr,
                    const double *dipvec, double *pot, double *grad,
                    double *hess, const int32_t *nt, const double *targ,
                    double *pottarg, double *gradtarg, double *hesstarg,
                    int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1525 */
void rfmm2d_st_cd_p_(const double *eps, const int32_t *ns,
                     const double *sources, const double *charge,
                     const double *dipstr, const double *dipvec, double *pot,
                     const int32_t *nt, const double *targ, double *pottarg,
                     int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1586 */
void rfmm2d_st_cd_g_(const double *eps, const int32_t *ns,
                     const double *sources, const double *charge,
                     const double *dipstr, const double *dipvec, double *pot,
                     double *grad, const int32_t *nt, const double *targ,
                     double *pottarg, double *gradtarg, int32_t *ier);
/* src/laplace/rfmm2dwrap.f:1649 */
void rfmm2d_st_cd_h_(const double *eps, const int32_t *ns,
                     const double *sources, const double *charge,
                     const double *dipstr, const double *dipvec, double *pot,
                     double *grad, double *hess, const int32_t *nt,
                     const double *targ, double *pottarg, double *gradtarg,
                     double *hesstarg, int32_t *ier);


/* ===================================================================== */
/* Vectorised wrappers {l,c,h,r}fmm2d_*_vec_: the same 27 flag sets per  */
/* family with a leading nd (number of densities); strengths (nd, n),    */
/* dipvec (nd, 2, n), pot (nd, n), grad (nd, 2, n) or (nd, n) for        */
/* cfmm2d, hess (nd, 3, n) or (nd, n) for cfmm2d.                        */
/* ===================================================================== */
/* src/laplace/lfmm2dwrap_vec.f:31 */
void lfmm2d_s_c_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, double _Complex *pot,
                       int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:91 */
void lfmm2d_s_c_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, double _Complex *pot,
                       double _Complex *grad, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:154 */
void lfmm2d_s_c_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, double _Complex *pot,
                       double _Complex *grad, double _Complex *hess,
                       int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:215 */
void lfmm2d_s_d_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, const double *dipvec,
                       double _Complex *pot, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:276 */
void lfmm2d_s_d_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, const double *dipvec,
                       double _Complex *pot, double _Complex *grad,
                       int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:340 */
void lfmm2d_s_d_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, const double *dipvec,
                       double _Complex *pot, double _Complex *grad,
                       double _Complex *hess, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:401 */
void lfmm2d_s_cd_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        double _Complex *pot, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:461 */
void lfmm2d_s_cd_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        double _Complex *pot, double _Complex *grad,
                        int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:523 */
void lfmm2d_s_cd_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        double _Complex *pot, double _Complex *grad,
                        double _Complex *hess, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:585 */
void lfmm2d_t_c_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:643 */
void lfmm2d_t_c_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       double _Complex *gradtarg, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:704 */
void lfmm2d_t_c_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       double _Complex *gradtarg, double _Complex *hesstarg,
                       int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:763 */
void lfmm2d_t_d_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, const double *dipvec,
                       const int32_t *nt, const double *targ,
                       double _Complex *pottarg, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:822 */
void lfmm2d_t_d_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, const double *dipvec,
                       const int32_t *nt, const double *targ,
                       double _Complex *pottarg, double _Complex *gradtarg,
                       int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:884 */
void lfmm2d_t_d_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, const double *dipvec,
                       const int32_t *nt, const double *targ,
                       double _Complex *pottarg, double _Complex *gradtarg,
                       double _Complex *hesstarg, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:944 */
void lfmm2d_t_cd_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1002 */
void lfmm2d_t_cd_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1062 */
void lfmm2d_t_cd_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        double _Complex *hesstarg, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1126 */
void lfmm2d_st_c_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge, double _Complex *pot,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1185 */
void lfmm2d_st_c_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge, double _Complex *pot,
                        double _Complex *grad, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        double _Complex *gradtarg, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1248 */
void lfmm2d_st_c_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge, double _Complex *pot,
                        double _Complex *grad, double _Complex *hess,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        double _Complex *hesstarg, int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1311 */
void lfmm2d_st_d_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *dipstr, const double *dipvec,
                        double _Complex *pot, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1371 */
void lfmm2d_st_d_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *dipstr, const double *dipvec,
                        double _Complex *pot, double _Complex *grad,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1436 */
void lfmm2d_st_d_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *dipstr, const double *dipvec,
                        double _Complex *pot, double _Complex *grad,
                        double _Complex *hess, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        double _Complex *gradtarg, double _Complex *hesstarg,
                        int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1500 */
void lfmm2d_st_cd_p_vec_(const int32_t *nd, const double *eps,
                         const int32_t *ns, const double *sources,
                         const double _Complex *charge,
                         const double _Complex *dipstr, const double *dipvec,
                         double _Complex *pot, const int32_t *nt,
                         const double *targ, double _Complex *pottarg,
                         int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1560 */
void lfmm2d_st_cd_g_vec_(const int32_t *nd, const double *eps,
                         const int32_t *ns, const double *sources,
                         const double _Complex *charge,
                         const double _Complex *dipstr, const double *dipvec,
                         double _Complex *pot, double _Complex *grad,
                         const int32_t *nt, const double *targ,
                         double _Complex *pottarg, double _Complex *gradtarg,
                         int32_t *ier);
/* src/laplace/lfmm2dwrap_vec.f:1623 */
void lfmm2d_st_cd_h_vec_(const int32_t *nd, const double *eps,
                         const int32_t *ns, const double *sources,
                         const double _Complex *charge,
                         const double _Complex *dipstr, const double *dipvec,
                         double _Complex *pot, double _Complex *grad,
                         double _Complex *hess, const int32_t *nt,
                         const double *targ, double _Complex *pottarg,
                         double _Complex *gradtarg, double _Complex *hesstarg,
                         int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:37 */
void cfmm2d_s_c_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, double _Complex *pot,
                       int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:96 */
void cfmm2d_s_c_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, double _Complex *pot,
                       double _Complex *grad, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:158 */
void cfmm2d_s_c_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, double _Complex *pot,
                       double _Complex *grad, double _Complex *hess,
                       int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:218 */
void cfmm2d_s_d_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, double _Complex *pot,
                       int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:277 */
void cfmm2d_s_d_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, double _Complex *pot,
                       double _Complex *grad, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:339 */
void cfmm2d_s_d_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, double _Complex *pot,
                       double _Complex *grad, double _Complex *hess,
                       int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:398 */
void cfmm2d_s_cd_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, double _Complex *pot,
                        int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:456 */
void cfmm2d_s_cd_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, double _Complex *pot,
                        double _Complex *grad, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:516 */
void cfmm2d_s_cd_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, double _Complex *pot,
                        double _Complex *grad, double _Complex *hess,
                        int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:576 */
void cfmm2d_t_c_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:633 */
void cfmm2d_t_c_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       double _Complex *gradtarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:693 */
void cfmm2d_t_c_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *charge, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       double _Complex *gradtarg, double _Complex *hesstarg,
                       int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:751 */
void cfmm2d_t_d_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:808 */
void cfmm2d_t_d_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       double _Complex *gradtarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:868 */
void cfmm2d_t_d_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double _Complex *dipstr, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       double _Complex *gradtarg, double _Complex *hesstarg,
                       int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:926 */
void cfmm2d_t_cd_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:982 */
void cfmm2d_t_cd_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        double _Complex *gradtarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1040 */
void cfmm2d_t_cd_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge,
                        const double _Complex *dipstr, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        double _Complex *gradtarg, double _Complex *hesstarg,
                        int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1102 */
void cfmm2d_st_c_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge, double _Complex *pot,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1160 */
void cfmm2d_st_c_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge, double _Complex *pot,
                        double _Complex *grad, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        double _Complex *gradtarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1222 */
void cfmm2d_st_c_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *charge, double _Complex *pot,
                        double _Complex *grad, double _Complex *hess,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        double _Complex *hesstarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1284 */
void cfmm2d_st_d_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *dipstr, double _Complex *pot,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1342 */
void cfmm2d_st_d_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *dipstr, double _Complex *pot,
                        double _Complex *grad, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        double _Complex *gradtarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1405 */
void cfmm2d_st_d_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double _Complex *dipstr, double _Complex *pot,
                        double _Complex *grad, double _Complex *hess,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        double _Complex *hesstarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1467 */
void cfmm2d_st_cd_p_vec_(const int32_t *nd, const double *eps,
                         const int32_t *ns, const double *sources,
                         const double _Complex *charge,
                         const double _Complex *dipstr, double _Complex *pot,
                         const int32_t *nt, const double *targ,
                         double _Complex *pottarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1525 */
void cfmm2d_st_cd_g_vec_(const int32_t *nd, const double *eps,
                         const int32_t *ns, const double *sources,
                         const double _Complex *charge,
                         const double _Complex *dipstr, double _Complex *pot,
                         double _Complex *grad, const int32_t *nt,
                         const double *targ, double _Complex *pottarg,
                         double _Complex *gradtarg, int32_t *ier);
/* src/laplace/cfmm2dwrap_vec.f:1586 */
void cfmm2d_st_cd_h_vec_(const int32_t *nd, const double *eps,
                         const int32_t *ns, const double *sources,
                         const double _Complex *charge,
                         const double _Complex *dipstr, double _Complex *pot,
                         double _Complex *grad, double _Complex *hess,
                         const int32_t *nt, const double *targ,
                         double _Complex *pottarg, double _Complex *gradtarg,
                         double _Complex *hesstarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:6 */
void hfmm2d_s_c_p_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *charge,
                       double _Complex *pot, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:70 */
void hfmm2d_s_c_g_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *charge,
                       double _Complex *pot, double _Complex *grad,
                       int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:138 */
void hfmm2d_s_c_h_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *charge,
                       double _Complex *pot, double _Complex *grad,
                       double _Complex *hess, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:205 */
void hfmm2d_s_d_p_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *dipstr,
                       const double *dipvec, double _Complex *pot,
                       int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:270 */
void hfmm2d_s_d_g_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *dipstr,
                       const double *dipvec, double _Complex *pot,
                       double _Complex *grad, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:339 */
void hfmm2d_s_d_h_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *dipstr,
                       const double *dipvec, double _Complex *pot,
                       double _Complex *grad, double _Complex *hess,
                       int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:407 */
void hfmm2d_s_cd_p_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        double _Complex *pot, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:472 */
void hfmm2d_s_cd_g_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        double _Complex *pot, double _Complex *grad,
                        int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:540 */
void hfmm2d_s_cd_h_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        double _Complex *pot, double _Complex *grad,
                        double _Complex *hess, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:609 */
void hfmm2d_t_c_p_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *charge,
                       const int32_t *nt, const double *targ,
                       double _Complex *pottarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:671 */
void hfmm2d_t_c_g_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *charge,
                       const int32_t *nt, const double *targ,
                       double _Complex *pottarg, double _Complex *gradtarg,
                       int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:737 */
void hfmm2d_t_c_h_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *charge,
                       const int32_t *nt, const double *targ,
                       double _Complex *pottarg, double _Complex *gradtarg,
                       double _Complex *hesstarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:803 */
void hfmm2d_t_d_p_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *dipstr,
                       const double *dipvec, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:866 */
void hfmm2d_t_d_g_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *dipstr,
                       const double *dipvec, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       double _Complex *gradtarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:933 */
void hfmm2d_t_d_h_vec_(const int32_t *nd, const double *eps,
                       const double _Complex *zk, const int32_t *ns,
                       const double *sources, const double _Complex *dipstr,
                       const double *dipvec, const int32_t *nt,
                       const double *targ, double _Complex *pottarg,
                       double _Complex *gradtarg, double _Complex *hesstarg,
                       int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1000 */
void hfmm2d_t_cd_p_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1063 */
void hfmm2d_t_cd_g_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1129 */
void hfmm2d_t_cd_h_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *charge,
                        const double _Complex *dipstr, const double *dipvec,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        double _Complex *hesstarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1196 */
void hfmm2d_st_c_p_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *charge,
                        double _Complex *pot, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1259 */
void hfmm2d_st_c_g_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *charge,
                        double _Complex *pot, double _Complex *grad,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1326 */
void hfmm2d_st_c_h_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *charge,
                        double _Complex *pot, double _Complex *grad,
                        double _Complex *hess, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        double _Complex *gradtarg, double _Complex *hesstarg,
                        int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1393 */
void hfmm2d_st_d_p_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *dipstr,
                        const double *dipvec, double _Complex *pot,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1457 */
void hfmm2d_st_d_g_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *dipstr,
                        const double *dipvec, double _Complex *pot,
                        double _Complex *grad, const int32_t *nt,
                        const double *targ, double _Complex *pottarg,
                        double _Complex *gradtarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1525 */
void hfmm2d_st_d_h_vec_(const int32_t *nd, const double *eps,
                        const double _Complex *zk, const int32_t *ns,
                        const double *sources, const double _Complex *dipstr,
                        const double *dipvec, double _Complex *pot,
                        double _Complex *grad, double _Complex *hess,
                        const int32_t *nt, const double *targ,
                        double _Complex *pottarg, double _Complex *gradtarg,
                        double _Complex *hesstarg, int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1593 */
void hfmm2d_st_cd_p_vec_(const int32_t *nd, const double *eps,
                         const double _Complex *zk, const int32_t *ns,
                         const double *sources, const double _Complex *charge,
                         const double _Complex *dipstr, const double *dipvec,
                         double _Complex *pot, const int32_t *nt,
                         const double *targ, double _Complex *pottarg,
                         int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1657 */
void hfmm2d_st_cd_g_vec_(const int32_t *nd, const double *eps,
                         const double _Complex *zk, const int32_t *ns,
                         const double *sources, const double _Complex *charge,
                         const double _Complex *dipstr, const double *dipvec,
                         double _Complex *pot, double _Complex *grad,
                         const int32_t *nt, const double *targ,
                         double _Complex *pottarg, double _Complex *gradtarg,
                         int32_t *ier);
/* src/helmholtz/hfmm2dwrap_vec.f:1724 */
void hfmm2d_st_cd_h_vec_(const int32_t *nd, const double *eps,
                         const double _Complex *zk, const int32_t *ns,
                         const double *sources, const double _Complex *charge,
                         const double _Complex *dipstr, const double *dipvec,
                         double _Complex *pot, double _Complex *grad,
                         double _Complex *hess, const int32_t *nt,
                         const double *targ, double _Complex *pottarg,
                         double _Complex *gradtarg, double _Complex *hesstarg,
                         int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:36 */
void rfmm2d_s_c_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *charge, double *pot, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:96 */
void rfmm2d_s_c_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *charge, double *pot, double *grad,
                       int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:159 */
void rfmm2d_s_c_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *charge, double *pot, double *grad,
                       double *hess, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:220 */
void rfmm2d_s_d_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *dipstr, const double *dipvec,
                       double *pot, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:281 */
void rfmm2d_s_d_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *dipstr, const double *dipvec,
                       double *pot, double *grad, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:345 */
void rfmm2d_s_d_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *dipstr, const double *dipvec,
                       double *pot, double *grad, double *hess, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:406 */
void rfmm2d_s_cd_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *charge, const double *dipstr,
                        const double *dipvec, double *pot, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:466 */
void rfmm2d_s_cd_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *charge, const double *dipstr,
                        const double *dipvec, double *pot, double *grad,
                        int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:528 */
void rfmm2d_s_cd_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *charge, const double *dipstr,
                        const double *dipvec, double *pot, double *grad,
                        double *hess, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:590 */
void rfmm2d_t_c_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *charge, const int32_t *nt,
                       const double *targ, double *pottarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:648 */
void rfmm2d_t_c_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *charge, const int32_t *nt,
                       const double *targ, double *pottarg, double *gradtarg,
                       int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:709 */
void rfmm2d_t_c_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *charge, const int32_t *nt,
                       const double *targ, double *pottarg, double *gradtarg,
                       double *hesstarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:768 */
void rfmm2d_t_d_p_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *dipstr, const double *dipvec,
                       const int32_t *nt, const double *targ, double *pottarg,
                       int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:827 */
void rfmm2d_t_d_g_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *dipstr, const double *dipvec,
                       const int32_t *nt, const double *targ, double *pottarg,
                       double *gradtarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:889 */
void rfmm2d_t_d_h_vec_(const int32_t *nd, const double *eps,
                       const int32_t *ns, const double *sources,
                       const double *dipstr, const double *dipvec,
                       const int32_t *nt, const double *targ, double *pottarg,
                       double *gradtarg, double *hesstarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:949 */
void rfmm2d_t_cd_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *charge, const double *dipstr,
                        const double *dipvec, const int32_t *nt,
                        const double *targ, double *pottarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1007 */
void rfmm2d_t_cd_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *charge, const double *dipstr,
                        const double *dipvec, const int32_t *nt,
                        const double *targ, double *pottarg, double *gradtarg,
                        int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1067 */
void rfmm2d_t_cd_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *charge, const double *dipstr,
                        const double *dipvec, const int32_t *nt,
                        const double *targ, double *pottarg, double *gradtarg,
                        double *hesstarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1131 */
void rfmm2d_st_c_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *charge, double *pot, const int32_t *nt,
                        const double *targ, double *pottarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1190 */
void rfmm2d_st_c_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *charge, double *pot, double *grad,
                        const int32_t *nt, const double *targ,
                        double *pottarg, double *gradtarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1253 */
void rfmm2d_st_c_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *charge, double *pot, double *grad,
                        double *hess, const int32_t *nt, const double *targ,
                        double *pottarg, double *gradtarg, double *hesstarg,
                        int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1316 */
void rfmm2d_st_d_p_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *dipstr, const double *dipvec,
                        double *pot, const int32_t *nt, const double *targ,
                        double *pottarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1376 */
void rfmm2d_st_d_g_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *dipstr, const double *dipvec,
                        double *pot, double *grad, const int32_t *nt,
                        const double *targ, double *pottarg, double *gradtarg,
                        int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1441 */
void rfmm2d_st_d_h_vec_(const int32_t *nd, const double *eps,
                        const int32_t *ns, const double *sources,
                        const double *dipstr, const double *dipvec,
                        double *pot, double *grad, double *hess,
                        const int32_t *nt, const double *targ,
                        double *pottarg, double *gradtarg, double *hesstarg,
                        int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1505 */
void rfmm2d_st_cd_p_vec_(const int32_t *nd, const double *eps,
                         const int32_t *ns, const double *sources,
                         const double *charge, const double *dipstr,
                         const double *dipvec, double *pot, const int32_t *nt,
                         const double *targ, double *pottarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1565 */
void rfmm2d_st_cd_g_vec_(const int32_t *nd, const double *eps,
                         const int32_t *ns, const double *sources,
                         const double *charge, const double *dipstr,
                         const double *dipvec, double *pot, double *grad,
                         const int32_t *nt, const double *targ,
                         double *pottarg, double *gradtarg, int32_t *ier);
/* src/laplace/rfmm2dwrap_vec.f:1628 */
void rfmm2d_st_cd_h_vec_(const int32_t *nd, const double *eps,
                         const int32_t *ns, const double *sources,
                         const double *charge, const double *dipstr,
                         const double *dipvec, double *pot, double *grad,
                         double *hess, const int32_t *nt, const double *targ,
                         double *pottarg, double *gradtarg, double *hesstarg,
                         int32_t *ier);

/* ===================================================================== */
/* Guru drivers (full flag sets, nd densities).  iper is ignored and set */
/* to 0, as in the reference (src/laplace/cfmm2d.f:150).                 */
/* ===================================================================== */
/* src/laplace/lfmm2d.f:29 */
void lfmm2d_(const int32_t *nd, const double *eps, const int32_t *ns,
             const double *sources, const int32_t *ifcharge,
             const double _Complex *charge, const int32_t *ifdipole,
             const double _Complex *dipstr, const double *dipvec,
             int32_t *iper, const int32_t *ifpgh, double _Complex *pot,
             double _Complex *grad, double _Complex *hess, const int32_t *nt,
             const double *targ, const int32_t *ifpghtarg,
             double _Complex *pottarg, double _Complex *gradtarg,
             double _Complex *hesstarg, int32_t *ier);
/* src/laplace/cfmm2d.f:23, c_translation/src/cfmm2d.c:1053 */
void cfmm2d_(const int32_t *nd, const double *eps, const int32_t *ns,
             const double *sources, const int32_t *ifcharge,
             const double _Complex *charge, const int32_t *ifdipole,
             const double _Complex *dipstr, int32_t *iper,
             const int32_t *ifpgh, double _Complex *pot, double _Complex *grad,
             double _Complex *hess, const int32_t *nt, const double *targ,
             const int32_t *ifpghtarg, double _Complex *pottarg,
             double _Complex *gradtarg, double _Complex *hesstarg,
             int32_t *ier);
/* src/helmholtz/hfmm2d.f:19, c_translation/src/hfmm2d.c:1529 */
void hfmm2d_(const int32_t *nd, const double *eps, const double _Complex *zk,
             const int32_t *ns, const double *sources,
             const int32_t *ifcharge, const double _Complex *charge,
             const int32_t *ifdipole, const double _Complex *dipstr,
             const double *dipvec, int32_t *iper, const int32_t *ifpgh,
             double _Complex *pot, double _Complex *grad,
             double _Complex *hess, const int32_t *nt, const double *targ,
             const int32_t *ifpghtarg, double _Complex *pottarg,
             double _Complex *gradtarg, double _Complex *hesstarg,
             int32_t *ier);

/* src/laplace/rfmm2d.f:27 (real charge(nd,ns), dipstr(nd,ns),
 * dipvec(nd,2,ns); real pot(nd,*), grad(nd,2,*), hess(nd,3,*)) */
void rfmm2d_(const int32_t *nd, const double *eps, const int32_t *ns,
             const double *sources, const int32_t *ifcharge,
             const double *charge, const int32_t *ifdipole,
             const double *dipstr, const double *dipvec, int32_t *iper,
             const int32_t *ifpgh, double *pot, double *grad, double *hess,
             const int32_t *nt, const double *targ, const int32_t *ifpghtarg,
             double *pottarg, double *gradtarg, double *hesstarg,
             int32_t *ier);

/* Drivers with caller-chosen leaf capacity ndiv, subdivision rule idivflag
 * (0 sources, 1 targets, 2 both), near-field switch ifnear and per-step
 * timings timeinfo(8) (MATLAB path, matlab/fmm2d.c:1256-1286). */
/* src/laplace/lfmm2d_ndiv.f:29, c_translation/src/lfmm2d_ndiv.c:57 */
void lfmm2d_ndiv_(const int32_t *nd, const double *eps, const int32_t *ns,
                  const double *sources, const int32_t *ifcharge,
                  const double _Complex *charge, const int32_t *ifdipole,
                  const double _Complex *dipstr, const double *dipvec,
                  int32_t *iper, const int32_t *ifpgh, double _Complex *pot,
                  double _Complex *grad, double _Complex *hess,
                  const int32_t *nt, const double *targ,
                  const int32_t *ifpghtarg, double _Complex *pottarg,
                  double _Complex *gradtarg, double _Complex *hesstarg,
                  const int32_t *ndiv, const int32_t *idivflag,
                  const int32_t *ifnear, double *timeinfo, int32_t *ier);
/* src/laplace/cfmm2d_ndiv.f:23, c_translation/src/cfmm2d_ndiv.c:94 */
void cfmm2d_ndiv_(const int32_t *nd, const double *eps, const int32_t *ns,
                  const double *sources, const int32_t *ifcharge,
                  const double _Complex *charge, const int32_t *ifdipole,
                  const double _Complex *dipstr, int32_t *iper,
                  const int32_t *ifpgh, double _Complex *pot,
                  double _Complex *grad, double _Complex *hess,
                  const int32_t *nt, const double *targ,
                  const int32_t *ifpghtarg, double _Complex *pottarg,
                  double _Complex *gradtarg, double _Complex *hesstarg,
                  const int32_t *ndiv, const int32_t *idivflag,
                  const int32_t *ifnear, double *timeinfo, int32_t *ier);
/* src/helmholtz/hfmm2d_ndiv.f:19, c_translation/src/hfmm2d_ndiv.c:68 */
void hfmm2d_ndiv_(const int32_t *nd, const double *eps,
                  const double _Complex *zk, const int32_t *ns,
                  const double *sources, const int32_t *ifcharge,
                  const double _Complex *charge, const int32_t *ifdipole,
                  const double _Complex *dipstr, const double *dipvec,
                  int32_t *iper, const int32_t *ifpgh, double _Complex *pot,
                  double _Complex *grad, double _Complex *hess,
                  const int32_t *nt, const double *targ,
                  const int32_t *ifpghtarg, double _Complex *pottarg,
                  double _Complex *gradtarg, double _Complex *hesstarg,
                  const int32_t *ndiv, const int32_t *idivflag,
                  const int32_t *ifnear, double *timeinfo, int32_t *ier);

/* src/laplace/rfmm2d_ndiv.f:27, c_translation/src/rfmm2d_ndiv.c:51 */
void rfmm2d_ndiv_(const int32_t *nd, const double *eps, const int32_t *ns,
                  const double *sources, const int32_t *ifcharge,
                  const double *charge, const int32_t *ifdipole,
                  const double *dipstr, const double *dipvec, int32_t *iper,
                  const int32_t *ifpgh, double *pot, double *grad,
                  double *hess, const int32_t *nt, const double *targ,
                  const int32_t *ifpghtarg, double *pottarg,
                  double *gradtarg, double *hesstarg, const int32_t *ndiv,
                  const int32_t *idivflag, const int32_t *ifnear,
                  double *timeinfo, int32_t *ier);

/* bind(c) entry, src/helmholtz_c.f03:5-15: eps, zk and ns by value, ns
 * and ier 64-bit (c_int64_t).  C++ callers pass zk as a struct of two
 * doubles, which has the calling convention of double _Complex. */
#ifdef __cplusplus
typedef struct { double re, im; } fmm2d_b200_zk_t;
void hfmm2d_s_c_p(double eps, fmm2d_b200_zk_t zk, int64_t ns,
                  const double *sources, const double *charge, double *pot,
                  int64_t *ier);
#else
void hfmm2d_s_c_p(double eps, double _Complex zk, int64_t ns,
                  const double *sources, const double _Complex *charge,
                  double _Complex *pot, int64_t *ier);
#endif

/* ===================================================================== */
/* Library entry points with no counterpart in the reference.           */
/* ===================================================================== */
const char *fmm2d_b200_version(void);
/* Message of the last failed call (any thread); returns its length. */
int fmm2d_b200_last_error(char *buf, int len);
/* Precision policy of later calls: 0 auto (mixed when eps >= 0.5e-6, else
 * all-FP64), 1 all-FP64, 2 mixed, 3 split (Laplace / Cauchy: every pass
 * FP64 except the M2L's terms of high total order, which run as TF32 x 3 on
 * the tensor cores; Helmholtz: all-FP64).
 * Also FMM2D_B200_PRECISION=auto|fp64|mixed|split. */
int fmm2d_b200_set_precision(int mode);
/* Run the calling thread's later calls on a caller-owned cudaStream_t. */
int fmm2d_b200_set_stream(void *stream);
int fmm2d_b200_reset_stream(void);
/* Return cached device workspace of the current device to the driver. */
int fmm2d_b200_release_memory(void);
/* Host-only rules: expansion order (l2dterms, c_translation/src/l2dterms.c:26)
 * and leaf capacity (src/laplace/lndiv2d.f:1) for a precision. */
int fmm2d_b200_laplace_nterms(double eps);
int fmm2d_b200_leaf_capacity(double eps, int ns, int nt);
/* Leaf capacity of the mixed-precision complex-Laplace mode (held to eps
 * against the direct sum, not to the reference's tree; the Cauchy form keeps
 * the reference's tree, whose branch terms its potential carries) for order
 * nterms.  Default: 24 for nterms >= 14, 40 below (measured on a B200).
 * ndiv = 0 clears a setting for that order; ndiv < 0 selects the
 * reference's rule (lndiv2d) for the orders without a setting.  The
 * environment variable FMM2D_B200_MIXED_NDIV overrides all of these.  The
 * second function returns the capacity a mixed call at eps would use. */
int fmm2d_b200_set_leaf_capacity(int nterms, int ndiv);
int fmm2d_b200_mixed_leaf_capacity(double eps, int ns, int nt);
/* Form of the mixed-mode M2L for order nterms: 0 tensor-core windows on the
 * dense levels and tensor-core slot tables on the rest (default), 1 slot
 * tables on the tensor cores only, 2 slot tables on the CUDA cores (FP32).
 * FMM2D_B200_M2L=tile|simt overrides. */
int fmm2d_b200_set_m2l_form(int nterms, int form);
int fmm2d_b200_m2l_form(int nterms);
/* Autotuner of the mixed-precision path for the order of eps: times full
 * evaluations (kernel 0 = lfmm2d, 1 = cfmm2d; nd = 1; the given flags) of
 * ns sources and nt targets -- the caller's points (host or device arrays,
 * 2 x n), or seeded uniform points in [0,1]^2 where a pointer is null --
 * over leaf capacities {12 .. 64} and the M2L forms above, and keeps the
 * fastest pair for that order (fmm2d_b200_set_leaf_capacity /
 * fmm2d_b200_set_m2l_form; the leaf capacity applies to lfmm2d, whose
 * mixed mode is free of the reference's tree).  Returns 0 and the choice
 * with its time per evaluation in ms, or 4. */
int fmm2d_b200_autotune(int kernel, double eps, int ns, const double *sources,
                        int nt, const double *targ, int ifcharge,
                        int ifdipole, int ifpgh, int ifpghtarg,
                        int *best_ndiv, int *best_form, double *best_ms);

/* Resident geometry (no counterpart in the reference): a plan keeps the
 * tree, its lists and the points in tree order of one lfmm2d (kernel 0) or
 * cfmm2d (kernel 1) problem on the device -- the geometry the drivers
 * rebuild on every call -- so that evaluating new strengths on the same
 * points (an iterative solver's operator applications) skips the tree.
 * Arguments as the guru drivers (src/laplace/lfmm2d.f:29,
 * src/laplace/cfmm2d.f:23) without the strengths and outputs; eps and the
 * precision policy in force at creation are fixed.  plan_eval takes the
 * strengths (charge and dipstr as (nd, ns) complex, dipvec (nd, 2, ns))
 * and overwrites the outputs in the guru drivers' layouts; host or device
 * arrays.  The first evaluation runs eagerly; the later ones replay a CUDA
 * graph of the whole evaluation captured over plan-owned staging buffers
 * (FMM2D_B200_PLAN_GRAPH=0 keeps them eager).  A plan is used on the
 * device it was made on; evaluations of one plan are serialised.  Each
 * returns 0 or 4; plan_uses_graph returns 1 once evaluations replay the
 * graph. */
int fmm2d_b200_plan_create(int kernel, int nd, double eps, int ns,
                           const double *sources, int ifcharge, int ifdipole,
                           int ifpgh, int nt, const double *targ,
                           int ifpghtarg, void **plan);
int fmm2d_b200_plan_eval(void *plan, const double _Complex *charge,
                         const double _Complex *dipstr, const double *dipvec,
                         double _Complex *pot, double _Complex *grad,
                         double _Complex *hess, double _Complex *pottarg,
                         double _Complex *gradtarg, double _Complex *hesstarg);
int fmm2d_b200_plan_destroy(void *plan);
int fmm2d_b200_plan_uses_graph(void *plan);

/* Batch of independent problems (no counterpart in the reference): nprob
 * lfmm2d (kernel 0) or cfmm2d (kernel 1) evaluations with nd = 1 and the
 * same eps and output flags, run as one forest of trees -- one launch per
 * level and pass for the whole batch.  Problem k has ns[k] sources
 * sources[k] (2 x ns[k]) with charge[k] / dipstr[k] (ns[k] complex;
 * pass charge = NULL or dipstr = NULL for none) and dipvec[k] (2 x ns[k],
 * lfmm2d dipoles), nt[k] targets targ[k] (nt may be NULL: no targets), and
 * its outputs in pot[k], grad[k], hess[k], pottarg[k], ... in the guru
 * drivers' layouts (overwritten).  Host or device arrays.  Each problem is
 * translated so that its bounding square is centred at the origin and all
 * trees share the largest root size, so the trees differ from the
 * one-problem calls' and the results agree with them to the accuracy eps
 * asks for, not to the bit.  Returns 0 or 4. */
int fmm2d_b200_fmm2d_batch(int kernel, int nprob, double eps, const int *ns,
                           const double *const *sources,
                           const double _Complex *const *charge,
                           const double _Complex *const *dipstr,
                           const double *const *dipvec, int ifpgh,
                           double _Complex *const *pot,
                           double _Complex *const *grad,
                           double _Complex *const *hess, const int *nt,
                           const double *const *targ, int ifpghtarg,
                           double _Complex *const *pottarg,
                           double _Complex *const *gradtarg,
                           double _Complex *const *hesstarg);

/* Direct sums on the GPU, incrementing the outputs (the reference's
 * l2d_direct* / c2d_direct* kernels, src/laplace/lapkernels2d.f,
 * src/laplace/cauchykernels2d.f): every target against every source. */
int fmm2d_b200_l2d_direct(int nd, int ns, const double *sources,
                          int ifcharge, const double _Complex *charge,
                          int ifdipole, const double _Complex *dipstr,
                          const double *dipvec, int nt, const double *targ,
                          int ifpgh, double _Complex *pot,
                          double _Complex *grad, double _Complex *hess,
                          double thresh);
int fmm2d_b200_c2d_direct(int nd, int ns, const double *sources,
                          int ifcharge, const double _Complex *charge,
                          int ifdipole, const double _Complex *dipstr, int nt,
                          const double *targ, int ifpgh, double _Complex *pot,
                          double _Complex *grad, double _Complex *hess,
                          double thresh);

/* Helmholtz direct sum (h2d_direct*, c_translation/src/helmkernels2d.c),
 * zk = {re, im}: increments pot(nd,nt), grad(nd,2,nt), hess(nd,3,nt);
 * pairs with |zk r| below thresh are skipped (<= for charge-only
 * potentials, < otherwise, as the reference kernels do). */
int fmm2d_b200_h2d_direct(int nd, const double *zk, int ns,
                          const double *sources, int ifcharge,
                          const double _Complex *charge, int ifdipole,
                          const double _Complex *dipstr, const double *dipvec,
                          int nt, const double *targ, int ifpgh,
                          double _Complex *pot, double _Complex *grad,
                          double _Complex *hess, double thresh);

/* Host-only Helmholtz helpers: the expansion order of a box
 * (h2dterms, c_translation/src/h2dterms.c:19; -1 when above 50000),
 * H0 and H1 at n points (z[2k], z[2k+1]) -> out[4k..4k+3], and the scaled
 * sequences H_k(z) rscale^k (h2dall, h2dcommon.c:35) and J_k(z) / rscale^k
 * (jbessel2d, cdjseval2d.c:11), k = 0..n, as interleaved complex. */
int fmm2d_b200_helm_nterms(double bsize, double zk_re, double zk_im,
                           double eps);
void fmm2d_b200_hankel01(int n, const double *z, double *out);
void fmm2d_b200_helm_hvec(int n, double z_re, double z_im, double rscale,
                          double *out);
void fmm2d_b200_helm_jvec(int n, double z_re, double z_im, double rscale,
                          double *out);

/* No counterpart in the reference.  fmm2d_b200_l2d_direct for callers
 * that cannot have device memory allocated for them (GPU memory owned by
 * another allocator or a fixed budget; callers that cannot accept an
 * allocation call's possible device synchronization).  Same arguments plus
 * a stream; device arrays of the current device only (host arrays, another
 * device's arrays and NULL arrays the flags require give ier = 4); scratch
 * is a fixed 4 MiB device array (nd * nt * outputs <= 262144, outputs = 1,
 * 3 or 6), held by every GPU that loads the library.  The first call on a
 * device sets the array up and should come before any stream capture; the
 * address it looks up is kept for the process, so the entry point must not
 * be used on a device after cudaDeviceReset.  Calls that overlap on the GPU
 * race on the shared array.  Returns after `stream` has finished the call. */
int fmm2d_b200_l2d_direct_noalloc(int nd, int ns, const double *sources,
                                  int ifcharge, const double _Complex *charge,
                                  int ifdipole, const double _Complex *dipstr,
                                  const double *dipvec, int nt,
                                  const double *targ, int ifpgh,
                                  double _Complex *pot, double _Complex *grad,
                                  double _Complex *hess, double thresh,
                                  void *stream);

/* Request loop for many independent evaluations on one GPU (no
 * counterpart in the reference).  `slots` worker threads, each on its own
 * stream, take queued requests whose estimated device footprint fits into
 * the HBM budget left (bytes), so requests that arrive while others run
 * are admitted as slots and memory free up and their work overlaps on the
 * device.  A request larger than the whole budget finishes at once with
 * ier = 4.  Arrays follow the guru drivers (host or device memory) and must
 * stay valid until fmm2d_b200_server_wait returns for the ticket. */
typedef struct {
    int kernel; /* 0 lfmm2d, 1 cfmm2d, 2 hfmm2d */
    int nd;
    double eps;
    double zk[2];
    int ns;
    const double *sources;
    int ifcharge;
    const double *charge;
    int ifdipole;
    const double *dipstr;
    const double *dipvec; /* lfmm2d / hfmm2d only */
    int ifpgh;
    double *pot, *grad, *hess;
    int nt;
    const double *targ;
    int ifpghtarg;
    double *pottarg, *gradtarg, *hesstarg;
    int precision; /* 0 auto (mixed when eps >= 1e-6), 1 all-FP64, 2 mixed */
} fmm2d_b200_request;
void *fmm2d_b200_server_create(int slots, double hbm_budget_bytes);
/* Returns a ticket (>= 0), or -1 for an invalid request. */
long long fmm2d_b200_server_submit(void *server, const fmm2d_b200_request *req);
/* Waits for a ticket; returns its ier and, if times_ms is not null, the
 * milliseconds spent queued, running and in total. */
int fmm2d_b200_server_wait(void *server, long long ticket, double *times_ms);
/* bytes in use, peak bytes in use, queued, running, rejected, peak running */
void fmm2d_b200_server_stats(void *server, double *out6);
/* The footprint estimate the server admits a request by (bytes). */
double fmm2d_b200_request_bytes(const fmm2d_b200_request *req);
/* Finishes the queued requests, then stops the workers. */
void fmm2d_b200_server_destroy(void *server);
/* Requests that ran in batches of two or more so far: a worker that takes
 * a small lfmm2d request (nd = 1, at most 50,000 points) also takes the
 * queued requests of the same eps, precision, strengths and output flags
 * that fit the budget (up to 64 requests, 200,000 points) and evaluates
 * them as one forest (fmm2d_b200_fmm2d_batch); their results agree with
 * the alone ones to the requested eps.  FMM2D_B200_SERVE_BATCH=0, read when
 * the server is made, turns this off. */
long long fmm2d_b200_server_batched(void *server);

/* Quadtree inspection in the reference's layout (pts_tree_mem/build/sort,
 * src/common/pts_tree2d.f:34,406,1222; computelists,
 * src/common/tree_routs2d.f:486). */
int fmm2d_b200_tree_build(const double *sources, int ns, const double *targ,
                          int nt, int ndiv, int idivflag, void **handle);
int fmm2d_b200_tree_sizes(void *handle, int *nlevels, int *nboxes,
                          int *ltree);
int fmm2d_b200_tree_export(void *handle, int *itree, int *iptr,
                           double *centers, double *boxsize, int *isrc,
                           int *isrcse, int *itarg, int *itargse);
int fmm2d_b200_tree_lists(void *handle, int *nlist1, int *list1,
                          int *nlist2, int *list2, int *nlist3, int *list3,
                          int *nlist4, int *list4);
void fmm2d_b200_tree_free(void *handle);

/* Failure injection for tests (no counterpart in the reference; host side
 * only, no GPU fault).  inject_alloc_failure: the nth device allocation from
 * now fails as out of memory, so the call returns ier = 4 (the reference's
 * allocation-failure code, src/helmholtz/hfmm2d.f:374-381); 0 turns it off.
 * inject_tc_stall: the tensor-core M2L kernels issue no MMAs and their
 * bounded waits give up after wait_ms, so a mixed-mode call returns ier = 4;
 * on = 0 restores the normal limit.  device_bytes_in_use: bytes of the
 * device's memory pool held by live allocations (to check that a failed
 * call released its workspace). */
int fmm2d_b200_inject_alloc_failure(long long nth);
int fmm2d_b200_inject_tc_stall(int on, double wait_ms);
int fmm2d_b200_device_bytes_in_use(unsigned long long *bytes);

/* Measurement helpers. */
int fmm2d_b200_set_profiling(int on);
int fmm2d_b200_last_profile(char *buf, int len);
unsigned long long fmm2d_b200_launch_count(void);
double fmm2d_b200_fp64_peak_tflops(void);
double fmm2d_b200_fp32_peak_tflops(void);
/* Dense tcgen05.mma kind::tf32 rate (128 x 256 x 8 MMAs, FP32
 * accumulation, one CTA per SM), TFLOP/s; 0 on failure. */
double fmm2d_b200_tf32_peak_tflops(void);

#ifdef __cplusplus
}
#undef _Complex
#endif
#endif /* FMM2D_B200_H */
