/*
 * fmm2d_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * An independent CPU restatement of what the fmm2d evaluation path
 * computes, used by tests/ and by bench.py's cpu_baseline leg as the
 * checker.  Nothing in the GPU library links or calls this file.
 *
 * It restates, from the reference's definitions:
 *   - the complex-Laplace direct sums (src/laplace/lapkernels2d.f,
 *     c_translation/src/lapkernels2d.c:19-494):
 *        u(x)  = sum_j q_j log|x-y_j| - d_j (v_j . (x-y_j)) / |x-y_j|^2
 *        grad  = (du/dx, du/dy),  hess = (u_xx, u_xy, u_yy);
 *   - the Cauchy direct sums (src/laplace/cauchykernels2d.f,
 *     c_translation/src/cauchykernels2d.c:31-442), z = x - y as complex:
 *        pot  += q log|z| + d / z,  grad += q / z - d / z^2,
 *        hess += -q / z^2 + 2 d / z^3;
 *   - the eps -> leaf capacity table (src/laplace/lndiv2d.f:1-39) and the
 *     eps -> expansion order rule (c_translation/src/l2dterms.c:26-67).
 * Pairs closer than `thresh` are skipped, as the reference kernels do.
 *
 * Outputs are INCREMENTED (like the reference kernels).  Complex arrays are
 * interleaved (re, im) doubles; layouts are the reference's column-major
 * ones with nd = 1: grad(2, n), hess(3, n) for the Laplace form and
 * grad(n), hess(n) for the Cauchy form.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b)
{
    cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cplx cscale(cplx a, double s)
{
    cplx r = {a.re * s, a.im * s};
    return r;
}
static inline void cacc(double *out, cplx v)
{
    out[0] += v.re;
    out[1] += v.im;
}

/* src/laplace/lndiv2d.f:1-39 */
int oracle_lndiv2d(double eps, int ns, int nt)
{
    if (eps >= 0.5e0) return 3;
    if (eps >= 0.5e-1) return 5;
    if (eps >= 0.5e-2) return 8;
    if (eps >= 0.5e-3) return 10;
    if (eps >= 0.5e-6) return 15;
    if (eps >= 0.5e-9) return 20;
    if (eps >= 0.5e-12) return 25;
    if (eps >= 0.5e-15) return 45;
    return ns + nt;
}

/* c_translation/src/l2dterms.c:26-67: the first j >= 2 with
 * (sqrt(2)/2)^j / 1.5^(j+1) < eps, else 1. */
int oracle_l2dterms(double eps)
{
    for (int j = 2; j <= 100; j++) {
        double t = pow(sqrt(2.0) / 2.0, (double)j) / pow(1.5, (double)(j + 1));
        if (t < eps) return j;
    }
    return 1;
}

/*
 * Complex-Laplace (lfmm2d) direct sum over all sources for targets
 * [t0, t1).  ifpgh: 1 pot, 2 pot+grad, 3 pot+grad+hess.
 */
void oracle_l2d_direct(int ns, const double *src, int ifcharge,
                       const double *charge, int ifdipole,
                       const double *dipstr, const double *dipvec,
                       int t0, int t1, const double *targ, int ifpgh,
                       double *pot, double *grad, double *hess, double thresh)
{
    double th2 = thresh * thresh;
    for (int j = t0; j < t1; j++) {
        for (int i = 0; i < ns; i++) {
            double dx = targ[2 * j] - src[2 * i];
            double dy = targ[2 * j + 1] - src[2 * i + 1];
            double r2 = dx * dx + dy * dy;
            if (r2 <= th2) continue;
            double r4 = r2 * r2;
            if (ifcharge) {
                cplx q = {charge[2 * i], charge[2 * i + 1]};
                cacc(&pot[2 * j], cscale(q, 0.5 * log(r2)));
                if (ifpgh >= 2) {
                    cacc(&grad[4 * j], cscale(q, dx / r2));
                    cacc(&grad[4 * j + 2], cscale(q, dy / r2));
                }
                if (ifpgh >= 3) {
                    cacc(&hess[6 * j], cscale(q, (r2 - 2 * dx * dx) / r4));
                    cacc(&hess[6 * j + 2], cscale(q, -2 * dx * dy / r4));
                    cacc(&hess[6 * j + 4], cscale(q, (r2 - 2 * dy * dy) / r4));
                }
            }
            if (ifdipole) {
                cplx d = {dipstr[2 * i], dipstr[2 * i + 1]};
                double v1 = dipvec[2 * i], v2 = dipvec[2 * i + 1];
                double vr = v1 * dx + v2 * dy;
                /* phi = -(v . r) / r^2 */
                cacc(&pot[2 * j], cscale(d, -vr / r2));
                if (ifpgh >= 2) {
                    /* d/dx [-(v.r)/r^2] = -v1/r^2 + 2 dx (v.r)/r^4 */
                    cacc(&grad[4 * j], cscale(d, -v1 / r2 + 2 * dx * vr / r4));
                    cacc(&grad[4 * j + 2],
                         cscale(d, -v2 / r2 + 2 * dy * vr / r4));
                }
                if (ifpgh >= 3) {
                    double r6 = r4 * r2;
                    /* second derivatives of -(v.r)/r^2 */
                    double hxx = 2 * v1 * dx / r4 + 2 * (v1 * dx + vr) / r4
                                 - 8 * dx * dx * vr / r6;
                    double hxy = 2 * v1 * dy / r4 + 2 * v2 * dx / r4
                                 - 8 * dx * dy * vr / r6;
                    double hyy = 2 * v2 * dy / r4 + 2 * (v2 * dy + vr) / r4
                                 - 8 * dy * dy * vr / r6;
                    cacc(&hess[6 * j], cscale(d, hxx));
                    cacc(&hess[6 * j + 2], cscale(d, hxy));
                    cacc(&hess[6 * j + 4], cscale(d, hyy));
                }
            }
        }
    }
}

/*
 * Cauchy (cfmm2d) direct sum over all sources for targets [t0, t1).
 */
void oracle_c2d_direct(int ns, const double *src, int ifcharge,
                       const double *charge, int ifdipole,
                       const double *dipstr, int t0, int t1,
                       const double *targ, int ifpgh, double *pot,
                       double *grad, double *hess, double thresh)
{
    double th2 = thresh * thresh;
    for (int j = t0; j < t1; j++) {
        for (int i = 0; i < ns; i++) {
            double dx = targ[2 * j] - src[2 * i];
            double dy = targ[2 * j + 1] - src[2 * i + 1];
            double r2 = dx * dx + dy * dy;
            if (r2 <= th2) continue;
            cplx zi = {dx / r2, -dy / r2};   /* 1/z */
            cplx zi2 = cmul(zi, zi);          /* 1/z^2 */
            if (ifcharge) {
                cplx q = {charge[2 * i], charge[2 * i + 1]};
                cacc(&pot[2 * j], cscale(q, 0.5 * log(r2)));
                if (ifpgh >= 2) cacc(&grad[2 * j], cmul(q, zi));
                if (ifpgh >= 3) cacc(&hess[2 * j], cscale(cmul(q, zi2), -1.0));
            }
            if (ifdipole) {
                cplx d = {dipstr[2 * i], dipstr[2 * i + 1]};
                cacc(&pot[2 * j], cmul(d, zi));
                if (ifpgh >= 2) cacc(&grad[2 * j], cscale(cmul(d, zi2), -1.0));
                if (ifpgh >= 3)
                    cacc(&hess[2 * j], cscale(cmul(d, cmul(zi2, zi)), 2.0));
            }
        }
    }
}
