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
 *     eps -> expansion order rule (c_translation/src/l2dterms.c:26-67);
 *   - the Helmholtz direct sums (helmkernels2d.c:21-520) with H0 and H1
 *     from textbook methods (end of this file).
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

/* ------------------------------------------------------------------------
 * Helmholtz direct sums (c_translation/src/helmkernels2d.c:21-520), nd = 1:
 *   pot  += (i/4) [q H0(k r) + d k H1(k r) (v . r) / r]
 *   grad, hess: its x / y derivatives, in the reference's closed forms.
 * Pairs with |k r| below thresh are skipped (<= for charge-only
 * potentials, < otherwise).  H0 and H1 come from the textbook methods
 * below (not from the reference's hank103 tables):
 *   |z| small: ascending series (Abramowitz & Stegun 9.1.10, 9.1.11);
 *   Im z >= 0 otherwise: H_nu(z) = (2/pi) i^-(nu+1) K_nu(-iz) with K0, K1
 *     by Temme's continued fraction (Steed's algorithm);
 *   Im z < 0, moderate |z|: Miller's recurrence for J and the Neumann
 *     series for Y;  large |z|: Hankel's asymptotic expansion.
 * ------------------------------------------------------------------------ */
#include <complex.h>

static const double kPiO = 3.14159265358979323846;
static const double kGammaO = 0.57721566490153286061;

static void o_hank_series(double complex z, double complex *h0, double complex *h1)
{
    double complex w = -z * z / 4.0, t0 = 1.0, t1 = 1.0, j0 = 1.0, j1s = 1.0;
    double complex s0 = 0.0, s1 = (1.0 - 2.0 * kGammaO);
    double hk = 0.0, mag = 1.0, aw = cabs(w);
    for (int k = 1; k < 40; k++) {
        t0 *= w / ((double)k * k);
        t1 *= w / ((double)k * (k + 1));
        hk += 1.0 / k;
        j0 += t0;
        j1s += t1;
        s0 += t0 * hk;
        s1 += t1 * (2.0 * hk + 1.0 / (k + 1) - 2.0 * kGammaO);
        mag *= aw / ((double)k * k);
        if (mag * (1.0 + hk) < 1e-18) break;
    }
    double complex lz = clog(z / 2.0), j1 = z / 2.0 * j1s;
    double complex y0 = 2.0 / kPiO * ((lz + kGammaO) * j0 - s0);
    double complex y1 = -2.0 / (kPiO * z) + 2.0 / kPiO * lz * j1 - z / 2.0 * s1 / kPiO;
    *h0 = j0 + I * y0;
    *h1 = j1 + I * y1;
}

static void o_hank_cf2(double complex z, double complex *h0, double complex *h1)
{
    double complex w = -I * z, b = 2.0 * (1.0 + w), d = 1.0 / b, h = d, delh = d;
    double complex q1 = 0.0, q2 = 1.0, q = 0.25, s = 1.0 + 0.25 * delh;
    double a = -0.25, c = 0.25;
    for (int i = 2; i < 2000; i++) {
        a -= 2.0 * (i - 1);
        c = -a * c / i;
        double complex qn = (q1 - b * q2) / a;
        q1 = q2;
        q2 = qn;
        q += c * qn;
        b += 2.0;
        d = 1.0 / (b + a * d);
        delh = (b * d - 1.0) * delh;
        h += delh;
        double complex dels = q * delh;
        s += dels;
        if (cabs(dels) < 1e-17 * cabs(s)) break;
    }
    double complex k0 = csqrt(kPiO / (2.0 * w)) * cexp(-w) / s;
    double complex k1 = k0 * (w + 0.5 - 0.25 * h) / w;
    *h0 = -2.0 * I / kPiO * k0;
    *h1 = -2.0 / kPiO * k1;
}

static void o_hank_neumann(double complex z, double complex *h0, double complex *h1)
{
    double az = cabs(z);
    int n = 2 * (int)((az + 40.0 + 6.0 * sqrt(az)) * 0.5) + 2;
    double complex zm = cimag(z) >= 0 ? -I : I, f = 1e-300, fp1 = 0.0;
    double complex psi = 0.0, sy0 = 0.0, sy1 = 0.0, zmk = cpow(zm, n % 4);
    for (int k = n; k >= 1; k--) {
        psi += zmk * f;
        zmk /= zm;
        if ((k & 1) == 0) {
            int m = k / 2;
            sy0 += f * ((m & 1) ? -1.0 : 1.0) / m;
        } else {
            int mlo = (k + 1) / 2, mhi = (k - 1) / 2;
            sy1 += f * ((mlo & 1) ? -1.0 : 1.0) / mlo;
            if (mhi >= 1) sy1 -= f * ((mhi & 1) ? -1.0 : 1.0) / mhi;
        }
        double complex fm1 = 2.0 * k / z * f - fp1;
        fp1 = f;
        f = fm1;
        if (cabs(f) > 1e250) {
            f *= 1e-250;
            fp1 *= 1e-250;
            psi *= 1e-250;
            sy0 *= 1e-250;
            sy1 *= 1e-250;
        }
    }
    double complex sc = (cimag(z) >= 0 ? cexp(-I * z) : cexp(I * z)) / (f + 2.0 * psi);
    double complex j0 = f * sc, j1 = fp1 * sc, lg = clog(z / 2.0) + kGammaO;
    double complex y0 = 2.0 / kPiO * lg * j0 - 4.0 / kPiO * sy0 * sc;
    double complex y1 = 2.0 / kPiO * lg * j1 - 2.0 / kPiO * j0 / z + 2.0 / kPiO * sy1 * sc;
    *h0 = j0 + I * y0;
    *h1 = j1 + I * y1;
}

static void o_hank_asym(double complex z, double complex *h0, double complex *h1)
{
    double complex izi = I / z, p0 = 1.0, p1 = 1.0, t0 = 1.0, t1 = 1.0;
    double az = cabs(z);
    for (int k = 1; k < 200; k++) {
        double o = 2.0 * k - 1.0;
        if (o * o > 8.0 * k * az) break;
        t0 *= izi * (-o * o / (8.0 * k));
        t1 *= izi * ((4.0 - o * o) / (8.0 * k));
        p0 += t0;
        p1 += t1;
        if (cabs(t0) + cabs(t1) < 1e-18) break;
    }
    double complex pre = csqrt(2.0 / (kPiO * z)) * cexp(I * z);
    *h0 = pre * cexp(-I * kPiO / 4.0) * p0;
    *h1 = pre * cexp(-3.0 * I * kPiO / 4.0) * p1;
}

static void o_hankel01(double complex z, double complex *h0, double complex *h1)
{
    double az = cabs(z);
    if (cimag(z) >= 0) {
        if (az <= 1.5 || (az <= 4.0 && cimag(z) < 1.5)) o_hank_series(z, h0, h1);
        else o_hank_cf2(z, h0, h1);
    } else if (az <= 4.0) {
        o_hank_series(z, h0, h1);
    } else if (az < 20.0) {
        o_hank_neumann(z, h0, h1);
    } else {
        o_hank_asym(z, h0, h1);
    }
}

void oracle_hankel01(int n, const double *z, double *out)
{
    for (int k = 0; k < n; k++) {
        double complex h0, h1;
        o_hankel01(z[2 * k] + I * z[2 * k + 1], &h0, &h1);
        out[4 * k] = creal(h0);
        out[4 * k + 1] = cimag(h0);
        out[4 * k + 2] = creal(h1);
        out[4 * k + 3] = cimag(h1);
    }
}

void oracle_h2d_direct(double zk_re, double zk_im, int ns, const double *src, int ifcharge,
                       const double *charge, int ifdipole, const double *dipstr,
                       const double *dipvec, int nt, const double *targ, int ifpgh,
                       double *pot, double *grad, double *hess, double thresh)
{
    const double complex zk = zk_re + I * zk_im, i4 = I / 4.0;
    const int le = ifcharge && !ifdipole && ifpgh == 1;
    for (int t = 0; t < nt; t++) {
        double complex p = 0, gx = 0, gy = 0, hxx = 0, hxy = 0, hyy = 0;
        for (int s = 0; s < ns; s++) {
            const double dx = targ[2 * t] - src[2 * s], dy = targ[2 * t + 1] - src[2 * s + 1];
            const double rr = dx * dx + dy * dy, r = sqrt(rr);
            const double complex z = zk * r;
            const double az = cabs(z);
            if (le ? (az <= thresh) : (az < thresh)) continue;
            double complex h0, h1;
            o_hankel01(z, &h0, &h1);
            if (ifcharge) {
                const double complex q = charge[2 * s] + I * charge[2 * s + 1];
                p += h0 * q * i4;
                const double complex cd = -h1 * (zk * i4 / r) * q;
                gx += cd * dx;
                gy += cd * dy;
                const double complex c2 = (zk * i4 / r) / rr * q, h2z = -z * h0 + 2.0 * h1;
                hxx += c2 * (h2z * dx * dx - rr * h1);
                hxy += c2 * (h2z * dx * dy);
                hyy += c2 * (h2z * dy * dy - rr * h1);
            }
            if (ifdipole) {
                const double complex d = dipstr[2 * s] + I * dipstr[2 * s + 1];
                const double v1 = dipvec[2 * s], v2 = dipvec[2 * s + 1];
                const double ct = dx / r, st = dy / r;
                const double complex h2 = 2.0 * h1 / z - h0, h3 = 4.0 * h2 / z - h1;
                p += h1 / r * zk * i4 * d * (dx * v1 + dy * v2);
                const double complex c2 = -zk * zk * i4 * d;
                const double complex f1 = h2 * (ct * ct - 0.5) - h0 / 2.0, f2 = h2 * ct * st;
                const double complex f3 = h2 * (st * st - 0.5) - h0 / 2.0;
                gx += c2 * (f1 * v1 + f2 * v2);
                gy += c2 * (f2 * v1 + f3 * v2);
                const double complex a1 = (h1 * 0.75 - h3 / 2.0 * (ct * ct - 0.5 - st * st)) * ct;
                const double complex a2 = (h1 * 0.25 - h3 / 2.0 * (1.5 * ct * ct - 0.5 * st * st)) * st;
                const double complex a3 = (h1 * 0.25 - h3 / 2.0 * (1.5 * st * st - 0.5 * ct * ct)) * ct;
                const double complex a4 = (h1 * 0.75 - h3 / 2.0 * (st * st - 0.5 - ct * ct)) * st;
                const double complex c3 = -zk * zk * zk * d * i4;
                hxx += c3 * (a1 * v1 + a2 * v2);
                hxy += c3 * (a2 * v1 + a3 * v2);
                hyy += c3 * (a3 * v1 + a4 * v2);
            }
        }
        pot[2 * t] += creal(p);
        pot[2 * t + 1] += cimag(p);
        if (ifpgh >= 2) {
            grad[4 * t] += creal(gx);
            grad[4 * t + 1] += cimag(gx);
            grad[4 * t + 2] += creal(gy);
            grad[4 * t + 3] += cimag(gy);
        }
        if (ifpgh >= 3) {
            hess[6 * t] += creal(hxx);
            hess[6 * t + 1] += cimag(hxx);
            hess[6 * t + 2] += creal(hxy);
            hess[6 * t + 3] += cimag(hxy);
            hess[6 * t + 4] += creal(hyy);
            hess[6 * t + 5] += cimag(hyy);
        }
    }
}
