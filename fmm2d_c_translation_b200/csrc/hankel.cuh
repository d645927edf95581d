// hankel.cuh -- complex Bessel/Hankel functions of orders 0 and 1, and the
// scaled order-n sequences of the Helmholtz expansions, for host and device.
//
// The reference gets H0, H1 from Rokhlin's hank103 (c_translation/src/
// hank103.c:66-153) and the scaled sequences from h2dall (h2dcommon.c:35-90,
// upward recurrence) and jbessel2d (cdjseval2d.c:11-160, Miller's downward
// recurrence normalised by exp(-/+ i z)).  H0 and H1 here are computed by
// three textbook methods, picked by |z| and Im z:
//   * |z| <= 4 (|z| <= 1.5 when Im z >= 1.5): the ascending series of J0,
//     J1, Y0, Y1 (Abramowitz & Stegun 9.1.10, 9.1.11);
//   * the rest of Im z >= 0: H from K via H_nu(z) = (2/pi) i^-(nu+1)
//     K_nu(-iz), with K0, K1 by Temme's continued fraction (Steed's
//     algorithm, CF2);
//   * 4 < |z| < 20, Im z < 0: J by Miller's recurrence and Y by the Neumann
//     series Y0 = (2/pi)(ln(z/2) + gamma) J0 - (4/pi) sum_k (-1)^k J_2k / k
//     and its derivative;
//   * |z| >= 20, Im z < 0: Hankel's asymptotic expansion (A&S 9.2.7).
// All work in FP64 complex arithmetic on double2.
#pragma once

#include <math.h>

#include "common.cuh"

namespace fmm2d {
namespace hk {

#define FMM_HD __host__ __device__ __forceinline__

constexpr double kPi = 3.14159265358979323846;
constexpr double kEulerGamma = 0.57721566490153286061;

FMM_HD double cabs_(double2 z) { return hypot(z.x, z.y); }

FMM_HD double2 cexp_(double2 z) {
    const double e = exp(z.x);
    return make_double2(e * cos(z.y), e * sin(z.y));
}

FMM_HD double2 clog_(double2 z) { return make_double2(log(hypot(z.x, z.y)), atan2(z.y, z.x)); }

// principal square root
FMM_HD double2 csqrt_(double2 z) {
    const double r = hypot(z.x, z.y);
    if (r == 0.0) return make_double2(0.0, 0.0);
    if (z.x >= 0.0) {
        const double t = sqrt(0.5 * (r + z.x));
        return make_double2(t, z.y / (2.0 * t));
    }
    const double t = sqrt(0.5 * (r - z.x));
    return make_double2(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}

// a / b (Smith's algorithm, no intermediate overflow)
FMM_HD double2 cdiv_(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    const double r = b.x / b.y, d = b.y + b.x * r;
    return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}

FMM_HD double2 cmuli(double2 z) { return make_double2(-z.y, z.x); }  // i z

// ---------------------------------------------------------------------------
// |z| <= 4: ascending series.
FMM_HD void hankel01_series(double2 z, double2 &h0, double2 &h1) {
    const double2 w = cscal(cmul(z, z), 0.25);     // z^2 / 4
    const double2 mw = make_double2(-w.x, -w.y);   // -z^2 / 4
    double2 t0 = make_double2(1.0, 0.0);  // (-w)^k / (k!)^2
    double2 t1 = make_double2(1.0, 0.0);  // (-w)^k / (k! (k+1)!)
    double2 j0 = t0, j1s = t1;
    double2 s0 = make_double2(0.0, 0.0);  // sum H_k (-w)^k / (k!)^2
    // sum (psi(k+1) + psi(k+2)) (-w)^k / (k!(k+1)!), psi(k+1) = -gamma + H_k
    double2 s1 = cscal(t1, 1.0 - 2.0 * kEulerGamma);
    double hk = 0.0;
    const double aw = cabs_(w);
    double mag = 1.0;
    for (int k = 1; k < 40; k++) {
        const double dk = (double)k;
        t0 = cscal(cmul(t0, mw), 1.0 / (dk * dk));
        t1 = cscal(cmul(t1, mw), 1.0 / (dk * (dk + 1.0)));
        hk += 1.0 / dk;
        j0 = cadd(j0, t0);
        j1s = cadd(j1s, t1);
        s0 = cadd(s0, cscal(t0, hk));
        s1 = cadd(s1, cscal(t1, 2.0 * hk + 1.0 / (dk + 1.0) - 2.0 * kEulerGamma));
        mag *= aw / (dk * dk);
        if (mag * (1.0 + hk) < 1e-18) break;
    }
    const double2 zh = cscal(z, 0.5);
    const double2 lz = clog_(zh);  // ln(z/2)
    const double2 j1 = cmul(zh, j1s);
    // Y0 = (2/pi) [(ln(z/2) + gamma) J0 - s0]
    const double2 y0 = cscal(csub(cmul(cadd(lz, make_double2(kEulerGamma, 0.0)), j0), s0),
                             2.0 / kPi);
    // Y1 = -2/(pi z) + (2/pi) ln(z/2) J1 - (1/pi)(z/2) s1
    const double2 y1 = cadd(cscal(cinv(z), -2.0 / kPi),
                            csub(cscal(cmul(lz, j1), 2.0 / kPi), cscal(cmul(zh, s1), 1.0 / kPi)));
    h0 = cadd(j0, cmuli(y0));
    h1 = cadd(j1, cmuli(y1));
}

// |z| >= 20: Hankel's expansion H_nu ~ sqrt(2/(pi z)) e^{i(z - nu pi/2 - pi/4)}
// sum_k i^k a_k(nu) / z^k, a_k = a_{k-1} (4 nu^2 - (2k-1)^2) / (8k).
FMM_HD void hankel01_asym(double2 z, double2 &h0, double2 &h1) {
    const double2 zi = cinv(z);
    const double2 izi = cmuli(zi);  // i / z
    double2 p0 = make_double2(1.0, 0.0), p1 = p0;
    double2 t0 = p0, t1 = p0;
    // the series diverges: stop at its smallest term
    const double az = cabs_(z);
    for (int k = 1; k < 200; k++) {
        const double o = (double)(2 * k - 1);
        if (o * o > 8.0 * k * az) break;  // terms grow from here on
        const double c0 = -o * o / (8.0 * k), c1 = (4.0 - o * o) / (8.0 * k);
        t0 = cscal(cmul(t0, izi), c0);
        t1 = cscal(cmul(t1, izi), c1);
        p0 = cadd(p0, t0);
        p1 = cadd(p1, t1);
        if (cabs_(t0) + cabs_(t1) < 1e-18) break;
    }
    const double2 pre = cscal(csqrt_(zi), sqrt(2.0 / kPi));
    // e^{iz} e^{-i pi/4} and e^{iz} e^{-3 i pi/4}
    const double2 eiz = cexp_(cmuli(z));
    const double r2 = 0.70710678118654752440;
    const double2 e0 = cmul(eiz, make_double2(r2, -r2));
    const double2 e1 = cmul(eiz, make_double2(-r2, -r2));
    h0 = cmul(cmul(pre, e0), p0);
    h1 = cmul(cmul(pre, e1), p1);
}

// K0(w), K1(w) for Re w >= 0, |w| >= 2 by Temme's CF2 (Steed's algorithm).
FMM_HD void bessel_k01_cf2(double2 w, double2 &k0, double2 &k1) {
    const double a1 = 0.25;
    double2 b = cscal(cadd(w, make_double2(1.0, 0.0)), 2.0);
    double2 d = cinv(b);
    double2 h = d, delh = d;
    double2 q1 = make_double2(0.0, 0.0), q2 = make_double2(1.0, 0.0);
    double2 q = make_double2(a1, 0.0);
    double c = a1, a = -a1;
    double2 s = cadd(make_double2(1.0, 0.0), cscal(delh, a1));
    for (int i = 2; i < 2000; i++) {
        a -= 2.0 * (i - 1);
        c = -a * c / i;
        const double2 qn = cscal(csub(q1, cmul(b, q2)), 1.0 / a);
        q1 = q2;
        q2 = qn;
        q = cadd(q, cscal(qn, c));
        b = cadd(b, make_double2(2.0, 0.0));
        d = cinv(cadd(b, cscal(d, a)));
        delh = cmul(csub(cmul(b, d), make_double2(1.0, 0.0)), delh);
        h = cadd(h, delh);
        const double2 dels = cmul(q, delh);
        s = cadd(s, dels);
        if (cabs_(dels) < 1e-17 * cabs_(s)) break;
    }
    h = cscal(h, a1);
    // K0 = sqrt(pi / (2w)) e^{-w} / s
    k0 = cdiv_(cmul(csqrt_(cscal(cinv(w), 0.5 * kPi)), cexp_(make_double2(-w.x, -w.y))), s);
    // K1 = K0 (w + 1/2 - h) / w
    k1 = cdiv_(cmul(k0, csub(cadd(w, make_double2(0.5, 0.0)), h)), w);
}

// Miller's recurrence for J0, J1, J2, ... normalised by
// exp(-i z) = J0 + 2 sum (-i)^k J_k (Im z >= 0) or exp(i z) = J0 + 2 sum i^k J_k
// (Im z < 0); Neumann series for Y0 and Y1.
FMM_HD void hankel01_neumann(double2 z, double2 &h0, double2 &h1) {
    const double az = cabs_(z);
    int n = 2 * (int)((az + 40.0 + 2.0 * sqrt(az) * 3.0) * 0.5) + 2;
    const double2 zinv = cinv(z);
    const double2 zm = z.y >= 0.0 ? make_double2(0.0, -1.0) : make_double2(0.0, 1.0);
    // downward: f_{k-1} = (2k/z) f_k - f_{k+1}
    double2 fp1 = make_double2(0.0, 0.0), f = make_double2(1e-300, 0.0);
    double2 psi = make_double2(0.0, 0.0);  // sum_{k>=1} zm^k f_k
    double2 sy0 = make_double2(0.0, 0.0);  // sum_{k>=1} (-1)^k f_2k / k
    double2 sy1 = make_double2(0.0, 0.0);  // sum_{k>=1} (-1)^k (f_{2k-1} - f_{2k+1}) / k
    // zm^k for the current k
    double2 zmk = make_double2(1.0, 0.0);
    for (int k = 0; k < (n & 3); k++) zmk = cmul(zmk, zm);
    const double2 zmi = make_double2(zm.x, -zm.y);  // 1 / zm
    for (int k = n; k >= 1; k--) {
        // f holds f_k, fp1 holds f_{k+1}
        psi = cadd(psi, cmul(zmk, f));
        zmk = cmul(zmk, zmi);
        if ((k & 1) == 0) {
            const int m = k >> 1;
            const double sg = (m & 1) ? -1.0 : 1.0;
            sy0 = cadd(sy0, cscal(f, sg / m));
        } else {
            // k = 2m - 1 : contributes +f_{2m-1} to term m; k = 2m + 1 : -f_{2m+1} to term m
            const int mlo = (k + 1) >> 1, mhi = (k - 1) >> 1;
            sy1 = cadd(sy1, cscal(f, ((mlo & 1) ? -1.0 : 1.0) / mlo));
            if (mhi >= 1) sy1 = csub(sy1, cscal(f, ((mhi & 1) ? -1.0 : 1.0) / mhi));
        }
        const double2 fm1 = csub(cscal(cmul(zinv, f), 2.0 * k), fp1);
        fp1 = f;
        f = fm1;
        const double mg = fabs(f.x) + fabs(f.y);
        if (mg > 1e250) {
            const double s = 1e-250;
            f = cscal(f, s);
            fp1 = cscal(fp1, s);
            psi = cscal(psi, s);
            sy0 = cscal(sy0, s);
            sy1 = cscal(sy1, s);
        }
    }
    const double2 f0 = f, f1 = fp1;
    const double2 norm = cadd(f0, cscal(psi, 2.0));
    const double2 ez = z.y >= 0.0 ? cexp_(make_double2(z.y, -z.x)) : cexp_(make_double2(-z.y, z.x));
    const double2 sc = cdiv_(ez, norm);
    const double2 j0 = cmul(f0, sc), j1 = cmul(f1, sc);
    const double2 y0s = cmul(sy0, sc), y1s = cmul(sy1, sc);
    const double2 lg = cadd(clog_(cscal(z, 0.5)), make_double2(kEulerGamma, 0.0));
    const double2 y0 = csub(cscal(cmul(lg, j0), 2.0 / kPi), cscal(y0s, 4.0 / kPi));
    const double2 y1 = cadd(csub(cscal(cmul(lg, j1), 2.0 / kPi), cscal(cmul(j0, zinv), 2.0 / kPi)),
                            cscal(y1s, 2.0 / kPi));
    h0 = cadd(j0, cmuli(y0));
    h1 = cadd(j1, cmuli(y1));
}

// H0^(1)(z), H1^(1)(z), principal branches, z != 0.
FMM_HD void hankel01(double2 z, double2 &h0, double2 &h1) {
    const double az = cabs_(z);
    if (z.y >= 0.0) {
        if (az <= 1.5 || (az <= 4.0 && z.y < 1.5)) {
            hankel01_series(z, h0, h1);
        } else {
            double2 k0, k1;
            bessel_k01_cf2(make_double2(z.y, -z.x), k0, k1);  // w = -i z
            h0 = cscal(make_double2(k0.y, -k0.x), 2.0 / kPi);  // (2/pi)(-i) K0
            h1 = cscal(k1, -2.0 / kPi);
        }
    } else if (az <= 4.0) {
        hankel01_series(z, h0, h1);
    } else if (az < 20.0) {
        hankel01_neumann(z, h0, h1);
    } else {
        hankel01_asym(z, h0, h1);
    }
}

#undef FMM_HD

}  // namespace hk
}  // namespace fmm2d
