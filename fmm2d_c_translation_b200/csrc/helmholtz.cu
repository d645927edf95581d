// helmholtz.cu -- the Helmholtz FMM (hfmm2dmain, c_translation/src/
// hfmm2d.c:619-1528) on the device.
//
// Conventions (those of helmrouts2d.c, so that every expansion matches the
// reference's to rounding): a multipole of a box with center c, order p and
// scale r holds M_n = sum_s q_s J_n(k rho_s) e^{-i n theta_s} / r^|n| and a
// local expansion L_n with the field sum_n L_n J_n(k rho) e^{i n theta} r^|n|
// times i/4; J_n / r^n and H_n r^n are the reference's scaled sequences
// (jbessel2d, h2dall).
//
// Kernels:
//   * P2M (h2dformmp*) and P2L (h2dformta*): one warp per box, lanes =
//     sources.  Each lane generates its Bessel sequence (Miller's downward
//     recurrence for J, two passes so the normalisation is known before the
//     coefficients are emitted; the upward recurrence for H) and the
//     coefficient contributions are summed across the warp per order.
//   * M2M, M2L, L2L (h2dmpmp, h2dmploc, h2dlocloc): all three are
//     out_i = S_i sum_j in_j T(i - j) r1^e(i, j) with T a table of J_m or H_m
//     times e^{-i m theta} for the (fixed, per level) offset between the two
//     centers, S_i and r1^e powers of the two scales.  One thread per output
//     coefficient; the tables are built on the host per level and offset.
//   * M2P + L2P (h2dmpeval*, h2dtaeval*): one thread per point, upward H
//     (multipoles of list 3) and downward J (the leaf's local expansion),
//     derivatives from the mk_mpoleg / mk_mpoleh coefficient recurrences
//     evaluated on the fly.
//   * P2P (hfmm2dpart_direct -> h2d_direct*): one thread per point over the
//     sources of list 1; H0, H1 per pair from hankel.cuh (the CUDA libm J0,
//     J1, Y0, Y1 below argument 8 for real wavenumbers).
#include "helmholtz.cuh"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "hankel.cuh"
#include "laplace.cuh"

namespace fmm2d {

// ---------------------------------------------------------------------------
// Host restatements of h2dall, jbessel2d and h2dterms.
// ---------------------------------------------------------------------------
void helm_hvec(int n, double2 z, double rscale, double2 *h) {
    if (hk::cabs_(z) < 1.0e-200) {
        for (int i = 0; i <= n; i++) h[i] = make_double2(0.0, 0.0);
        return;
    }
    double2 h0, h1;
    hk::hankel01(z, h0, h1);
    h[0] = h0;
    if (n >= 1) h[1] = cscal(h1, rscale);
    const double2 zinv = cscal(cinv(z), rscale);
    const double scal2 = rscale * rscale;
    for (int i = 1; i <= n - 1; i++)
        h[i + 1] = csub(cmul(cscal(zinv, 2.0 * i), h[i]), cscal(h[i - 1], scal2));
}

void helm_jvec(int nterms, double2 z, double rscale, double2 *fjs) {
    if (hk::cabs_(z) < 1.0e-200) {
        fjs[0] = make_double2(1.0, 0.0);
        for (int i = 1; i <= nterms; i++) fjs[i] = make_double2(0.0, 0.0);
        return;
    }
    const double upbound2 = 1.0e40, upbound2inv = 1.0e-40;
    // upward from nterms until the magnitude has grown by 1e20
    int ntop = nterms + 10000;
    const double2 zinv = cinv(z);
    double2 fn = make_double2(1.0, 0.0), fnm1 = make_double2(0.0, 0.0);
    for (int i = nterms; i <= nterms + 10000; i++) {
        const double2 t = csub(cmul(cscal(zinv, 2.0 * i), fn), fnm1);
        if (t.x * t.x + t.y * t.y > upbound2) {
            ntop = i + 1;
            break;
        }
        fnm1 = fn;
        fn = t;
    }
    std::vector<double2> f(ntop + 1);
    std::vector<char> isc(ntop + 1, 0);
    f[ntop] = make_double2(0.0, 0.0);
    f[ntop - 1] = make_double2(1.0, 0.0);
    for (int i = ntop - 1; i >= 1; i--) {
        const double2 t = csub(cmul(cscal(zinv, 2.0 * i), f[i]), f[i + 1]);
        f[i - 1] = t;
        if (t.x * t.x + t.y * t.y > upbound2) {
            f[i] = cscal(f[i], upbound2inv);
            f[i - 1] = cscal(f[i - 1], upbound2inv);
            isc[i] = 1;
        }
    }
    double sctot = 1.0;
    const double scalinv = 1.0 / rscale;
    for (int i = 1; i <= ntop; i++) {
        sctot *= scalinv;
        if (isc[i - 1]) sctot *= upbound2inv;
        f[i] = cscal(f[i], sctot);
    }
    // exp(-/+ i z) = J0 + 2 sum (-/+ i)^k J_k
    const double2 zmul = z.y < 0 ? make_double2(0.0, 1.0) : make_double2(0.0, -1.0);
    const double2 zmulinv = make_double2(zmul.x, -zmul.y);
    double2 zsn = make_double2(1.0, 0.0);
    for (int i = 0; i < ntop % 4; i++) zsn = cmul(zsn, zmul);
    double2 psi = make_double2(0.0, 0.0);
    for (int i = ntop; i >= 1; i--) {
        psi = cadd(cscal(psi, rscale), cmul(f[i], zsn));
        zsn = cmul(zsn, zmulinv);
    }
    psi = cadd(cscal(psi, 2.0 * rscale), f[0]);
    const double2 ez = z.y < 0 ? hk::cexp_(make_double2(-z.y, z.x)) : hk::cexp_(make_double2(z.y, -z.x));
    const double2 zscale = hk::cdiv_(ez, psi);
    for (int i = 0; i <= nterms; i++) fjs[i] = cmul(f[i], zscale);
}

namespace {
std::mutex g_nterms_mu;
std::map<std::tuple<double, double, double, double>, int> g_nterms_cache;
}  // namespace

int helm_nterms(double bsize, double2 zk, double eps) {
    const auto key = std::make_tuple(bsize, zk.x, zk.y, eps);
    {
        std::lock_guard<std::mutex> g(g_nterms_mu);
        auto it = g_nterms_cache.find(key);
        if (it != g_nterms_cache.end()) return it->second;
    }
    const int ntmax = 50000;
    const double pi2 = 8.0 * std::atan(1.0);
    const double2 zb = cscal(zk, bsize);
    const double2 z1 = cscal(zb, 1.5);
    double rscale = 1.0;
    if (hk::cabs_(zb) < pi2) rscale = hk::cabs_(zb);
    std::vector<double2> hfun(ntmax + 1), jfun(ntmax + 1);
    helm_hvec(ntmax, z1, rscale, hfun.data());
    const double2 z2 = cscal(zb, std::sqrt(2.0) / 2.0);
    helm_jvec(ntmax, z2, rscale, jfun.data());
    const double xtemp0 = hk::cabs_(cmul(jfun[0], hfun[0])) + hk::cabs_(cmul(jfun[1], hfun[1]));
    const double h0 = hk::cabs_(hfun[0]);
    int nterms = -1;
    for (int j = 2; j <= ntmax; j++) {
        const double x1 = hk::cabs_(cmul(jfun[j], hfun[j]));
        const double x2 = hk::cabs_(cmul(jfun[j - 1], hfun[j - 1]));
        if ((x1 + x2) * h0 < eps * xtemp0) {
            nterms = j + 1;
            break;
        }
    }
    std::lock_guard<std::mutex> g(g_nterms_mu);
    g_nterms_cache[key] = nterms;
    return nterms;
}

namespace {

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
struct HLevel {
    long long off;  // offset (in double2) of the level's first box block
    int p;          // expansion order
    int lstart;     // first box id of the level
    double rs;      // scale rscales(l)
    int flag;       // Im(zk) * boxsize(l) < 40 (zkiupbound of hfmm2dmain)
    int pad;
};

// Pointer to coefficient n = 0, channel 0 of box b (level L).
__device__ __forceinline__ const double2 *coef0(const double2 *base, const HLevel &L, int b, int nd) {
    return base + L.off + (long long)(b - L.lstart) * (2 * L.p + 1) * nd + (long long)L.p * nd;
}
__device__ __forceinline__ double2 *coef0(double2 *base, const HLevel &L, int b, int nd) {
    return base + L.off + (long long)(b - L.lstart) * (2 * L.p + 1) * nd + (long long)L.p * nd;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double2 cconj(double2 z) { return make_double2(z.x, -z.y); }

// zm^k for zm = -i (Im z >= 0) or +i (Im z < 0)
__device__ __forceinline__ double2 zm_pow(int k, bool lower) {
    const int r = k & 3;
    const double s = lower ? 1.0 : -1.0;
    if (r == 0) return make_double2(1.0, 0.0);
    if (r == 1) return make_double2(0.0, s);
    if (r == 2) return make_double2(-1.0, 0.0);
    return make_double2(0.0, -s);
}

// Top order of jbessel2d's downward recurrence for `nterms` terms.
__device__ int jb_ntop(int nterms, double2 zinv) {
    double2 fn = make_double2(1.0, 0.0), fnm1 = make_double2(0.0, 0.0);
    for (int i = nterms; i <= nterms + 10000; i++) {
        const double2 t = csub(cmul(cscal(zinv, 2.0 * i), fn), fnm1);
        if (t.x * t.x + t.y * t.y > 1.0e40) return i + 1;
        fnm1 = fn;
        fn = t;
    }
    return nterms + 10000;
}

// ---------------------------------------------------------------------------
// Coefficient contributions of one source (ctompole / dtompole,
// helmrouts2d.c:43-105) to orders +n and -n.  bn = sequence value of order
// n, bnm1 / bnp1 of n-1 / n+1; pw = zmul^n with zmul = e^{-i theta};
// rsd = the scale dtompole is given.
// ---------------------------------------------------------------------------
struct SrcGeo {
    double2 em, ep;  // e^{-i theta}, e^{i theta}
};

__device__ __forceinline__ void contrib(int n, double2 bnm1, double2 bn, double2 bnp1,
                                        double2 pw, const SrcGeo &g, double2 zk, double rsd,
                                        bool ifc, double2 q, bool ifd, double2 d, double2 v,
                                        double2 &cp, double2 &cm) {
    cp = make_double2(0.0, 0.0);
    cm = make_double2(0.0, 0.0);
    const double2 zkh = cscal(zk, 0.5);
    if (n == 0) {
        if (ifc) cp = cmul(q, bn);
        if (ifd) {
            // -d J_1 (k/2) r ((zmul + zinv) v1 + (zmul - zinv) i v2)
            const double2 a = cscal(cadd(g.em, g.ep), v.x);
            const double2 b = hk::cmuli(cscal(csub(g.em, g.ep), v.y));
            const double2 t = cscal(cmul(cmul(d, bnp1), zkh), -rsd);
            cp = cadd(cp, cmul(t, cadd(a, b)));
        }
        return;
    }
    const double sg = (n & 1) ? -1.0 : 1.0;  // (-1)^n
    const double2 pwc = cconj(pw);           // zinv^n
    if (ifc) {
        const double2 qb = cmul(q, bn);
        cp = cmul(qb, pw);
        cm = cscal(cmul(qb, pwc), sg);
    }
    if (ifd) {
        const double rinv = 1.0 / rsd;
        const double2 t7 = cmul(cscal(g.ep, rinv), make_double2(-v.x, v.y));
        const double2 t8 = cmul(cscal(g.em, rsd), make_double2(v.x, v.y));
        const double2 t9 = cmul(cscal(g.em, rinv), make_double2(-v.x, -v.y));
        const double2 t10 = cmul(cscal(g.ep, rsd), make_double2(v.x, -v.y));
        // ztemp1 = -(k/2) zmul^n, ztemp2 = (k/2) (-1)^(n-1) zinv^n
        const double2 zt1 = cscal(cmul(zkh, pw), -1.0);
        const double2 zt2 = cscal(cmul(zkh, pwc), -sg);
        const double2 a = cadd(cmul(bnm1, t7), cmul(bnp1, t8));
        const double2 b = cadd(cmul(bnm1, t9), cmul(bnp1, t10));
        cp = cadd(cp, cmul(cmul(a, zt1), d));
        cm = cadd(cm, cmul(cmul(b, zt2), d));
    }
}

// Sums cp / cm over the warp and adds them to the box's coefficients.
__device__ __forceinline__ void emit_warp(double2 *E, int n, int nd, int c, double2 cp, double2 cm,
                                         int lane) {
    const double a = warp_sum(cp.x), b = warp_sum(cp.y);
    double e = 0.0, f = 0.0;
    if (n != 0) {
        e = warp_sum(cm.x);
        f = warp_sum(cm.y);
    }
    if (lane == 0) {
        double2 &o = E[(long long)n * nd + c];
        o = make_double2(o.x + a, o.y + b);
        if (n != 0) {
            double2 &u = E[-(long long)n * nd + c];
            u = make_double2(u.x + e, u.y + f);
        }
    }
}

// emit_warp over a group of W lanes (W = 32 or 16, mask the group's lanes).
template <int W>
__device__ __forceinline__ double group_sum(double v, unsigned mask) {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}
template <int W>
__device__ __forceinline__ void emit_group(double2 *E, int n, int nd, int c, double2 cp,
                                           double2 cm, int lane, unsigned mask) {
    const double a = group_sum<W>(cp.x, mask), b = group_sum<W>(cp.y, mask);
    double e = 0.0, f = 0.0;
    if (n != 0) {
        e = group_sum<W>(cm.x, mask);
        f = group_sum<W>(cm.y, mask);
    }
    if (lane == 0) {
        double2 &o = E[(long long)n * nd + c];
        o = make_double2(o.x + a, o.y + b);
        if (n != 0) {
            double2 &u = E[-(long long)n * nd + c];
            u = make_double2(u.x + e, u.y + f);
        }
    }
}

// ---------------------------------------------------------------------------
// P2M (h2dformmpc/d/cd, helmrouts2d.c:294-393): a group of W lanes (a warp,
// or a half warp for leaves of few sources) per leaf at level >= 2; every
// shuffle stays within the group.
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(256) helm_p2m_kernel(
    int nb, const int *__restrict__ nchild, const int *__restrict__ level,
    const int2 *__restrict__ sse, const double2 *__restrict__ centers,
    const HLevel *__restrict__ lv, const double2 *__restrict__ src,
    const double2 *__restrict__ charge, const double2 *__restrict__ dipstr,
    const double2 *__restrict__ dipvec, int ifc, int ifd, int nd, double2 zk,
    double2 *__restrict__ mp) {
    const int lane = threadIdx.x & (W - 1);
    const unsigned gmask = W == 32 ? 0xffffffffu : (0xffffu << (threadIdx.x & 16));
    const int nw = (gridDim.x * blockDim.x) / W;
    for (int b = (blockIdx.x * blockDim.x + threadIdx.x) / W; b < nb; b += nw) {
        if (nchild[b] != 0) continue;
        const int l = level[b];
        if (l < 2) continue;
        const HLevel L = lv[l];
        if (!L.flag) continue;
        const int2 r = sse[b];
        if (r.y <= r.x) continue;
        const int p = L.p;
        const double rs = L.rs, rs2 = rs * rs;
        double2 *M = const_cast<double2 *>(coef0(mp, L, b, nd));
        const double2 ctr = centers[b];
        for (int k0 = r.x; k0 < r.y; k0 += W) {
            const int k = k0 + lane;
            const bool valid = k < r.y;
            SrcGeo g{make_double2(1.0, 0.0), make_double2(1.0, 0.0)};
            double2 z = make_double2(0.0, 0.0), zr = z;
            int ntop = 0;
            bool tiny = false, lower = false;
            if (valid) {
                const double dx = src[k].x - ctr.x, dy = src[k].y - ctr.y;
                const double rr = sqrt(dx * dx + dy * dy);
                const double th = (dx == 0.0 && dy == 0.0) ? 0.0 : atan2(dy, dx);
                double sn, cs;
                sincos(th, &sn, &cs);
                g.em = make_double2(cs, -sn);
                g.ep = make_double2(cs, sn);
                z = cscal(zk, rr);
                lower = z.y < 0.0;
                if (hk::cabs_(z) < 1.0e-200) {
                    tiny = true;
                } else {
                    const double2 zinv = cinv(z);
                    zr = cscal(zinv, rs);
                    ntop = jb_ntop(p + 1, zinv);
                }
            }
            // pass A: normalisation and the number of rescalings
            double2 zscale = make_double2(0.0, 0.0);
            int nev = 0;
            if (ntop > 0) {
                double2 gp1 = make_double2(0.0, 0.0), gc = make_double2(1.0, 0.0);
                double2 psi = make_double2(0.0, 0.0);
                for (int i = ntop - 1; i >= 1; i--) {
                    double2 gm1 = csub(cmul(cscal(zr, 2.0 * i), gc), cscal(gp1, rs2));
                    if (gm1.x * gm1.x + gm1.y * gm1.y > 1.0e40) {
                        gc = cscal(gc, 1.0e-40);
                        gm1 = cscal(gm1, 1.0e-40);
                        psi = cscal(psi, 1.0e-40);
                        nev++;
                    }
                    psi = cadd(cscal(psi, rs), cmul(gc, zm_pow(i, lower)));
                    gp1 = gc;
                    gc = gm1;
                }
                psi = cadd(cscal(psi, 2.0 * rs), gc);
                const double2 ez = lower ? hk::cexp_(make_double2(-z.y, z.x))
                                         : hk::cexp_(make_double2(z.y, -z.x));
                zscale = hk::cdiv_(ez, psi);
            }
            // pass B: the same recurrence, emitting normalised J_i downward
            int nmax = ntop;
#pragma unroll
            for (int o = W / 2; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(gmask, nmax, o));
            double2 gp1 = make_double2(0.0, 0.0), gc = make_double2(0.0, 0.0);
            int ev = 0;
            double2 ja = make_double2(0.0, 0.0), jb = ja, jc = ja;  // J_i, J_{i+1}, J_{i+2}
            // e^{-i p theta}
            double2 pw = make_double2(1.0, 0.0);
            for (int m = 0; m < p; m++) pw = cmul(pw, g.em);
            for (int i = max(nmax - 1, p); i >= 0; i--) {
                double2 ji = make_double2(0.0, 0.0);
                if (ntop > 0 && i <= ntop - 1) {
                    if (i == ntop - 1) {
                        gp1 = make_double2(0.0, 0.0);
                        gc = make_double2(1.0, 0.0);
                    }
                    double2 gm1 = make_double2(0.0, 0.0);
                    if (i >= 1) {
                        gm1 = csub(cmul(cscal(zr, 2.0 * i), gc), cscal(gp1, rs2));
                        if (gm1.x * gm1.x + gm1.y * gm1.y > 1.0e40) {
                            gc = cscal(gc, 1.0e-40);
                            gm1 = cscal(gm1, 1.0e-40);
                            ev++;
                        }
                    }
                    double2 f = zscale;
                    for (int q = ev; q < nev; q++) f = cscal(f, 1.0e-40);
                    ji = cmul(gc, f);
                    if (i >= 1) {
                        gp1 = gc;
                        gc = gm1;
                    }
                } else if (tiny && i == 0) {
                    ji = make_double2(1.0, 0.0);
                }
                jc = jb;
                jb = ja;
                ja = ji;
                const int n = i + 1;
                if (n <= p) {
                    for (int c = 0; c < nd; c++) {
                        double2 cp = make_double2(0.0, 0.0), cm = cp;
                        if (valid)
                            contrib(n, ja, jb, jc, pw, g, zk, rs, ifc,
                                    ifc ? charge[(long long)k * nd + c] : cp, ifd,
                                    ifd ? dipstr[(long long)k * nd + c] : cp,
                                    ifd ? dipvec[(long long)k * nd + c] : cp, cp, cm);
                        emit_group<W>(M, n, nd, c, cp, cm, lane, gmask);
                    }
                    pw = cmul(pw, g.ep);
                }
            }
            for (int c = 0; c < nd; c++) {
                double2 cp = make_double2(0.0, 0.0), cm = cp;
                if (valid)
                    contrib(0, cm, ja, jb, make_double2(1.0, 0.0), g, zk, rs, ifc,
                            ifc ? charge[(long long)k * nd + c] : cp, ifd,
                            ifd ? dipstr[(long long)k * nd + c] : cp,
                            ifd ? dipvec[(long long)k * nd + c] : cp, cp, cm);
                emit_group<W>(M, 0, nd, c, cp, cm, lane, gmask);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// P2L (h2dformtac/d/cd, helmrouts2d.c:513-614) over list 4: warp per box.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) helm_p2l_kernel(
    int nb, const int *__restrict__ level, const int *__restrict__ nlist4,
    const int *__restrict__ list4, const int2 *__restrict__ sse,
    const double2 *__restrict__ centers, const HLevel *__restrict__ lv,
    const double2 *__restrict__ src, const double2 *__restrict__ charge,
    const double2 *__restrict__ dipstr, const double2 *__restrict__ dipvec, int ifc,
    int ifd, int nd, double2 zk, double2 *__restrict__ loc) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += nw) {
        const int n4 = nlist4[b];
        if (n4 == 0) continue;
        const int l = level[b];
        if (l < 2) continue;
        const HLevel L = lv[l];
        if (!L.flag) continue;
        const int p = L.p;
        const double rs = L.rs, rs2 = rs * rs;
        double2 *E = const_cast<double2 *>(coef0(loc, L, b, nd));
        const double2 ctr = centers[b];
        for (int e4 = 0; e4 < n4; e4++) {
            const int sb = list4[b * 5 + e4];
            const int2 r = sse[sb];
            for (int k0 = r.x; k0 < r.y; k0 += 32) {
                const int k = k0 + lane;
                const bool valid = k < r.y;
                SrcGeo g{make_double2(1.0, 0.0), make_double2(1.0, 0.0)};
                double2 hz0 = make_double2(0.0, 0.0), hz1 = hz0, zr = hz0;
                bool act = false;
                if (valid) {
                    const double dx = src[k].x - ctr.x, dy = src[k].y - ctr.y;
                    const double rr = sqrt(dx * dx + dy * dy);
                    const double th = (dx == 0.0 && dy == 0.0) ? 0.0 : atan2(dy, dx);
                    double sn, cs;
                    sincos(th, &sn, &cs);
                    g.em = make_double2(cs, -sn);
                    g.ep = make_double2(cs, sn);
                    const double2 z = cscal(zk, rr);
                    if (hk::cabs_(z) >= 1.0e-200) {
                        act = true;
                        double2 h0, h1;
                        hk::hankel01(z, h0, h1);
                        hz0 = h0;
                        hz1 = cscal(h1, rs);
                        zr = cscal(cinv(z), rs);
                    }
                }
                // upward: h_m for m = 0 .. p+1; emit order n = m - 1
                double2 hm2 = make_double2(0.0, 0.0), hm1 = hm2, hc = hm2;  // h_{m-2}, h_{m-1}, h_m
                double2 pw = make_double2(1.0, 0.0);
                for (int m = 0; m <= p + 1; m++) {
                    double2 hn;
                    if (!act) hn = make_double2(0.0, 0.0);
                    else if (m == 0) hn = hz0;
                    else if (m == 1) hn = hz1;
                    else hn = csub(cmul(cscal(zr, 2.0 * (m - 1)), hc), cscal(hm1, rs2));
                    hm2 = hm1;
                    hm1 = hc;
                    hc = hn;
                    if (m == 0) continue;
                    // emit n = m - 1 with h_{n-1} = hm2, h_n = hm1, h_{n+1} = hc
                    const int n = m - 1;
                    for (int c = 0; c < nd; c++) {
                        double2 cp = make_double2(0.0, 0.0), cm = cp;
                        if (act)
                            contrib(n, hm2, hm1, hc, pw, g, zk, 1.0 / rs, ifc,
                                    ifc ? charge[(long long)k * nd + c] : cp, ifd,
                                    ifd ? dipstr[(long long)k * nd + c] : cp,
                                    ifd ? dipvec[(long long)k * nd + c] : cp, cp, cm);
                        emit_warp(E, n, nd, c, cp, cm, lane);
                    }
                    pw = cmul(pw, g.em);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// M2M / L2L / M2L: out_i (+)= S_|i| sum_j in_j T(i - j) pw[e(i, j)], one
// thread per (box, i, channel).  kind 0: M2M (e = |j| + |i-j| - |i|),
// 1: L2L (e = |i-j| + |i| - |j|), 2: M2L (e = |i| + |j| - |i-j|).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 toeplitz_sum(const double2 *__restrict__ in, int n1, int nd,
                                                const double2 *__restrict__ T, int i,
                                                const double *__restrict__ pw, int kind) {
    double2 acc = make_double2(0.0, 0.0);
    const int ai = abs(i);
    for (int j = -n1; j <= n1; j++) {
        const int aj = abs(j), aij = abs(i - j);
        const int e = kind == 0 ? aj + aij - ai : (kind == 1 ? aij + ai - aj : ai + aj - aij);
        const double2 t = cmul(in[(long long)j * nd], T[i - j]);
        acc.x = fma(t.x, pw[e], acc.x);
        acc.y = fma(t.y, pw[e], acc.y);
    }
    return acc;
}

// M2M for the parents of level l (children at l + 1).
__global__ void __launch_bounds__(256) helm_m2m_kernel(
    int lo, int hi, int nd, const int *__restrict__ nchild, const int *__restrict__ child,
    const int2 *__restrict__ sse, const HLevel *__restrict__ lv, int l,
    const double2 *__restrict__ T, const double *__restrict__ S, const double *__restrict__ pw,
    double2 *__restrict__ mp) {
    const HLevel Lp = lv[l], Lc = lv[l + 1];
    const int n2 = Lp.p, n1 = Lc.p, N = n1 + n2, w2 = 2 * n2 + 1;
    const int64_t tot = (int64_t)(hi - lo) * w2 * nd;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = lo + (int)(t / ((int64_t)w2 * nd));
        const int rem = (int)(t % ((int64_t)w2 * nd));
        const int i = rem / nd - n2, c = rem % nd;
        if (nchild[b] == 0) continue;
        double2 acc = make_double2(0.0, 0.0);
        for (int cs = 0; cs < 4; cs++) {
            const int cb = child[4 * b + cs];
            if (cb < 0) continue;
            const int2 r = sse[cb];
            if (r.y <= r.x) continue;
            const double2 *in = coef0(mp, Lc, cb, nd) + c;
            const double2 s = toeplitz_sum(in, n1, nd, T + (size_t)cs * (2 * N + 1) + N, i, pw, 0);
            acc = cadd(acc, s);
        }
        double2 *o = coef0(mp, Lp, b, nd) + (long long)i * nd + c;
        *o = cscal(acc, S[abs(i)]);
    }
}

// L2L from the boxes of level l to their children.
__global__ void __launch_bounds__(256) helm_l2l_kernel(
    int lo, int hi, int nd, const int *__restrict__ parent, const int *__restrict__ child,
    const HLevel *__restrict__ lv, int l, const double2 *__restrict__ T,
    const double *__restrict__ S, const double *__restrict__ pw, double2 *__restrict__ loc) {
    const HLevel Lp = lv[l], Lc = lv[l + 1];
    const int n1 = Lp.p, n2 = Lc.p, N = n1 + n2, w2 = 2 * n2 + 1;
    const int64_t tot = (int64_t)(hi - lo) * w2 * nd;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = lo + (int)(t / ((int64_t)w2 * nd));
        const int rem = (int)(t % ((int64_t)w2 * nd));
        const int i = rem / nd - n2, c = rem % nd;
        const int pb = parent[b];
        int cs = 0;
        for (int j = 1; j < 4; j++)
            if (child[4 * pb + j] == b) cs = j;
        const double2 *in = coef0(loc, Lp, pb, nd) + c;
        const double2 s = toeplitz_sum(in, n1, nd, T + (size_t)cs * (2 * N + 1) + N, i, pw, 1);
        double2 *o = coef0(loc, Lc, b, nd) + (long long)i * nd + c;
        *o = cadd(*o, cscal(s, S[abs(i)]));
    }
}

// M2L over list 2 at level l; tables per offset (ix, iy) in [-3, 3]^2.
__global__ void __launch_bounds__(256) helm_m2l_kernel(
    int lo, int hi, int nd, const int *__restrict__ nlist2, const int *__restrict__ list2,
    const double2 *__restrict__ centers, const int2 *__restrict__ sse,
    const int2 *__restrict__ tse, int sp, int tp, double bs, const HLevel *__restrict__ lv,
    int l, const double2 *__restrict__ T, const double *__restrict__ pw,
    const double2 *__restrict__ mp, double2 *__restrict__ loc) {
    const HLevel L = lv[l];
    const int p = L.p, w = 2 * p + 1, tw = 4 * p + 1;
    const int64_t tot = (int64_t)(hi - lo) * w * nd;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = lo + (int)(t / ((int64_t)w * nd));
        const int rem = (int)(t % ((int64_t)w * nd));
        const int i = rem / nd - p, c = rem % nd;
        const int n2l = nlist2[b];
        if (n2l == 0) continue;
        int npts = 0;
        if (sp) npts += sse[b].y - sse[b].x;
        if (tp) npts += tse[b].y - tse[b].x;
        if (npts <= 0) continue;
        const double2 cb = centers[b];
        double2 acc = make_double2(0.0, 0.0);
        for (int e = 0; e < n2l; e++) {
            const int sb = list2[b * 27 + e];
            const double2 cs = centers[sb];
            const int ix = (int)rint((cb.x - cs.x) / bs), iy = (int)rint((cb.y - cs.y) / bs);
            const double2 *Tt = T + (size_t)((iy + 3) * 7 + (ix + 3)) * tw + 2 * p;
            const double2 s = toeplitz_sum(coef0(mp, L, sb, nd) + c, p, nd, Tt, i, pw, 2);
            acc = cadd(acc, s);
        }
        double2 *o = coef0(loc, L, b, nd) + (long long)i * nd + c;
        *o = cadd(*o, acc);
    }
}

// M2L over list 2 at level l for tiles of kHTile target boxes with the
// same child position (plan_slots): every slot is one offset for the whole
// tile, so a thread per two consecutive output coefficients (i0, i0 + 1,
// channel) reads each table entry once for the tile's boxes and both
// outputs (T[i0 + 1 - j] is the previous step's T[i0 - j]), and the source
// coefficients are broadcasts.  A block of at most 128 threads takes as
// many tiles at once as it has groups of p + 1 (times nd) threads, at most
// kHGroups, packed
// without padding (a warp may span two tiles: fewer idle lanes measured
// faster than whole warps per tile); with more coefficients than threads
// one tile loops over them.  Missing sources read the zero block `zero`
// ((2p + 1) nd zeros), so every slot does the same work.
//
// The weight rs^e, e = |i| + |j| - |i - j|, of helm_m2l_kernel
// (toeplitz_sum, kind 2) is 1 when i and j differ in sign or one is 0, and
// rs^(2 min(|i|, |j|)) otherwise; it factors as rs^|i| rs^|j| rs^-|i - j|.
// SC (scaled form): T holds T_q rs^-|q| and mp the multipoles times rs^|j|
// (helm_scale_mp_kernel), so the j loop is a plain complex multiply-add and
// rs^|i| (pw[|i|]) scales the sum; the host takes it where those powers
// stay far inside the FP64 range.  Otherwise the weight is applied per
// term, from the case split above.
constexpr int kHTile = 4;  // boxes per tile (8 measured slower: registers)
constexpr int kHGroups = 8;
struct HTiles {
    int tb[5];     // tiles of the level's four segments: [tb[c], tb[c + 1])
    int start[4];  // first target of each segment
    int count[4];  // targets of each segment
};

template <bool SC, bool SPLIT>
__global__ void __launch_bounds__(128, 5) helm_m2l_tile_kernel(
    HTiles lt, const int *__restrict__ boxes, const int *__restrict__ slots,
    const int2 *__restrict__ dxy, int nd, const HLevel *__restrict__ lv, int l,
    const double2 *__restrict__ T, const double *__restrict__ pw,
    const double2 *__restrict__ zero, const double2 *__restrict__ mp,
    double2 *__restrict__ loc, double2 *__restrict__ part) {
    constexpr int R = kHTile;
    __shared__ int s_src[kHGroups][R][27];
    __shared__ int s_trg[kHGroups][R];
    __shared__ int s_q[kHGroups][R];
    __shared__ int s_cp[kHGroups];
    const HLevel L = lv[l];
    const int p = L.p, tw = 4 * p + 1, wn = (p + 1) * nd;  // a thread per two outputs
    const int G = wn <= (int)blockDim.x ? min(kHGroups, (int)blockDim.x / wn) : 1;
    const int ntiles = lt.tb[4] - lt.tb[0];
    // slots [k0, k1) of slice blockIdx.y; with several slices each writes
    // its own partial sums (part: [slice][level target][(2p + 1) nd])
    const int k0 = SPLIT ? blockIdx.y * 27 / gridDim.y : 0;
    const int k1 = SPLIT ? (blockIdx.y + 1) * 27 / gridDim.y : 27;
    for (int base = blockIdx.x * G; base < ntiles; base += gridDim.x * G) {
        __syncthreads();  // the previous pass's reads of the shared tables are done
        for (int e = threadIdx.x; e < G * R * 27; e += blockDim.x) {
            const int g = e / (R * 27), r = (e / 27) % R, k = e % 27;
            const int tile = base + g;
            int v = -1, tb = -1, cp = 0;
            if (tile < ntiles) {
                const int t = lt.tb[0] + tile;
                while (cp < 3 && t >= lt.tb[cp + 1]) cp++;
                const int q = lt.start[cp] + (t - lt.tb[cp]) * R + r;
                if (q < lt.start[cp] + lt.count[cp]) {
                    v = slots[(size_t)q * 27 + k];
                    tb = boxes[q];
                    if (k == 0) s_q[g][r] = q - lt.start[0];
                }
            }
            s_src[g][r][k] = v;
            if (k == 0) s_trg[g][r] = tb;
            if (k == 0 && r == 0) s_cp[g] = cp;
        }
        __syncthreads();
        for (int u = threadIdx.x; u < G * wn; u += blockDim.x) {
            const int g = u / wn, o = u - g * wn;
            if (s_trg[g][0] < 0) continue;  // past the last tile
            // outputs i0 and i0 + 1 (the second absent for i0 = p)
            const int i0 = 2 * (o / nd) - p, c = o - (o / nd) * nd;
            const bool two = i0 < p;
            const int i1 = i0 + 1, ai0 = abs(i0), ai1 = abs(i1), cp = s_cp[g];
            const double c0 = pw[2 * ai0], c1 = pw[2 * min(ai1, p)], w0 = pw[0];
            double2 acc0[R], acc1[R];
#pragma unroll
            for (int r = 0; r < R; r++) acc0[r] = acc1[r] = make_double2(0.0, 0.0);
            for (int k = k0; k < k1; k++) {
                const double2 *in[R];
                bool any = false;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const int sb = s_src[g][r][k];
                    // coefficient j = -p of this channel
                    in[r] = (sb >= 0 ? coef0(mp, L, sb, nd) : zero + (size_t)p * nd) + c -
                            (size_t)p * nd;
                    any |= sb >= 0;
                }
                if (!any) continue;
                const int2 d = dxy[cp * 27 + k];
                // T[i0 - j] from j = -p down; T[i1 - j] is the previous step's T[i0 - j]
                const double2 *tp = T + (size_t)((3 - d.y) * 7 + (3 - d.x)) * tw + 2 * p + i0 + p;
                double2 tb = two ? tp[1] : make_double2(0.0, 0.0);
                for (int j = -p; j <= p; j++, tp--) {
                    const double2 ta = *tp;
                    double2 t0 = ta, t1 = tb;
                    tb = ta;
                    if (!SC) {
                        const int aj = abs(j);
                        const bool s0 = (i0 > 0 && j > 0) || (i0 < 0 && j < 0);
                        const bool s1 = (i1 > 0 && j > 0) || (i1 < 0 && j < 0);
                        const double pj = pw[2 * min(aj, p)];
                        const double w0j = s0 ? (aj <= ai0 ? pj : c0) : w0;
                        const double w1j = s1 ? (aj <= ai1 ? pj : c1) : w0;
                        t0 = make_double2(t0.x * w0j, t0.y * w0j);
                        t1 = make_double2(t1.x * w1j, t1.y * w1j);
                    }
#pragma unroll
                    for (int r = 0; r < R; r++) {
                        const double2 m = *in[r];
                        in[r] += nd;
                        acc0[r].x = fma(m.x, t0.x, acc0[r].x);
                        acc0[r].x = fma(-m.y, t0.y, acc0[r].x);
                        acc0[r].y = fma(m.x, t0.y, acc0[r].y);
                        acc0[r].y = fma(m.y, t0.x, acc0[r].y);
                        acc1[r].x = fma(m.x, t1.x, acc1[r].x);
                        acc1[r].x = fma(-m.y, t1.y, acc1[r].x);
                        acc1[r].y = fma(m.x, t1.y, acc1[r].y);
                        acc1[r].y = fma(m.y, t1.x, acc1[r].y);
                    }
                }
            }
            const double sc0 = SC ? pw[ai0] : 1.0, sc1 = SC ? pw[min(ai1, p)] : 1.0;
#pragma unroll
            for (int r = 0; r < R; r++) {
                if (s_trg[g][r] < 0) continue;
                const double2 v0 = SC ? cscal(acc0[r], sc0) : acc0[r];
                const double2 v1 = SC ? cscal(acc1[r], sc1) : acc1[r];
                if (SPLIT) {  // this slice's partial sums, added in order by helm_m2l_sum_kernel
                    const int nq = lt.start[3] + lt.count[3] - lt.start[0];
                    double2 *op = part + ((size_t)blockIdx.y * nq + s_q[g][r]) * (2 * p + 1) * nd +
                                  (size_t)(i0 + p) * nd + c;
                    op[0] = v0;
                    if (two) op[nd] = v1;
                } else {
                    double2 *op = coef0(loc, L, s_trg[g][r], nd) + (long long)i0 * nd + c;
                    *op = cadd(*op, v0);
                    if (two) op[nd] = cadd(op[nd], v1);
                }
            }
        }
    }
}

// Sum of the slices' partial M2L sums of helm_m2l_tile_kernel, in slice
// order, into the local expansions of the level's targets.
__global__ void __launch_bounds__(256) helm_m2l_sum_kernel(
    int nq, int wf, int nslice, const double2 *__restrict__ part, const int *__restrict__ boxes,
    int q_lo, const HLevel *__restrict__ lv, int l, int nd, double2 *__restrict__ loc) {
    const HLevel L = lv[l];
    const long long n = (long long)nq * wf;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(t / wf), o = (int)(t - (long long)q * wf);
        double2 acc = make_double2(0.0, 0.0);
        for (int y = 0; y < nslice; y++) acc = cadd(acc, part[(size_t)y * n + t]);
        double2 *op = coef0(loc, L, boxes[q_lo + q], nd) - (long long)L.p * nd + o;
        *op = cadd(*op, acc);
    }
}

// Scaled multipoles of the level-l boxes for the scaled M2L form:
// out = mp * rs^|j| for coefficient j (pw[|j|]).
__global__ void __launch_bounds__(256) helm_scale_mp_kernel(
    long long off, long long n, int p, int nd, const double *__restrict__ pw,
    const double2 *__restrict__ mp, double2 *__restrict__ out) {
    const int wn = (2 * p + 1) * nd;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t % wn) / nd - p;
        out[off + t] = cscal(mp[off + t], pw[abs(j)]);
    }
}

// The tile form of the Helmholtz M2L unless FMM2D_B200_HELM_M2L=box.
bool helm_m2l_tiled() {
    const char *e = getenv("FMM2D_B200_HELM_M2L");
    return !(e && !strcmp(e, "box"));
}

// The tensor-core form in the mixed mode unless FMM2D_B200_HELM_M2L is
// "box" or "tile" (both FP64).
bool helm_m2l_tc_enabled() {
    const char *e = getenv("FMM2D_B200_HELM_M2L");
    return !(e && (!strcmp(e, "box") || !strcmp(e, "tile")));
}

// ---------------------------------------------------------------------------
// M2P + L2P for one point set: thread per point.
// ---------------------------------------------------------------------------
struct DScale {
    double2 z1, z2, z3, z4;  // k/(2s), k s/2, i k/(2s), i k s/2
};

__device__ __forceinline__ DScale dscale(double2 zk, double s) {
    DScale d;
    d.z1 = cscal(zk, 0.5 / s);
    d.z2 = cscal(zk, 0.5 * s);
    d.z3 = hk::cmuli(d.z1);
    d.z4 = hk::cmuli(d.z2);
    return d;
}

struct Coefs {
    const double2 *c0;  // coefficient 0 of the channel
    int p, nd;
    __device__ __forceinline__ double2 at(int n) const {
        return (n < -p || n > p) ? make_double2(0.0, 0.0) : c0[(long long)n * nd];
    }
    // mk_mpoleg (helmrouts2d.c:187-233): x- and y-derivative sequences
    __device__ __forceinline__ double2 dx(int n, const DScale &d) const {
        const double2 a = n >= 0 ? d.z2 : d.z1, b = n >= 1 ? d.z1 : d.z2;
        return csub(cmul(a, at(n + 1)), cmul(b, at(n - 1)));
    }
    __device__ __forceinline__ double2 dy(int n, const DScale &d) const {
        const double2 a = n >= 0 ? d.z4 : d.z3, b = n >= 1 ? d.z3 : d.z4;
        return cadd(cmul(a, at(n + 1)), cmul(b, at(n - 1)));
    }
    // mk_mpoleh (helmrouts2d.c:235-292): the same recurrences applied again
    __device__ __forceinline__ double2 dxx(int n, const DScale &d) const {
        const double2 a = n >= 0 ? d.z2 : d.z1, b = n >= 1 ? d.z1 : d.z2;
        return csub(cmul(a, dx(n + 1, d)), cmul(b, dx(n - 1, d)));
    }
    __device__ __forceinline__ double2 dxy(int n, const DScale &d) const {
        const double2 a = n >= 0 ? d.z4 : d.z3, b = n >= 1 ? d.z3 : d.z4;
        return cadd(cmul(a, dx(n + 1, d)), cmul(b, dx(n - 1, d)));
    }
    __device__ __forceinline__ double2 dyy(int n, const DScale &d) const {
        const double2 a = n >= 0 ? d.z4 : d.z3, b = n >= 1 ? d.z3 : d.z4;
        return cadd(cmul(a, dy(n + 1, d)), cmul(b, dy(n - 1, d)));
    }
};

struct Acc {
    double2 p, gx, gy, hxx, hxy, hyy;
    __device__ void zero() {
        p = gx = gy = hxx = hxy = hyy = make_double2(0.0, 0.0);
    }
    __device__ void scale(double2 s) {
        p = cmul(p, s);
        gx = cmul(gx, s);
        gy = cmul(gy, s);
        hxx = cmul(hxx, s);
        hxy = cmul(hxy, s);
        hyy = cmul(hyy, s);
    }
    __device__ void scale(double s) {
        p = cscal(p, s);
        gx = cscal(gx, s);
        gy = cscal(gy, s);
        hxx = cscal(hxx, s);
        hxy = cscal(hxy, s);
        hyy = cscal(hyy, s);
    }
    __device__ void add(const Acc &o) {
        p = cadd(p, o.p);
        gx = cadd(gx, o.gx);
        gy = cadd(gy, o.gy);
        hxx = cadd(hxx, o.hxx);
        hxy = cadd(hxy, o.hxy);
        hyy = cadd(hyy, o.hyy);
    }
};

// Adds the order +n / -n terms with basis values ep = E_n, em = E_-n.
template <int PGH>
__device__ __forceinline__ void acc_terms(Acc &a, const Coefs &C, const DScale &d, int n,
                                          double2 ep, double2 em) {
    const int p = C.p;
    if (n <= p) {
        cfma(a.p, C.at(n), ep);
        if (n) cfma(a.p, C.at(-n), em);
    }
    if (PGH >= 2 && n <= p + 1) {
        cfma(a.gx, C.dx(n, d), ep);
        cfma(a.gy, C.dy(n, d), ep);
        if (n) {
            cfma(a.gx, C.dx(-n, d), em);
            cfma(a.gy, C.dy(-n, d), em);
        }
    }
    if (PGH >= 3) {
        cfma(a.hxx, C.dxx(n, d), ep);
        cfma(a.hxy, C.dxy(n, d), ep);
        cfma(a.hyy, C.dyy(n, d), ep);
        if (n) {
            cfma(a.hxx, C.dxx(-n, d), em);
            cfma(a.hxy, C.dxy(-n, d), em);
            cfma(a.hyy, C.dyy(-n, d), em);
        }
    }
}

template <int PGH>
__global__ void __launch_bounds__(128) helm_far_kernel(
    int n, const double2 *__restrict__ pos, const int *__restrict__ leaf,
    const int *__restrict__ level, const double2 *__restrict__ centers,
    const int *__restrict__ nlist3, const int *__restrict__ list3, const HLevel *__restrict__ lv,
    int nlevels, const double2 *__restrict__ mp, const double2 *__restrict__ loc, int nd,
    double2 zk, double2 *__restrict__ pot, double2 *__restrict__ grad,
    double2 *__restrict__ hess) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int b = leaf[t];
        const int l = level[b];
        const double2 x = pos[t];
        for (int c = 0; c < nd; c++) {
            Acc tot;
            tot.zero();
            // M2P over list 3 (boxes of level l + 1)
            if (l + 1 <= nlevels && lv[l + 1].flag) {
                const HLevel L3 = lv[l + 1];
                const int nl3 = nlist3[b];
                const double rs = L3.rs;
                const DScale ds = dscale(zk, rs);
                const int N = L3.p + PGH - 1;
                for (int e = 0; e < nl3; e++) {
                    const int jb = list3[b * 20 + e];
                    const double2 cc = centers[jb];
                    const double dx = x.x - cc.x, dy = x.y - cc.y;
                    const double r = sqrt(dx * dx + dy * dy);
                    const double2 z = cscal(zk, r);
                    if (hk::cabs_(z) < 1.0e-200) continue;
                    const double th = (dx == 0.0 && dy == 0.0) ? 0.0 : atan2(dy, dx);
                    double sn, cs;
                    sincos(th, &sn, &cs);
                    const double2 w = make_double2(cs, sn);
                    double2 h0, h1;
                    hk::hankel01(z, h0, h1);
                    const double2 zr = cscal(cinv(z), rs);
                    const Coefs C{coef0(mp, L3, jb, nd) + c, L3.p, nd};
                    Acc a;
                    a.zero();
                    acc_terms<PGH>(a, C, ds, 0, h0, h0);
                    double2 hm1 = h0, hc = cscal(h1, rs), wn = w;
                    for (int m = 1; m <= N; m++) {
                        if (m >= 2) {
                            const double2 hn = csub(cmul(cscal(zr, 2.0 * (m - 1)), hc), cscal(hm1, rs * rs));
                            hm1 = hc;
                            hc = hn;
                        }
                        const double2 ep = cmul(wn, hc);
                        const double2 em = cscal(cmul(cconj(wn), hc), (m & 1) ? -1.0 : 1.0);
                        acc_terms<PGH>(a, C, ds, m, ep, em);
                        wn = cmul(wn, w);
                    }
                    tot.add(a);
                }
            }
            // L2P of the leaf's own local expansion
            if (l >= 2 && lv[l].flag) {
                const HLevel L = lv[l];
                const double rs = L.rs, rs2 = rs * rs;
                const DScale ds = dscale(zk, 1.0 / rs);
                const Coefs C{coef0(loc, L, b, nd) + c, L.p, nd};
                const double2 cc = centers[b];
                const double dx = x.x - cc.x, dy = x.y - cc.y;
                const double r = sqrt(dx * dx + dy * dy);
                const double2 z = cscal(zk, r);
                const double th = (dx == 0.0 && dy == 0.0) ? 0.0 : atan2(dy, dx);
                double sn, cs;
                sincos(th, &sn, &cs);
                const double2 w = make_double2(cs, sn);
                const int N = L.p + PGH - 1;
                Acc a;
                a.zero();
                if (hk::cabs_(z) < 1.0e-200) {
                    acc_terms<PGH>(a, C, ds, 0, make_double2(1.0, 0.0), make_double2(1.0, 0.0));
                } else {
                    const double2 zinv = cinv(z), zr = cscal(zinv, rs);
                    const bool lower = z.y < 0.0;
                    const int ntop = jb_ntop(L.p + 3, zinv);
                    double2 wn = make_double2(1.0, 0.0);
                    for (int m = 0; m < N; m++) wn = cmul(wn, w);  // w^N
                    const double2 wc = cconj(w);
                    double2 gp1 = make_double2(0.0, 0.0), gc = make_double2(1.0, 0.0);
                    double2 psi = make_double2(0.0, 0.0);
                    for (int i = ntop - 1; i >= 1; i--) {
                        double2 gm1 = csub(cmul(cscal(zr, 2.0 * i), gc), cscal(gp1, rs2));
                        if (gm1.x * gm1.x + gm1.y * gm1.y > 1.0e40) {
                            gc = cscal(gc, 1.0e-40);
                            gm1 = cscal(gm1, 1.0e-40);
                            psi = cscal(psi, 1.0e-40);
                            a.scale(1.0e-40);
                        }
                        psi = cadd(cscal(psi, rs), cmul(gc, zm_pow(i, lower)));
                        if (i <= N) {
                            const double2 ep = cmul(wn, gc);
                            const double2 em = cscal(cmul(cconj(wn), gc), (i & 1) ? -1.0 : 1.0);
                            acc_terms<PGH>(a, C, ds, i, ep, em);
                            wn = cmul(wn, wc);
                        }
                        gp1 = gc;
                        gc = gm1;
                    }
                    psi = cadd(cscal(psi, 2.0 * rs), gc);
                    acc_terms<PGH>(a, C, ds, 0, gc, gc);
                    const double2 ez = lower ? hk::cexp_(make_double2(-z.y, z.x))
                                             : hk::cexp_(make_double2(z.y, -z.x));
                    a.scale(hk::cdiv_(ez, psi));
                }
                tot.add(a);
            }
            tot.scale(make_double2(0.0, 0.25));  // i / 4
            if (PGH >= 1) pot[(long long)t * nd + c] = tot.p;
            if (PGH >= 2) {
                grad[((long long)t * 2 + 0) * nd + c] = tot.gx;
                grad[((long long)t * 2 + 1) * nd + c] = tot.gy;
            }
            if (PGH >= 3) {
                hess[((long long)t * 3 + 0) * nd + c] = tot.hxx;
                hess[((long long)t * 3 + 1) * nd + c] = tot.hxy;
                hess[((long long)t * 3 + 2) * nd + c] = tot.hyy;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// P2P pairs (h2d_direct*, helmkernels2d.c:21-520).
// ---------------------------------------------------------------------------
template <bool REALK>
__device__ __forceinline__ void pair_h01(double2 z, double2 &h0, double2 &h1) {
    if (REALK && z.x < 8.0) {
        h0 = make_double2(j0(z.x), y0(z.x));
        h1 = make_double2(j1(z.x), y1(z.x));
    } else {
        hk::hankel01(z, h0, h1);
    }
}

// Adds the interaction of one source with one target to a, for channel c.
template <int PGH, bool REALK>
__device__ __forceinline__ void pair_add(Acc &a, double dx, double dy, double2 zk, double thresh,
                                         bool le, bool ifc, double2 q, bool ifd, double2 d,
                                         double2 v) {
    const double rr = dx * dx + dy * dy;
    const double r = sqrt(rr);
    const double2 z = cscal(zk, r);
    const double az = hk::cabs_(z);
    if (le ? (az <= thresh) : (az < thresh)) return;
    double2 h0, h1;
    pair_h01<REALK>(z, h0, h1);
    const double2 i4 = make_double2(0.0, 0.25);
    if (ifc) {
        cfma(a.p, cmul(h0, i4), q);
        if (PGH >= 2) {
            // cdd = -h1 (k i/4 / r)
            const double2 cdd = cscal(cmul(h1, cscal(cmul(zk, i4), 1.0 / r)), -1.0);
            const double2 cd = cmul(cdd, q);
            a.gx = cadd(a.gx, cscal(cd, dx));
            a.gy = cadd(a.gy, cscal(cd, dy));
            if (PGH >= 3) {
                const double2 cdd2 = cscal(cmul(zk, i4), 1.0 / r / rr);
                const double2 h2z = cadd(cscal(cmul(z, h0), -1.0), cscal(h1, 2.0));
                const double2 hf1 = csub(cscal(h2z, dx * dx), cscal(h1, rr));
                const double2 hf2 = cscal(h2z, dx * dy);
                const double2 hf3 = csub(cscal(h2z, dy * dy), cscal(h1, rr));
                const double2 c2 = cmul(cdd2, q);
                cfma(a.hxx, c2, hf1);
                cfma(a.hxy, c2, hf2);
                cfma(a.hyy, c2, hf3);
            }
        }
    }
    if (ifd) {
        const double2 cdd = cmul(cscal(h1, 1.0 / r), cmul(zk, i4));
        const double dot = dx * v.x + dy * v.y;
        cfma(a.p, cmul(cdd, d), make_double2(dot, 0.0));
        if (PGH >= 2) {
            const double ct = dx / r, st = dy / r;
            const double2 zi = cinv(z);
            const double2 h2 = csub(cmul(cscal(h1, 2.0), zi), h0);
            const double2 cdd2 = cscal(cmul(cmul(zk, zk), i4), -1.0);
            const double2 hh0 = cscal(h0, 0.5);
            const double2 hf1 = csub(cscal(h2, ct * ct - 0.5), hh0);
            const double2 hf2 = cscal(h2, ct * st);
            const double2 hf3 = csub(cscal(h2, st * st - 0.5), hh0);
            const double2 cd = cmul(cdd2, d);
            const double2 hxx = cmul(cd, hf1), hxy = cmul(cd, hf2), hyy = cmul(cd, hf3);
            a.gx = cadd(a.gx, cadd(cscal(hxx, v.x), cscal(hxy, v.y)));
            a.gy = cadd(a.gy, cadd(cscal(hxy, v.x), cscal(hyy, v.y)));
            if (PGH >= 3) {
                const double2 h3 = csub(cmul(cscal(h2, 4.0), zi), h1);
                const double2 mh1 = cscal(h1, -0.5), mh3 = cscal(h3, -0.5);
                const double2 hxxx1 = cscal(cadd(cscal(mh1, -1.5), cscal(mh3, ct * ct - 0.5 - st * st)), ct);
                const double2 hxxy1 = cscal(cadd(cscal(mh1, -0.5), cscal(mh3, 1.5 * ct * ct - 0.5 * st * st)), st);
                const double2 hxyy1 = cscal(cadd(cscal(mh1, -0.5), cscal(mh3, 1.5 * st * st - 0.5 * ct * ct)), ct);
                const double2 hyyy1 = cscal(cadd(cscal(mh1, -1.5), cscal(mh3, st * st - 0.5 - ct * ct)), st);
                const double2 cd3 = cscal(cmul(cmul(cmul(cmul(zk, zk), zk), d), i4), -1.0);
                a.hxx = cadd(a.hxx, cmul(cd3, cadd(cscal(hxxx1, v.x), cscal(hxxy1, v.y))));
                a.hxy = cadd(a.hxy, cmul(cd3, cadd(cscal(hxxy1, v.x), cscal(hxyy1, v.y))));
                a.hyy = cadd(a.hyy, cmul(cd3, cadd(cscal(hxyy1, v.x), cscal(hyyy1, v.y))));
            }
        }
    }
}

template <int PGH>
__device__ __forceinline__ void store_add(const Acc &a, long long t, int nd, int c, double2 *pot,
                                          double2 *grad, double2 *hess) {
    double2 &o = pot[t * nd + c];
    o = cadd(o, a.p);
    if (PGH >= 2) {
        double2 &g0 = grad[(t * 2 + 0) * nd + c];
        g0 = cadd(g0, a.gx);
        double2 &g1 = grad[(t * 2 + 1) * nd + c];
        g1 = cadd(g1, a.gy);
    }
    if (PGH >= 3) {
        double2 &h0 = hess[(t * 3 + 0) * nd + c];
        h0 = cadd(h0, a.hxx);
        double2 &h1 = hess[(t * 3 + 1) * nd + c];
        h1 = cadd(h1, a.hxy);
        double2 &h2 = hess[(t * 3 + 2) * nd + c];
        h2 = cadd(h2, a.hyy);
    }
}

// P2P over list 1 for one point set (the outputs already hold the far field).
template <int PGH, bool REALK>
__global__ void __launch_bounds__(128) helm_p2p_kernel(
    int n, const double2 *__restrict__ pos, const int *__restrict__ leaf,
    const int *__restrict__ nlist1, const int *__restrict__ list1, const int2 *__restrict__ sse,
    const double2 *__restrict__ src, const double2 *__restrict__ charge,
    const double2 *__restrict__ dipstr, const double2 *__restrict__ dipvec, int ifc, int ifd,
    int nd, double2 zk, double thresh, double2 *__restrict__ pot, double2 *__restrict__ grad,
    double2 *__restrict__ hess) {
    const bool le = ifc && !ifd && PGH == 1;
    const double2 zero = make_double2(0.0, 0.0);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int b = leaf[t];
        const double2 x = pos[t];
        const int nl = nlist1[b];
        for (int c = 0; c < nd; c++) {
            Acc a;
            a.zero();
            for (int e = 0; e < nl; e++) {
                const int2 r = sse[list1[b * 13 + e]];
                for (int k = r.x; k < r.y; k++) {
                    const double2 y = src[k];
                    const long long kc = (long long)k * nd + c;
                    pair_add<PGH, REALK>(a, x.x - y.x, x.y - y.y, zk, thresh, le, ifc,
                                         ifc ? charge[kc] : zero, ifd, ifd ? dipstr[kc] : zero,
                                         ifd ? dipvec[kc] : zero);
                }
            }
            store_add<PGH>(a, t, nd, c, pot, grad, hess);
        }
    }
}

// P2P over list 1 for one point set with one warp per leaf (nd = 1): the
// leaf's list-1 sources are staged in shared memory in chunks, and the
// (target, source block) items of up to 32 targets are dealt to the lanes,
// each item summing its block into registers; the target's lane then adds
// the blocks' partial sums in block order.  Every lane runs the same
// number of pairs, where one thread per target ran as many pairs as its
// own leaf's list 1 held (lanes of one warp spanning leaves of different
// sizes idled).  Deterministic: every sum has a fixed order.
constexpr int kHfStage = 64;
constexpr int kHfWarps = 4;
constexpr int kHfItems = 64;

template <int PGH>
constexpr int hf_outs() { return PGH >= 3 ? 6 : (PGH >= 2 ? 3 : 1); }

template <int PGH>
constexpr size_t helm_p2p_flat_warp_bytes() {
    return (size_t)kHfStage * 4 * sizeof(double2) + 32 * sizeof(double2) +
           (size_t)kHfItems * hf_outs<PGH>() * sizeof(double2);
}

template <int PGH, bool REALK>
__global__ void __launch_bounds__(kHfWarps * 32) helm_p2p_flat_kernel(
    int nb, const int *__restrict__ nchild, const int2 *__restrict__ tse,
    const double2 *__restrict__ pos, const int *__restrict__ nlist1,
    const int *__restrict__ list1, const int2 *__restrict__ sse, const double2 *__restrict__ src,
    const double2 *__restrict__ charge, const double2 *__restrict__ dipstr,
    const double2 *__restrict__ dipvec, int ifc, int ifd, double2 zk, double thresh,
    double2 *__restrict__ pot, double2 *__restrict__ grad, double2 *__restrict__ hess) {
    constexpr int NO = hf_outs<PGH>();
    extern __shared__ __align__(16) unsigned char hf_smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double2 *s_pos = reinterpret_cast<double2 *>(hf_smem + (size_t)wib * helm_p2p_flat_warp_bytes<PGH>());
    double2 *s_q = s_pos + kHfStage, *s_d = s_q + kHfStage, *s_v = s_d + kHfStage;
    double2 *s_tgt = s_v + kHfStage;
    double2 *part = s_tgt + 32;
    const bool le = ifc && !ifd && PGH == 1;
    const double2 zero = make_double2(0.0, 0.0);
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += nwarps) {
        if (nchild[b] != 0) continue;
        const int2 tr = tse[b];
        const int ntot = tr.y - tr.x;
        const int n1 = nlist1[b];
        if (ntot <= 0 || n1 == 0) continue;
        int jstart = 0, jcount = 0;  // lane e < n1 holds list-1 entry e
        if (lane < n1) {
            const int2 r = sse[list1[b * 13 + lane]];
            jstart = r.x;
            jcount = r.y - r.x;
        }
        int jofs = jcount;
#pragma unroll
        for (int dd = 1; dd < 16; dd <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, jofs, dd);
            if (lane >= dd) jofs += o;
        }
        const int nsrc = __shfl_sync(0xffffffffu, jofs, n1 - 1);
        jofs -= jcount;
        if (nsrc == 0) continue;
        const int nchunk = (ntot + 31) / 32, T0 = (ntot + nchunk - 1) / nchunk;
        const int ns_eff = min(nsrc, kHfStage);
        for (int t0 = 0; t0 < ntot; t0 += T0) {
            const int T = min(T0, ntot - t0);
            __syncwarp();
            if (lane < T) s_tgt[lane] = pos[tr.x + t0 + lane];
            int B = 1, best = 1 << 30;
            for (int bb = 1; bb * T <= kHfItems; bb++) {
                const int cost = ((T * bb + 31) >> 5) * ((ns_eff + bb - 1) / bb);
                if (cost < best) {
                    best = cost;
                    B = bb;
                }
            }
            const int nit = T * B;
            Acc tot;
            tot.zero();
            for (int s0 = 0; s0 < nsrc; s0 += kHfStage) {
                const int nst = min(kHfStage, nsrc - s0);
                __syncwarp();
                for (int i0 = 0; i0 < nst; i0 += 32) {  // warp-uniform trip count
                    const int i = i0 + lane, gi = s0 + i;
                    int e = 0;
                    for (int u = 1; u < n1; u++)
                        if (__shfl_sync(0xffffffffu, jofs, u) <= gi) e = u;
                    const int k = __shfl_sync(0xffffffffu, jstart, e) + gi -
                                  __shfl_sync(0xffffffffu, jofs, e);
                    if (i >= nst) continue;
                    s_pos[i] = src[k];
                    s_q[i] = ifc ? charge[k] : zero;
                    s_d[i] = ifd ? dipstr[k] : zero;
                    s_v[i] = ifd ? dipvec[k] : zero;
                }
                __syncwarp();
                const int sb = (nst + B - 1) / B;
                for (int it = lane; it < nit; it += 32) {
                    const int t = it % T, blk = it / T;
                    const double2 x = s_tgt[t];
                    Acc a;
                    a.zero();
                    const int j1 = min(nst, blk * sb + sb);
                    for (int kk = blk * sb; kk < j1; kk++) {
                        const double2 y = s_pos[kk];
                        pair_add<PGH, REALK>(a, x.x - y.x, x.y - y.y, zk, thresh, le, ifc, s_q[kk],
                                             ifd, s_d[kk], s_v[kk]);
                    }
                    double2 *pp = part + (size_t)it * NO;
                    pp[0] = a.p;
                    if (PGH >= 2) {
                        pp[1] = a.gx;
                        pp[2] = a.gy;
                    }
                    if (PGH >= 3) {
                        pp[3] = a.hxx;
                        pp[4] = a.hxy;
                        pp[5] = a.hyy;
                    }
                }
                __syncwarp();
                if (lane < T) {
                    for (int blk = 0; blk < B; blk++) {
                        const double2 *pp = part + (size_t)(lane + blk * T) * NO;
                        tot.p = cadd(tot.p, pp[0]);
                        if (PGH >= 2) {
                            tot.gx = cadd(tot.gx, pp[1]);
                            tot.gy = cadd(tot.gy, pp[2]);
                        }
                        if (PGH >= 3) {
                            tot.hxx = cadd(tot.hxx, pp[3]);
                            tot.hxy = cadd(tot.hxy, pp[4]);
                            tot.hyy = cadd(tot.hyy, pp[5]);
                        }
                    }
                }
            }
            if (lane < T) store_add<PGH>(tot, (long long)(tr.x + t0 + lane), 1, 0, pot, grad, hess);
        }
    }
}

// All-pairs direct sum for one point set (adds).
template <int PGH, bool REALK>
__global__ void __launch_bounds__(128) helm_direct_kernel(
    int n, const double2 *__restrict__ pos, int ns, const double2 *__restrict__ src,
    const double2 *__restrict__ charge, const double2 *__restrict__ dipstr,
    const double2 *__restrict__ dipvec, int ifc, int ifd, int nd, double2 zk, double thresh,
    double2 *__restrict__ pot, double2 *__restrict__ grad, double2 *__restrict__ hess) {
    const bool le = ifc && !ifd && PGH == 1;
    const double2 zero = make_double2(0.0, 0.0);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const double2 x = pos[t];
        for (int c = 0; c < nd; c++) {
            Acc a;
            a.zero();
            for (int k = 0; k < ns; k++) {
                const double2 y = src[k];
                const long long kc = (long long)k * nd + c;
                pair_add<PGH, REALK>(a, x.x - y.x, x.y - y.y, zk, thresh, le, ifc,
                                     ifc ? charge[kc] : zero, ifd, ifd ? dipstr[kc] : zero,
                                     ifd ? dipvec[kc] : zero);
            }
            store_add<PGH>(a, t, nd, c, pot, grad, hess);
        }
    }
}

// List-2 pairs per level for the roofline (target boxes holding points of
// a set with outputs, as the M2L plan takes them).
__global__ void helm_count_m2l_kernel(int nb, const int *__restrict__ lev,
                                      const int *__restrict__ n2, const int2 *__restrict__ sse,
                                      const int2 *__restrict__ tse, int sp, int tp,
                                      unsigned long long *__restrict__ per_level) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int np = (sp ? sse[b].y - sse[b].x : 0) + (tp ? tse[b].y - tse[b].x : 0);
        if (lev[b] >= 2 && np > 0 && n2[b] > 0)
            atomicAdd(&per_level[lev[b]], (unsigned long long)n2[b]);
    }
}

__global__ void helm_leaf_of_kernel(int nb, const int *__restrict__ nchild,
                                    const int2 *__restrict__ se, int *__restrict__ leaf) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        if (nchild[b] != 0) continue;
        const int2 r = se[b];
        for (int k = r.x; k < r.y; k++) leaf[k] = b;
    }
}

unsigned grid_for(int64_t work, int block) {
    int64_t g = (work + block - 1) / block;
    if (g > (int64_t)kNumSM * 16) g = (int64_t)kNumSM * 16;
    if (g < 1) g = 1;
    return (unsigned)g;
}

// The per-level translation tables (host).
// T(m), m = -N..N, for the shift from center1 to center2 = center1 + d:
// T(0) = B_0, T(m) = zmul^m B_m, T(-m) = (-1)^m zinv^m B_m with
// zmul = e^{-i (atan2(d) - pi)} and B the scaled J (M2M, L2L) or H (M2L)
// sequence of k |d| (h2dmpmp / h2dlocloc / h2dmploc, helmrouts2d.c:736-1042).
void shift_table(double2 zk, double dx, double dy, int N, double rs1, bool hankel,
                 double2 *T) {
    const double r = std::sqrt(dx * dx + dy * dy);
    const double pi = 4.0 * std::atan(1.0);
    const double th = ((dx == 0.0 && dy == 0.0) ? 0.0 : std::atan2(dy, dx)) - pi;
    const double2 z = cscal(zk, r);
    std::vector<double2> B(N + 4);
    if (hankel)
        helm_hvec(N + 1, z, rs1, B.data());
    else
        helm_jvec(N + 3, z, rs1, B.data());
    const double2 zmul = make_double2(std::cos(th), -std::sin(th));
    const double2 zinv = make_double2(zmul.x, -zmul.y);
    double2 *T0 = T + N;
    T0[0] = B[0];
    double2 t1 = zmul, t2 = make_double2(-zinv.x, -zinv.y);
    for (int j = 1; j <= N; j++) {
        T0[j] = cmul(t1, B[j]);
        T0[-j] = cmul(t2, B[j]);
        t1 = cmul(t1, zmul);
        t2 = cscal(cmul(t2, zinv), -1.0);
    }
}

}  // namespace

namespace {

// Host translation tables of one evaluation.  Layout per level: M2M
// [4][2N+1] + S + pw, L2L likewise, M2L [49][4p+1] + pw (+ the scaled M2L
// table where it applies).
struct LevTab {
    size_t m2m = 0, m2m_s = 0, m2m_pw = 0, l2l = 0, l2l_s = 0, l2l_pw = 0, m2l = 0, m2l_pw = 0;
    size_t m2l_sc = 0;   // M2L table of the scaled form, T_q rs^-|q|
    bool sc_ok = false;  // the scaled form applies on this level
    double m2l_max = 0;  // largest |T_q| of the M2L table (tensor-core form's scale)
};
struct HTables {
    std::vector<LevTab> lt;
    std::vector<double2> ct;  // complex tables
    std::vector<double> rt;   // real tables
};
using HTabKey = std::tuple<double, double, double, double, int>;  // zk, eps, root box, depth

// The last kHTabCache table sets, shared by the threads of the process.
constexpr size_t kHTabCache = 16;
std::mutex g_htab_mu;
std::vector<std::pair<HTabKey, std::shared_ptr<HTables>>> g_htab;

std::shared_ptr<HTables> htables_find(const HTabKey &k) {
    std::lock_guard<std::mutex> lock(g_htab_mu);
    for (auto &e : g_htab)
        if (e.first == k) return e.second;
    return nullptr;
}

void htables_store(const HTabKey &k, const std::shared_ptr<HTables> &t) {
    std::lock_guard<std::mutex> lock(g_htab_mu);
    for (auto &e : g_htab)
        if (e.first == k) return;
    if (g_htab.size() >= kHTabCache) g_htab.erase(g_htab.begin());
    g_htab.emplace_back(k, t);
}

}  // namespace

void helmholtz_fmm(const Tree &T, const HelmProblem &P, cudaStream_t s) {
    const int nl = T.nlevels, nd = P.nd;
    const double2 zk = P.zk;
    const double pi = 4.0 * std::atan(1.0);
    // ---- per-level order, scale and bounds (hfmm2d.c, driver) ----
    std::vector<HLevel> hl(nl + 2);
    long long off = 0;
    for (int l = 0; l <= nl; l++) {
        HLevel &L = hl[l];
        const double bs = T.boxsize[l];
        const double2 zt = cscal(zk, bs / (2.0 * pi));
        L.rs = std::min(hk::cabs_(zt), 1.0);
        const int nt = helm_nterms(bs, zk, P.eps);
        if (nt < 0)
            throw FmmError(4, "Helmholtz expansion order exceeds 50000 (box too large "
                              "for the wavenumber)");
        L.p = nt;
        L.lstart = T.lstart[l];
        L.flag = zk.y * bs < 40.0 ? 1 : 0;
        L.off = off;
        off += (long long)(T.lend[l] - T.lstart[l]) * (2 * L.p + 1) * nd;
    }
    hl[nl + 1] = hl[nl];
    hl[nl + 1].flag = 0;
    DevBuf<HLevel> d_lv(nl + 2, s);
    FMM_CUDA(cudaMemcpyAsync(d_lv.get(), hl.data(), (nl + 2) * sizeof(HLevel),
                             cudaMemcpyHostToDevice, s));
    DevBuf<double2> mp(std::max<long long>(off, 1), s), loc(std::max<long long>(off, 1), s);
    mp.zero(s);
    loc.zero(s);
    // ---- translation tables (kept for calls with the same zk, eps, root
    // box and depth, which fix every level's order, scale and offsets) ----
    const HTabKey tkey{zk.x, zk.y, P.eps, T.boxsize[0], nl};
    std::shared_ptr<HTables> tabs = htables_find(tkey);
    if (!tabs) {
        tabs = std::make_shared<HTables>();
        std::vector<LevTab> &lt = tabs->lt;
        std::vector<double2> &ct = tabs->ct;
        std::vector<double> &rt = tabs->rt;
        lt.resize(nl + 1);
        auto powtab = [&](double r, int n) {
            const size_t o = rt.size();
            double v = 1.0;
            for (int e = 0; e <= n; e++) {
                rt.push_back(v);
                v *= r;
            }
            return o;
        };
        for (int l = 2; l <= nl; l++) {
            const HLevel &L = hl[l];
            if (l + 1 <= nl) {
                const HLevel &C = hl[l + 1];
                const double hb = T.boxsize[l + 1] / 2.0;
                // M2M: child (scale r1) -> parent (scale r2), d = parent - child
                {
                    const int n1 = C.p, n2 = L.p, N = n1 + n2;
                    lt[l].m2m = ct.size();
                    ct.resize(ct.size() + (size_t)4 * (2 * N + 1));
                    for (int cs = 0; cs < 4; cs++) {
                        const double sx = (cs & 1) ? 1.0 : -1.0, sy = (cs & 2) ? 1.0 : -1.0;
                        shift_table(zk, -sx * hb, -sy * hb, N, C.rs, false,
                                    ct.data() + lt[l].m2m + (size_t)cs * (2 * N + 1));
                    }
                    lt[l].m2m_s = rt.size();
                    double f = 1.0;
                    for (int i = 0; i <= n2; i++) {
                        rt.push_back(f);
                        f = f * C.rs / L.rs;
                    }
                    lt[l].m2m_pw = powtab(C.rs, 2 * n1);
                }
                // L2L: parent (scale r1) -> child (scale r2), d = child - parent
                {
                    const int n1 = L.p, n2 = C.p, N = n1 + n2;
                    lt[l].l2l = ct.size();
                    ct.resize(ct.size() + (size_t)4 * (2 * N + 1));
                    for (int cs = 0; cs < 4; cs++) {
                        const double sx = (cs & 1) ? 1.0 : -1.0, sy = (cs & 2) ? 1.0 : -1.0;
                        shift_table(zk, sx * hb, sy * hb, N, L.rs, false,
                                    ct.data() + lt[l].l2l + (size_t)cs * (2 * N + 1));
                    }
                    lt[l].l2l_s = rt.size();
                    double f = 1.0;
                    for (int i = 0; i <= n2; i++) {
                        rt.push_back(f);
                        f = f * C.rs / L.rs;
                    }
                    lt[l].l2l_pw = powtab(L.rs, 2 * n2);
                }
            }
            // M2L: d = target - source = (ix, iy) * boxsize
            {
                const int p = L.p, N = 2 * p;
                lt[l].m2l = ct.size();
                ct.resize(ct.size() + (size_t)49 * (2 * N + 1), make_double2(0.0, 0.0));
                for (int iy = -3; iy <= 3; iy++)
                    for (int ix = -3; ix <= 3; ix++) {
                        if (std::abs(ix) <= 1 && std::abs(iy) <= 1) continue;
                        shift_table(zk, ix * T.boxsize[l], iy * T.boxsize[l], N, L.rs, true,
                                    ct.data() + lt[l].m2l + (size_t)((iy + 3) * 7 + (ix + 3)) * (2 * N + 1));
                    }
                lt[l].m2l_pw = powtab(L.rs, 2 * p);
                {
                    double mx = 0.0;
                    const size_t n = (size_t)49 * (2 * N + 1);
                    for (size_t e = 0; e < n; e++) {
                        const double2 v = ct[lt[l].m2l + e];
                        mx = std::max(mx, std::max(std::fabs(v.x), std::fabs(v.y)));
                    }
                    lt[l].m2l_max = mx;
                }
                // the scaled form where rs^(2p) and the scaled entries stay
                // inside 1e-250 .. 1e250
                if (L.rs > 0.0 && 2.0 * p * std::fabs(std::log10(L.rs)) < 250.0) {
                    const size_t n = (size_t)49 * (2 * N + 1), o = ct.size();
                    ct.resize(o + n);
                    bool fine = true;
                    std::vector<double> f(N + 1);  // rs^-q
                    f[0] = 1.0;
                    for (int q = 1; q <= N; q++) f[q] = f[q - 1] / L.rs;
                    for (size_t e = 0; e < n; e++) {
                        const int q = (int)(e % (2 * N + 1)) - N;
                        const double2 v = cscal(ct[lt[l].m2l + e], f[std::abs(q)]);
                        if (!(std::fabs(v.x) <= 1e250 && std::fabs(v.y) <= 1e250)) fine = false;
                        ct[o + e] = v;
                    }
                    if (fine) {
                        lt[l].m2l_sc = o;
                        lt[l].sc_ok = true;
                    } else {
                        ct.resize(o);
                    }
                }
            }
        }
        htables_store(tkey, tabs);
    }
    const std::vector<LevTab> &lt = tabs->lt;
    const std::vector<double2> &ct = tabs->ct;
    const std::vector<double> &rt = tabs->rt;
    DevBuf<double2> d_ct(std::max<size_t>(ct.size(), 1), s);
    DevBuf<double> d_rt(std::max<size_t>(rt.size(), 1), s);
    if (!ct.empty())
        FMM_CUDA(cudaMemcpyAsync(d_ct.get(), ct.data(), ct.size() * sizeof(double2),
                                 cudaMemcpyHostToDevice, s));
    if (!rt.empty())
        FMM_CUDA(cudaMemcpyAsync(d_rt.get(), rt.data(), rt.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
    prof_mark("h_tables", s);
    const int nb = T.nboxes;
    const int ifc = P.ifcharge, ifd = P.ifdipole;
    // ---- P2M, P2L ----
    // half warps per leaf when the leaves hold about 12 sources or fewer
    // (leaves are about three quarters of the boxes)
    if ((double)P.sset.n <= 9.0 * nb)
        helm_p2m_kernel<16><<<grid_for((int64_t)nb * 16, 256), 256, 0, s>>>(
            nb, T.nchild.get(), T.level.get(), T.srcse.get(), T.centers.get(), d_lv.get(), P.src,
            P.charge, P.dipstr, P.dipvec, ifc, ifd, nd, zk, mp.get());
    else
        helm_p2m_kernel<32><<<grid_for((int64_t)nb * 32, 256), 256, 0, s>>>(
            nb, T.nchild.get(), T.level.get(), T.srcse.get(), T.centers.get(), d_lv.get(), P.src,
            P.charge, P.dipstr, P.dipvec, ifc, ifd, nd, zk, mp.get());
    FMM_CHECK_LAUNCH();
    helm_p2l_kernel<<<grid_for((int64_t)nb * 32, 256), 256, 0, s>>>(
        nb, T.level.get(), T.nlist4.get(), T.list4.get(), T.srcse.get(), T.centers.get(),
        d_lv.get(), P.src, P.charge, P.dipstr, P.dipvec, ifc, ifd, nd, zk, loc.get());
    FMM_CHECK_LAUNCH();
    prof_mark("h_p2m_p2l", s);
    // ---- M2M, upward (parents at levels nl-1 .. 2) ----
    for (int l = nl - 1; l >= 2; l--) {
        if (!hl[l].flag) continue;
        const int lo = T.lstart[l], hi = T.lend[l];
        const int64_t work = (int64_t)(hi - lo) * (2 * hl[l].p + 1) * nd;
        helm_m2m_kernel<<<grid_for(work, 256), 256, 0, s>>>(
            lo, hi, nd, T.nchild.get(), T.child.get(), T.srcse.get(), d_lv.get(), l,
            d_ct.get() + lt[l].m2m, d_rt.get() + lt[l].m2m_s, d_rt.get() + lt[l].m2m_pw,
            mp.get());
        FMM_CHECK_LAUNCH();
    }
    prof_mark("h_m2m", s);
    // ---- M2L ----
    const int sp = P.sset.pgh > 0 ? 1 : 0, tp = P.tset.pgh > 0 ? 1 : 0;
    SlotPlan spl;
    const bool tiled = helm_m2l_tiled() && plan_slots(T, sp, tp, kHTile, s, spl);
    int pmax = 0;
    for (int l = 2; l <= nl; l++) pmax = std::max(pmax, hl[l].p);
    DevBuf<double2> zero(tiled ? (size_t)(2 * pmax + 1) * nd : 0, s), mps;
    if (tiled) zero.zero(s);
    // mixed mode: levels of order <= 23 on the tensor cores (tiles of
    // 128 / nd target boxes)
    SlotPlan spl_tc;
    const bool tc = P.mixed && nd <= 128 && helm_m2l_tc_enabled() &&
                    plan_slots(T, sp, tp, 128 / nd, s, spl_tc);
    DevBuf<int> tc_err(tc ? 1 : 0, s);
    if (tc) FMM_CUDA(cudaMemsetAsync(tc_err.get(), 0, sizeof(int), s));
    bool tc_used = false;
    std::vector<char> tc_lev(nl + 1, 0);
    const bool hf_on = !(getenv("FMM2D_B200_HELM_HF") && !strcmp(getenv("FMM2D_B200_HELM_HF"), "0"));
    for (int l = 2; l <= nl; l++) {
        if (!hl[l].flag) continue;
        if (hf_on && helm_hf_level(hk::cabs_(zk) * T.boxsize[l] / (2.0 * pi), hl[l].rs)) {
            helm_m2l_hf(T, l, hl[l].p, nd, hl[l].off, d_ct.get() + lt[l].m2l, mp.get(), loc.get(),
                        sp, tp, s);
            continue;
        }
        if (tc && hl[l].p <= helm_m2l_tc_max_order()) {
            HtLevel hv;
            hv.level = l;
            hv.p = hl[l].p;
            hv.nd = nd;
            hv.lstart = hl[l].lstart;
            hv.nbox = T.lend[l] - T.lstart[l];
            hv.off = hl[l].off;
            hv.maxabs = lt[l].m2l_max;
            hv.table = d_ct.get() + lt[l].m2l;
            hv.pw = d_rt.get() + lt[l].m2l_pw;
            if (helm_m2l_tc_level(hv, spl_tc, mp.get(), loc.get(), tc_err.get(), s)) {
                tc_used = true;
                tc_lev[l] = 1;
                continue;
            }
        }
        if (tiled) {
            if (spl.ntiles == 0) continue;
            HTiles ht;
            const int g0 = 4 * (l - 2);
            for (int c = 0; c <= 4; c++) ht.tb[c] = spl.tile_base[g0 + c];
            for (int c = 0; c < 4; c++) {
                ht.start[c] = spl.start[g0 + c];
                ht.count[c] = spl.count[g0 + c];
            }
            const int ntl = ht.tb[4] - ht.tb[0];
            if (ntl == 0) continue;
            // 128 threads at most: groups of wn threads (two outputs
            // each), one tile per group
            const int wn = (hl[l].p + 1) * nd;
            const int G = wn <= 128 ? std::min(kHGroups, 128 / wn) : 1;
            const int threads = std::min(128, (G * wn + 31) / 32 * 32);
            const int nblk = (ntl + G - 1) / G;
            // levels with fewer blocks than SMs (few boxes, high
            // orders) split the 27 slots over slices of blocks
            const int nslice = nblk < kNumSM ? std::min(27, std::max(2, 2 * kNumSM / nblk)) : 1;
            const dim3 grid(std::min(nblk, kNumSM * 64), nslice);
            const int q_lo = ht.start[0], nq = ht.start[3] + ht.count[3] - q_lo;
            const int wf = (2 * hl[l].p + 1) * nd;
            DevBuf<double2> part(nslice > 1 ? (size_t)nslice * nq * wf : 0, s);
            const double *pw = d_rt.get() + lt[l].m2l_pw;
            if (lt[l].sc_ok) {
                if (!mps.get()) mps.alloc(std::max<long long>(off, 1), s);
                const long long n = (long long)(T.lend[l] - T.lstart[l]) * (2 * hl[l].p + 1) * nd;
                helm_scale_mp_kernel<<<grid_for(n, 256), 256, 0, s>>>(hl[l].off, n, hl[l].p, nd,
                                                                      pw, mp.get(), mps.get());
                FMM_CHECK_LAUNCH();
#define HM2L(SC_, SPLIT_, TAB_, MP_)                                                       \
    helm_m2l_tile_kernel<SC_, SPLIT_><<<grid, threads, 0, s>>>(                            \
        ht, spl.boxes, spl.slots, spl.dxy, nd, d_lv.get(), l, TAB_, pw, zero.get(), MP_, \
        loc.get(), part.get())
                if (nslice > 1) HM2L(true, true, d_ct.get() + lt[l].m2l_sc, mps.get());
                else HM2L(true, false, d_ct.get() + lt[l].m2l_sc, mps.get());
            } else {
                if (nslice > 1) HM2L(false, true, d_ct.get() + lt[l].m2l, mp.get());
                else HM2L(false, false, d_ct.get() + lt[l].m2l, mp.get());
#undef HM2L
            }
            FMM_CHECK_LAUNCH();
            if (nslice > 1) {
                helm_m2l_sum_kernel<<<grid_for((int64_t)nq * wf, 256), 256, 0, s>>>(
                    nq, wf, nslice, part.get(), spl.boxes, q_lo, d_lv.get(), l, nd, loc.get());
                FMM_CHECK_LAUNCH();
            }
            continue;
        }
        const int lo = T.lstart[l], hi = T.lend[l];
        const int64_t work = (int64_t)(hi - lo) * (2 * hl[l].p + 1) * nd;
        helm_m2l_kernel<<<grid_for(work, 256), 256, 0, s>>>(
            lo, hi, nd, T.nlist2.get(), T.list2.get(), T.centers.get(), T.srcse.get(),
            T.trgse.get(), sp, tp, T.boxsize[l], d_lv.get(), l, d_ct.get() + lt[l].m2l,
            d_rt.get() + lt[l].m2l_pw, mp.get(), loc.get());
        FMM_CHECK_LAUNCH();
    }
    prof_mark("h_m2l", s);
    if (profiling_enabled()) {
        // F_M2L = 8 sum_l pairs_l (2 p_l + 1)^2 nd, and the part on the tensor cores
        DevBuf<unsigned long long> cnt(nl + 1, s);
        cnt.zero(s);
        helm_count_m2l_kernel<<<kNumSM * 2, 256, 0, s>>>(nb, T.level.get(), T.nlist2.get(),
                                                         T.srcse.get(), T.trgse.get(), sp, tp,
                                                         cnt.get());
        FMM_CHECK_LAUNCH();
        std::vector<unsigned long long> h(nl + 1);
        FMM_CUDA(cudaMemcpyAsync(h.data(), cnt.get(), h.size() * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s));
        FMM_CUDA(cudaStreamSynchronize(s));
        double f = 0.0, ftc = 0.0, pairs = 0.0;
        for (int l = 2; l <= nl; l++) {
            if (!hl[l].flag) continue;
            const double w = 2.0 * hl[l].p + 1.0, fl = 8.0 * (double)h[l] * w * w * nd;
            f += fl;
            pairs += (double)h[l];
            if (tc_lev[l]) ftc += fl;
        }
        prof_set_count("h_m2l_pairs", pairs);
        prof_set_count("h_m2l_flops", f);
        prof_set_count("h_m2l_tc_flops", ftc);
        prof_set_count("nlevels", (double)nl);
        prof_set_count("nboxes", (double)nb);
        // the mark above closed the M2L phase; this sync belongs to no phase
        prof_mark("h_count", s);
    }
    if (tc_used && read_scalar(tc_err.get(), s) != 0)
        throw FmmError(4, "tensor-core Helmholtz M2L: a wait for an MMA or operand barrier timed out");
    // ---- L2L, downward (parents at levels 2 .. nl-1) ----
    for (int l = 2; l <= nl - 1; l++) {
        if (!hl[l].flag) continue;
        const int lo = T.lstart[l + 1], hi = T.lend[l + 1];
        const int64_t work = (int64_t)(hi - lo) * (2 * hl[l + 1].p + 1) * nd;
        helm_l2l_kernel<<<grid_for(work, 256), 256, 0, s>>>(
            lo, hi, nd, T.parent.get(), T.child.get(), d_lv.get(), l, d_ct.get() + lt[l].l2l,
            d_rt.get() + lt[l].l2l_s, d_rt.get() + lt[l].l2l_pw, loc.get());
        FMM_CHECK_LAUNCH();
    }
    prof_mark("h_l2l", s);
    // ---- M2P + L2P, then P2P, per point set ----
    const double thresh = hk::cabs_(zk) * T.boxsize[0] * std::ldexp(1.0, -51);
    const bool realk = zk.y == 0.0 && zk.x > 0.0;
    for (int set = 0; set < 2; set++) {
        const HPointSet &X = set == 0 ? P.sset : P.tset;
        if (X.pgh <= 0 || X.n <= 0) continue;
        DevBuf<int> leaf(X.n, s);
        helm_leaf_of_kernel<<<grid_for(nb, 256), 256, 0, s>>>(nb, T.nchild.get(), X.se, leaf.get());
        FMM_CHECK_LAUNCH();
        const unsigned g = grid_for(X.n, 128);
#define HFAR(PG)                                                                           \
    helm_far_kernel<PG><<<g, 128, 0, s>>>(X.n, X.pos, leaf.get(), T.level.get(),           \
                                          T.centers.get(), T.nlist3.get(), T.list3.get(),  \
                                          d_lv.get(), nl, mp.get(), loc.get(), nd, zk,     \
                                          X.pot, X.grad, X.hess)
        if (X.pgh == 1) HFAR(1);
        else if (X.pgh == 2) HFAR(2);
        else HFAR(3);
#undef HFAR
        FMM_CHECK_LAUNCH();
        prof_mark(set == 0 ? "h_eval_src" : "h_eval_trg", s);
        if (!P.ifnear) continue;
#define HP2P(PG, RK)                                                                        \
    helm_p2p_kernel<PG, RK><<<g, 128, 0, s>>>(X.n, X.pos, leaf.get(), T.nlist1.get(),       \
                                              T.list1.get(), T.srcse.get(), P.src, P.charge, \
                                              P.dipstr, P.dipvec, ifc, ifd, nd, zk, thresh,  \
                                              X.pot, X.grad, X.hess)
#define HP2PF(PG, RK)                                                                        \
    do {                                                                                     \
        constexpr size_t sm = kHfWarps * helm_p2p_flat_warp_bytes<PG>();                     \
        auto kern = helm_p2p_flat_kernel<PG, RK>;                                            \
        raise_smem_limit((const void *)kern, sm);                                            \
        const int gw = std::max(1, std::min((nb + kHfWarps - 1) / kHfWarps, kNumSM * 16));   \
        kern<<<gw, kHfWarps * 32, sm, s>>>(nb, T.nchild.get(), X.se, X.pos, T.nlist1.get(),   \
                                          T.list1.get(), T.srcse.get(), P.src, P.charge,      \
                                          P.dipstr, P.dipvec, ifc, ifd, zk, thresh, X.pot,    \
                                          X.grad, X.hess);                                    \
    } while (0)
        // one warp per leaf (nd = 1; FMM2D_B200_HELM_P2P=point keeps a thread per point)
        const char *pm = getenv("FMM2D_B200_HELM_P2P");
        const bool flat = nd == 1 && !(pm && !strcmp(pm, "point"));
        if (flat) {
            if (realk) {
                if (X.pgh == 1) HP2PF(1, true);
                else if (X.pgh == 2) HP2PF(2, true);
                else HP2PF(3, true);
            } else {
                if (X.pgh == 1) HP2PF(1, false);
                else if (X.pgh == 2) HP2PF(2, false);
                else HP2PF(3, false);
            }
        } else if (realk) {
            if (X.pgh == 1) HP2P(1, true);
            else if (X.pgh == 2) HP2P(2, true);
            else HP2P(3, true);
        } else {
            if (X.pgh == 1) HP2P(1, false);
            else if (X.pgh == 2) HP2P(2, false);
            else HP2P(3, false);
        }
#undef HP2P
#undef HP2PF
        FMM_CHECK_LAUNCH();
        prof_mark(set == 0 ? "h_p2p_src" : "h_p2p_trg", s);
    }
}

void helmholtz_direct(const HelmProblem &P, int ns, HPointSet X, double thresh, cudaStream_t s) {
    if (X.pgh <= 0 || X.n <= 0) return;
    const bool realk = P.zk.y == 0.0 && P.zk.x > 0.0;
    const unsigned g = grid_for(X.n, 128);
#define HD(PG, RK)                                                                             \
    helm_direct_kernel<PG, RK><<<g, 128, 0, s>>>(X.n, X.pos, ns, P.src, P.charge, P.dipstr,    \
                                                 P.dipvec, P.ifcharge, P.ifdipole, P.nd, P.zk, \
                                                 thresh, X.pot, X.grad, X.hess)
    if (realk) {
        if (X.pgh == 1) HD(1, true);
        else if (X.pgh == 2) HD(2, true);
        else HD(3, true);
    } else {
        if (X.pgh == 1) HD(1, false);
        else if (X.pgh == 2) HD(2, false);
        else HD(3, false);
    }
#undef HD
    FMM_CHECK_LAUNCH();
}

}  // namespace fmm2d
