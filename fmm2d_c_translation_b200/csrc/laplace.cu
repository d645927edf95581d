// laplace.cu -- FP64 Cauchy-kernel FMM passes (P2M, P2L, M2M, M2L, L2L,
// M2P, L2P, P2P) on the device.
//
// Mapping: one warp per box.  For the expansion operators the lanes run over
// expansion coefficients (32 per chunk, ceil((p+1)/32) chunks) and powers of
// the scaled offset come from a warp prefix product; for the evaluations
// the lanes run over the box's points and the series is summed by Horner's
// rule.  Every box's expansion and every point's output has exactly one
// writer, so no pass needs atomics.  Formulas follow
// c_translation/src/laprouts2d.c and cauchykernels2d.c term by term.
#include "laplace.cuh"

#include <algorithm>
#include <complex>
#include <mutex>
#include <stdlib.h>
#include <string.h>

namespace fmm2d {

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kBlock = kWarpsPerBlock * 32;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_global() {
    return (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
}
__device__ __forceinline__ int warp_count() { return (gridDim.x * blockDim.x) >> 5; }

__device__ __forceinline__ double2 shfl_up2(double2 v, int d) {
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, d),
                        __shfl_up_sync(0xffffffffu, v.y, d));
}

// Lane k receives z^k (lane 0: 1), by a warp prefix product.
__device__ __forceinline__ double2 warp_powers(double2 z) {
    const int lane = lane_id();
    double2 v = lane == 0 ? make_double2(1.0, 0.0) : z;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        double2 o = shfl_up2(v, d);
        if (lane >= d) v = cmul(o, v);
    }
    return v;
}

// z^n by binary powering (n >= 0).
__device__ __forceinline__ double2 zpow_int(double2 z, int n) {
    double2 r = make_double2(1.0, 0.0);
    while (n > 0) {
        if (n & 1) r = cmul(r, z);
        z = cmul(z, z);
        n >>= 1;
    }
    return r;
}

// z^(kb + lane) for the current coefficient chunk.
__device__ __forceinline__ double2 chunk_power(double2 pw, double2 z, int kb) {
    return kb == 0 ? pw : cmul(zpow_int(z, kb), pw);
}

__device__ __forceinline__ int count(const int2 *se, int b) {
    return se[b].y - se[b].x;
}

struct EvalCounts {
    const int2 *sse, *tse;
    int spgh, tpgh;
    // the reference's "npts" of a box for steps 2, 4, 5
    // (src/laplace/cfmm2d.f:837-858, 990-1010, 1040-1060)
    __device__ __forceinline__ int npts(int b) const {
        int n = 0;
        if (tpgh > 0) n += count(tse, b);
        if (spgh > 0) n += count(sse, b);
        return n;
    }
};

// ---------------------------------------------------------------------------
// Step 4, M2L over list 2 (l2dmploc, laprouts2d.c:886-994), source c1 ->
// target c2, same level (r1 = r2 = r):
//   h~_j = h_j (-r/z0)^j,  z0 = c1 - c2
//   L_0 += h~_0 log|z0| + sum_{j>=1} h~_j
//   L_i += [-h~_0/i + sum_{j>=1} C(i+j-1, j-1) h~_j] (r/z0)^i
// ---------------------------------------------------------------------------
template <int CH>
__global__ void __launch_bounds__(kBlock) m2l_kernel(
    int lo, int hi, EvalCounts ec, const int *__restrict__ nlist2,
    const int *__restrict__ list2, const double2 *__restrict__ centers,
    double r, int ndc, int c0, int p, const double *__restrict__ binom,
    const double2 *__restrict__ mp, double2 *__restrict__ loc) {
    extern __shared__ double sh_m2l[];
    // binomial block B[i][j] = C(i+j-1, j-1), 1 <= i, j <= p, row stride p+1
    double *B = sh_m2l;
    const int bstr = p + 1;
    for (int e = threadIdx.x; e < (p + 1) * (p + 1); e += blockDim.x) {
        const int i = e / bstr, j = e % bstr;
        B[e] = (i >= 1 && j >= 1) ? binom[(size_t)(i + j - 1) * (kLdc + 1) + (j - 1)] : 0.0;
    }
    __syncthreads();
    const int lane = lane_id();
    const int wib = threadIdx.x >> 5;
    double2 *ht = reinterpret_cast<double2 *>(sh_m2l + (((p + 1) * (p + 1) + 1) & ~1)) +
                  (size_t)wib * (p + 1) * CH;
    const int stride = (p + 1) * ndc;
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        const int n2 = nlist2[b];
        if (ec.npts(b) <= 0) continue;
        const double2 c2 = centers[b];
        for (int kb = 0; kb <= p; kb += 32) {
            const int i = kb + lane;
            double2 acc[CH];
#pragma unroll
            for (int q = 0; q < CH; q++) acc[q] = make_double2(0.0, 0.0);
            for (int e = 0; e < n2; e++) {
                const int sb = list2[kMaxList2 * b + e];
                if (count(ec.sse, sb) <= 0) continue;  // no multipole
                const double2 c1 = centers[sb];
                const double2 z0 = make_double2(c1.x - c2.x, c1.y - c2.y);
                const double2 zi = cinv(z0);
                const double2 w1 = cscal(zi, -r);
                const double2 w2 = cscal(zi, r);
                const double lz = 0.5 * log(z0.x * z0.x + z0.y * z0.y);
                const double2 pw1 = warp_powers(w1);
                for (int jb = 0; jb <= p; jb += 32) {
                    const int j = jb + lane;
                    const double2 wj = chunk_power(pw1, w1, jb);
                    if (j <= p)
#pragma unroll
                        for (int q = 0; q < CH; q++)
                            ht[j * CH + q] = cmul(mp[(size_t)sb * stride + (size_t)j * ndc + c0 + q], wj);
                }
                __syncwarp();
                const double2 wi = chunk_power(warp_powers(w2), w2, kb);
                if (i <= p) {
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        double2 t;
                        if (i == 0) {
                            t = cscal(ht[q], lz);
                            for (int j = 1; j <= p; j++) t = cadd(t, ht[j * CH + q]);
                        } else {
                            t = cscal(ht[q], -1.0 / i);
                            const double *brow = B + (size_t)i * bstr;
                            for (int j = 1; j <= p; j++) {
                                const double cb_ = brow[j];
                                t.x = fma(cb_, ht[j * CH + q].x, t.x);
                                t.y = fma(cb_, ht[j * CH + q].y, t.y);
                            }
                            t = cmul(t, wi);
                        }
                        acc[q] = cadd(acc[q], t);
                    }
                }
                __syncwarp();
            }
            // first writer of this box's local expansion
            if (i <= p) {
#pragma unroll
                for (int q = 0; q < CH; q++)
                    loc[(size_t)b * stride + (size_t)i * ndc + c0 + q] = acc[q];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Precision of the evaluation passes: FP64 throughout (plain), or FP32
// series and pair arithmetic with FP64 point differences and FP64 output
// accumulation (mixed).
// ---------------------------------------------------------------------------
template <bool MIXED> struct Real;
template <> struct Real<false> {
    typedef double T;
    typedef double2 T2;
    static __device__ __forceinline__ T log_(T x) { return log(x); }
    static __device__ __forceinline__ T rcp(T x) { return 1.0 / x; }
};
template <> struct Real<true> {
    typedef float T;
    typedef float2 T2;
    static __device__ __forceinline__ T log_(T x) { return __logf(x); }
    static __device__ __forceinline__ T rcp(T x) { return __fdividef(1.0f, x); }
};

template <class T2> __device__ __forceinline__ T2 mk2(double a, double b);
template <> __device__ __forceinline__ double2 mk2<double2>(double a, double b) { return make_double2(a, b); }
template <> __device__ __forceinline__ float2 mk2<float2>(double a, double b) { return make_float2((float)a, (float)b); }
template <class T2> __device__ __forceinline__ T2 cv2(double2 v) { return mk2<T2>(v.x, v.y); }
template <class T2> __device__ __forceinline__ T2 cvf(float2 v);
template <> __device__ __forceinline__ float2 cvf<float2>(float2 v) { return v; }
template <> __device__ __forceinline__ double2 cvf<double2>(float2 v) { return make_double2(v.x, v.y); }

template <class T2> __device__ __forceinline__ T2 zmul(T2 a, T2 b) {
    T2 r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <class T2> __device__ __forceinline__ void zfma(T2 &acc, T2 a, T2 b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
template <class T2, class T> __device__ __forceinline__ T2 zscal(T2 a, T s) {
    T2 r;
    r.x = a.x * s;
    r.y = a.y * s;
    return r;
}
template <class T2> __device__ __forceinline__ T2 zadd(T2 a, T2 b) {
    T2 r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}
template <class T2> __device__ __forceinline__ void add_out(double2 &o, T2 v) {
    o.x += (double)v.x;
    o.y += (double)v.y;
}

// Leaf of every point of a set, in tree order.
__global__ void leaf_of_kernel(int nb, const int *__restrict__ nchild,
                               const int2 *__restrict__ se, int *__restrict__ leaf) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        if (nchild[b] != 0) continue;
        const int2 r = se[b];
        for (int k = r.x; k < r.y; k++) leaf[k] = b;
    }
}

// ---------------------------------------------------------------------------
// Steps 6 and 7 for one point set, one thread per point: M2P over the
// leaf's list 3 (l2dmpevalp/g/h, laprouts2d.c:193-356) and L2P of the
// leaf's local expansion (l2dtaevalp/g/h, :508-664), both by Horner's rule
// with the first and second derivatives carried along as requested.
// This pass stores the outputs (it is their first writer); P2P adds.
// ---------------------------------------------------------------------------
template <int CH, int PGH, bool MIXED>
__global__ void __launch_bounds__(256) eval_far_points_kernel(
    int n, const int *__restrict__ leaf, const int *__restrict__ level,
    const double2 *__restrict__ centers, const double *__restrict__ bs,
    const int *__restrict__ nlist3, const int *__restrict__ list3,
    const int2 *__restrict__ sse, PointSet set, int ndc, int c0, int p,
    int nlevels, const double2 *__restrict__ mp,
    const double2 *__restrict__ loc, const float2 *__restrict__ mp32,
    const float2 *__restrict__ loc32) {
    typedef typename Real<MIXED>::T R;
    typedef typename Real<MIXED>::T2 R2;
    const int stride = (p + 1) * ndc;
    // coefficient m of an expansion at base offset `o`: from the FP32 copy
    // when there is one (mixed mode), else converted from FP64
    auto mcoef = [&](size_t o) -> R2 { return MIXED && mp32 ? cvf<R2>(mp32[o]) : cv2<R2>(mp[o]); };
    auto lcoef = [&](size_t o) -> R2 { return MIXED && loc32 ? cvf<R2>(loc32[o]) : cv2<R2>(loc[o]); };
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int b = leaf[k];
        const int lb = level[b];
        const double2 x = set.pos[k];
        R2 po[CH], gr[CH], he[CH];
#pragma unroll
        for (int q = 0; q < CH; q++) po[q] = gr[q] = he[q] = mk2<R2>(0.0, 0.0);
        const int n3 = (lb >= 1 && lb <= nlevels - 1) ? nlist3[b] : 0;
        // mixed mode with both channels of a pair side by side in the FP32
        // multipoles: one 16-byte load per coefficient for both Horner
        // chains, and 1/z from one FP32 reciprocal of |z|^2 (the FP64
        // divisions of the general form cost most of this pass's
        // instructions where leaves sit on two levels)
        bool pair3 = false;
        if constexpr (MIXED && CH == 2) pair3 = mp32 && (ndc & 1) == 0 && (c0 & 1) == 0;
        for (int e = 0; e < n3; e++) {
            const int jb = list3[kMaxList3 * b + e];
            if (sse[jb].y <= sse[jb].x) continue;  // no multipole
            const double2 cj = centers[jb];
            const double r = bs[level[jb]];
            const double zx = x.x - cj.x, zy = x.y - cj.y;
            if constexpr (MIXED && CH == 2) {
                if (pair3) {
                    const R fx = (R)zx, fy = (R)zy, rf = (R)r;
                    const R zzf = fx * fx + fy * fy;
                    const R izz = Real<MIXED>::rcp(zzf);
                    const R2 zi = mk2<R2>(fx * izz, -fy * izz);  // 1/z
                    const R2 w = zscal(zi, rf);                   // r/z
                    const R lz = (R)0.5 * Real<MIXED>::log_(zzf);
                    const R rinv = Real<MIXED>::rcp(rf);
                    const int s4 = ndc >> 1;
                    const float4 *M4 = reinterpret_cast<const float4 *>(mp32 + (size_t)jb * stride + c0);
                    float4 v = M4[(size_t)p * s4];
                    R2 a0[2] = {mk2<R2>(v.x, v.y), mk2<R2>(v.z, v.w)};
                    R2 a1[2] = {mk2<R2>(0.0, 0.0), mk2<R2>(0.0, 0.0)};
                    R2 a2[2] = {mk2<R2>(0.0, 0.0), mk2<R2>(0.0, 0.0)};
                    for (int m = p - 1; m >= 1; m--) {
                        v = M4[(size_t)m * s4];
                        const R2 c[2] = {mk2<R2>(v.x, v.y), mk2<R2>(v.z, v.w)};
#pragma unroll
                        for (int q = 0; q < 2; q++) {
                            if (PGH >= 3) a2[q] = zadd(zmul(a2[q], w), a1[q]);
                            if (PGH >= 2) a1[q] = zadd(zmul(a1[q], w), a0[q]);
                            a0[q] = zadd(zmul(a0[q], w), c[q]);
                        }
                    }
                    v = M4[0];
                    const R2 m0[2] = {mk2<R2>(v.x, v.y), mk2<R2>(v.z, v.w)};
#pragma unroll
                    for (int q = 0; q < 2; q++) {
                        if (PGH >= 3) a2[q] = zadd(zmul(a2[q], w), a1[q]);
                        if (PGH >= 2) a1[q] = zadd(zmul(a1[q], w), a0[q]);
                        a0[q] = zmul(a0[q], w);
                        po[q] = zadd(po[q], zadd(zscal(m0[q], lz), a0[q]));
                        if (PGH >= 2) {
                            const R2 w2 = zmul(w, w);
                            gr[q] = zadd(gr[q], zadd(zmul(m0[q], zi), zscal(zmul(a1[q], w2), -rinv)));
                            if (PGH >= 3) {
                                const R2 w3 = zmul(w2, w), w4 = zmul(w2, w2);
                                R2 h = zscal(zmul(m0[q], zmul(zi, zi)), (R)-1);
                                h = zadd(h, zscal(zmul(a2[q], w4), (R)2 * rinv * rinv));
                                h = zadd(h, zscal(zmul(a1[q], w3), (R)2 * rinv * rinv));
                                he[q] = zadd(he[q], h);
                            }
                        }
                    }
                    continue;
                }
            }
            const double zz = zx * zx + zy * zy;
            const R2 zi = mk2<R2>(zx / zz, -zy / zz);                 // 1/z
            const R2 w = mk2<R2>(r * zx / zz, -r * zy / zz);          // r/z
            const R lz = (R)0.5 * Real<MIXED>::log_((R)zz);
            const R rinv = (R)(1.0 / r);
#pragma unroll
            for (int q = 0; q < CH; q++) {
                const size_t mo = (size_t)jb * stride + c0 + q;
                R2 q0 = mcoef(mo + (size_t)p * ndc), q1 = mk2<R2>(0.0, 0.0), q2 = mk2<R2>(0.0, 0.0);
                for (int m = p - 1; m >= 1; m--) {
                    if (PGH >= 3) q2 = zadd(zmul(q2, w), q1);
                    if (PGH >= 2) q1 = zadd(zmul(q1, w), q0);
                    q0 = zadd(zmul(q0, w), mcoef(mo + (size_t)m * ndc));
                }
                if (PGH >= 3) q2 = zadd(zmul(q2, w), q1);
                if (PGH >= 2) q1 = zadd(zmul(q1, w), q0);
                q0 = zmul(q0, w);
                const R2 M0 = mcoef(mo);
                po[q] = zadd(po[q], zadd(zscal(M0, lz), q0));
                if (PGH >= 2) {
                    const R2 w2 = zmul(w, w);
                    gr[q] = zadd(gr[q], zadd(zmul(M0, zi), zscal(zmul(q1, w2), -rinv)));
                    if (PGH >= 3) {
                        const R2 w3 = zmul(w2, w), w4 = zmul(w2, w2);
                        R2 h = zscal(zmul(M0, zmul(zi, zi)), (R)-1);
                        h = zadd(h, zscal(zmul(q2, w4), (R)2 * rinv * rinv));
                        h = zadd(h, zscal(zmul(q1, w3), (R)2 * rinv * rinv));
                        he[q] = zadd(he[q], h);
                    }
                }
            }
        }
        // the two channels of a pair side by side in the FP32 locals: one
        // 16-byte load per coefficient for both Horner chains
        bool paired = false;
        if constexpr (MIXED && CH == 2) {
            if (loc32 && (ndc & 1) == 0 && (c0 & 1) == 0) {
                paired = true;
                const double2 cb = centers[b];
                const double rbi = 1.0 / bs[lb];
                const R2 z = mk2<R2>((x.x - cb.x) * rbi, (x.y - cb.y) * rbi);
                const R rinv = (R)rbi;
                const int s4 = ndc >> 1;
                const float4 *L4 = reinterpret_cast<const float4 *>(loc32 + (size_t)b * stride + c0);
                float4 v = L4[(size_t)p * s4];
                R2 a0[2] = {mk2<R2>(v.x, v.y), mk2<R2>(v.z, v.w)};
                R2 a1[2] = {mk2<R2>(0.0, 0.0), mk2<R2>(0.0, 0.0)};
                R2 a2[2] = {mk2<R2>(0.0, 0.0), mk2<R2>(0.0, 0.0)};
                for (int m = p - 1; m >= 0; m--) {
                    v = L4[(size_t)m * s4];
                    const R2 c[2] = {mk2<R2>(v.x, v.y), mk2<R2>(v.z, v.w)};
#pragma unroll
                    for (int q = 0; q < 2; q++) {
                        if (PGH >= 3) a2[q] = zadd(zmul(a2[q], z), a1[q]);
                        if (PGH >= 2) a1[q] = zadd(zmul(a1[q], z), a0[q]);
                        a0[q] = zadd(zmul(a0[q], z), c[q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    po[q] = zadd(po[q], a0[q]);
                    if (PGH >= 2) gr[q] = zadd(gr[q], zscal(a1[q], rinv));
                    if (PGH >= 3) he[q] = zadd(he[q], zscal(a2[q], (R)2 * rinv * rinv));
                }
            }
        }
        if (!paired) {
            const double2 cb = centers[b];
            const double rb = bs[lb];
            const R2 z = mk2<R2>((x.x - cb.x) / rb, (x.y - cb.y) / rb);
            const R rinv = (R)(1.0 / rb);
#pragma unroll
            for (int q = 0; q < CH; q++) {
                const size_t lo_ = (size_t)b * stride + c0 + q;
                R2 q0 = lcoef(lo_ + (size_t)p * ndc), q1 = mk2<R2>(0.0, 0.0), q2 = mk2<R2>(0.0, 0.0);
                for (int m = p - 1; m >= 0; m--) {
                    if (PGH >= 3) q2 = zadd(zmul(q2, z), q1);
                    if (PGH >= 2) q1 = zadd(zmul(q1, z), q0);
                    q0 = zadd(zmul(q0, z), lcoef(lo_ + (size_t)m * ndc));
                }
                po[q] = zadd(po[q], q0);
                if (PGH >= 2) gr[q] = zadd(gr[q], zscal(q1, rinv));
                if (PGH >= 3) he[q] = zadd(he[q], zscal(q2, (R)2 * rinv * rinv));
            }
        }
#pragma unroll
        for (int q = 0; q < CH; q++) {
            const size_t o = (size_t)k * ndc + c0 + q;
            set.pot[o] = make_double2((double)po[q].x, (double)po[q].y);
            if (PGH >= 2) set.grad[o] = make_double2((double)gr[q].x, (double)gr[q].y);
            if (PGH >= 3) set.hess[o] = make_double2((double)he[q].x, (double)he[q].y);
        }
    }
}

// ---------------------------------------------------------------------------
// Step 8, P2P over list 1 (c2d_direct*, cauchykernels2d.c:31-442):
//   pot += q log|z| + d/z,  grad += q/z - d/z^2,  hess += -q/z^2 + 2d/z^3,
// z = t - s; pairs with |z|^2 <= thresh^2 (pot only) or < thresh^2 skipped.
// A warp takes up to 32 targets of one box; when the box has fewer, lane
// groups split the sources and are summed at the end.  Point differences
// are formed in FP64 in both precisions.
// ---------------------------------------------------------------------------
// One warp per box takes the box's targets of both point sets (targets
// first, then sources as targets).  The sources of all list-1 boxes are
// staged once into shared memory (FP64 positions, strengths in the pass's
// precision), in chunks of kP2PStage; the targets are split into chunks of
// T <= 32 chosen to keep as many lanes busy as possible, each chunk's
// lanes forming G = 32 / T groups that split the staged sources and are
// summed at the end.  Point differences are formed in FP64 in both
// precisions.
// (compile-time sizes; -DFMM2D_P2P_STAGE / -DFMM2D_P2P_WARPS override them
// for measurements of other shapes)
// (64 staged sources and 8 warps per block: measured on a B200, 10^7 +
// 10^7 uniform points, mixed mode, the near field took 4.64 ms against
// 5.53 ms with 128 sources and 4 warps -- less shared memory per warp,
// more warps resident)
#ifndef FMM2D_P2P_STAGE
#define FMM2D_P2P_STAGE 64
#endif
#ifndef FMM2D_P2P_WARPS
#define FMM2D_P2P_WARPS 8
#endif
constexpr int kP2PStage = FMM2D_P2P_STAGE;
constexpr int kP2PWarps = FMM2D_P2P_WARPS;

// Point positions as the near field reads them: FP64 (x, y), or for the
// mixed pass a float4 (x_hi, x_lo, y_hi, y_lo) with x = x_hi + x_lo, whose
// FP32 difference (x_hi - x'_hi) + (x_lo - x'_lo) carries the FP64
// difference to FP32 accuracy without FP64 instructions.
template <bool MIXED> struct PosT { typedef double2 T; };
template <> struct PosT<true> { typedef float4 T; };


__device__ __forceinline__ void pos_diff(double2 a, double2 b, double &dx, double &dy) {
    dx = a.x - b.x;
    dy = a.y - b.y;
}
__device__ __forceinline__ void pos_diff(float4 a, float4 b, float &dx, float &dy) {
    dx = (a.x - b.x) + (a.y - b.y);
    dy = (a.z - b.z) + (a.w - b.w);
}

__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float half_ln_fast(float x) {  // 0.5 * ln(x)
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r * 0.34657359027997264f;  // ln(2) / 2
}
__device__ __forceinline__ double rcp_pair(double x) { return 1.0 / x; }
__device__ __forceinline__ float rcp_pair(float x) { return rcp_fast(x); }
__device__ __forceinline__ double half_ln_pair(double x) { return 0.5 * log(x); }
__device__ __forceinline__ float half_ln_pair(float x) { return half_ln_fast(x); }

// Steps 6 and 7 with one warp per leaf: the warp evaluates the leaf's
// list-3 multipoles and local expansion at all of the leaf's points and
// stores them (the near field adds to them afterwards).  The expansion
// coefficients are staged once per box in shared memory, in the pass's
// precision, instead of being loaded (and converted) by every point.  Same
// arithmetic, in the same order, as eval_far_points_kernel.
// Whether steps 6-7 run with one warp per leaf (coefficients staged once per
// box) or one thread per point.  Measured on a B200 (10^7 + 10^7 uniform
// points): per leaf is faster in FP64 at p = 37 (3.9 against 4.1 ms), per
// point in the mixed mode at p = 18 (2.0 against 2.4 ms), where a leaf's
// ~19 points leave a third of the warp idle.  FMM2D_B200_FAR=leaf / point
// overrides.
bool far_per_leaf(const CauchyProblem &P) {
    const char *m = getenv("FMM2D_B200_FAR");
    if (m && !strcmp(m, "leaf")) return true;
    if (m && !strcmp(m, "point")) return false;
    return !P.mixed;
}

constexpr int kFarWarps = 4;

struct FarArgs {
    int p = 0, nlevels = 0;
    const int *level = nullptr;
    const double2 *centers = nullptr;
    const double *bs = nullptr;
    const int *nlist3 = nullptr, *list3 = nullptr;
    const double2 *mp = nullptr, *loc = nullptr;
};

template <int CH, int PGH, bool MIXED>
__device__ __forceinline__ void far_field_box(int b, int ntb, int2 tr, int2 sr0, int ntot,
                                              const FarArgs &fa, const int2 *__restrict__ sse,
                                              const PointSet &sset, const PointSet &tset,
                                              int ndc, int c0, typename Real<MIXED>::T2 *sm) {
    typedef typename Real<MIXED>::T R;
    typedef typename Real<MIXED>::T2 R2;
    const int lane = lane_id();
    const int p = fa.p, stride = (p + 1) * ndc, nc = (p + 1) * CH;
    R2 *s_loc = sm, *s_mp = sm + nc;
    for (int i = lane; i < nc; i += 32) {
        const int m = i / CH, q = i - m * CH;
        s_loc[i] = cv2<R2>(fa.loc[(size_t)b * stride + (size_t)m * ndc + c0 + q]);
    }
    const int lb = fa.level[b];
    const int n3 = (lb >= 1 && lb <= fa.nlevels - 1) ? fa.nlist3[b] : 0;
    const double2 cb = fa.centers[b];
    const double rb = fa.bs[lb];
    for (int t0 = 0; t0 < ntot; t0 += 32) {
        const int t = t0 + lane;
        const bool act = t < ntot, is_t = t < ntb;
        const int k = is_t ? tr.x + t : sr0.x + t - ntb;
        const double2 x = act ? (is_t ? tset.pos : sset.pos)[k] : cb;
        R2 po[CH], gr[CH], he[CH];
#pragma unroll
        for (int q = 0; q < CH; q++) po[q] = gr[q] = he[q] = mk2<R2>(0.0, 0.0);
        for (int e = 0; e < n3; e++) {
            const int jb = fa.list3[kMaxList3 * b + e];
            if (sse[jb].y <= sse[jb].x) continue;  // no multipole
            __syncwarp();
            for (int i = lane; i < nc; i += 32) {
                const int m = i / CH, q = i - m * CH;
                s_mp[i] = cv2<R2>(fa.mp[(size_t)jb * stride + (size_t)m * ndc + c0 + q]);
            }
            __syncwarp();
            if (!act) continue;
            const double2 cj = fa.centers[jb];
            const double r = fa.bs[fa.level[jb]];
            const double zx = x.x - cj.x, zy = x.y - cj.y;
            const double zz = zx * zx + zy * zy;
            const R2 zi = mk2<R2>(zx / zz, -zy / zz);         // 1/z
            const R2 w = mk2<R2>(r * zx / zz, -r * zy / zz);  // r/z
            const R lz = (R)0.5 * Real<MIXED>::log_((R)zz);
            const R rinv = (R)(1.0 / r);
#pragma unroll
            for (int q = 0; q < CH; q++) {
                R2 q0 = s_mp[p * CH + q], q1 = mk2<R2>(0.0, 0.0), q2 = mk2<R2>(0.0, 0.0);
                for (int m = p - 1; m >= 1; m--) {
                    if (PGH >= 3) q2 = zadd(zmul(q2, w), q1);
                    if (PGH >= 2) q1 = zadd(zmul(q1, w), q0);
                    q0 = zadd(zmul(q0, w), s_mp[m * CH + q]);
                }
                if (PGH >= 3) q2 = zadd(zmul(q2, w), q1);
                if (PGH >= 2) q1 = zadd(zmul(q1, w), q0);
                q0 = zmul(q0, w);
                const R2 M0 = s_mp[q];
                po[q] = zadd(po[q], zadd(zscal(M0, lz), q0));
                if (PGH >= 2) {
                    const R2 w2 = zmul(w, w);
                    gr[q] = zadd(gr[q], zadd(zmul(M0, zi), zscal(zmul(q1, w2), -rinv)));
                    if (PGH >= 3) {
                        const R2 w3 = zmul(w2, w), w4 = zmul(w2, w2);
                        R2 h = zscal(zmul(M0, zmul(zi, zi)), (R)-1);
                        h = zadd(h, zscal(zmul(q2, w4), (R)2 * rinv * rinv));
                        h = zadd(h, zscal(zmul(q1, w3), (R)2 * rinv * rinv));
                        he[q] = zadd(he[q], h);
                    }
                }
            }
        }
        __syncwarp();
        if (!act) continue;
        {
            const R2 z = mk2<R2>((x.x - cb.x) / rb, (x.y - cb.y) / rb);
            const R rinv = (R)(1.0 / rb);
#pragma unroll
            for (int q = 0; q < CH; q++) {
                R2 q0 = s_loc[p * CH + q], q1 = mk2<R2>(0.0, 0.0), q2 = mk2<R2>(0.0, 0.0);
                for (int m = p - 1; m >= 0; m--) {
                    if (PGH >= 3) q2 = zadd(zmul(q2, z), q1);
                    if (PGH >= 2) q1 = zadd(zmul(q1, z), q0);
                    q0 = zadd(zmul(q0, z), s_loc[m * CH + q]);
                }
                po[q] = zadd(po[q], q0);
                if (PGH >= 2) gr[q] = zadd(gr[q], zscal(q1, rinv));
                if (PGH >= 3) he[q] = zadd(he[q], zscal(q2, (R)2 * rinv * rinv));
            }
        }
        const int pg = is_t ? tset.pgh : sset.pgh;
        double2 *opot = is_t ? tset.pot : sset.pot;
        double2 *ograd = is_t ? tset.grad : sset.grad;
        double2 *ohess = is_t ? tset.hess : sset.hess;
#pragma unroll
        for (int q = 0; q < CH; q++) {
            const size_t o = (size_t)k * ndc + c0 + q;
            opot[o] = make_double2((double)po[q].x, (double)po[q].y);
            if (PGH >= 2 && pg >= 2) ograd[o] = make_double2((double)gr[q].x, (double)gr[q].y);
            if (PGH >= 3 && pg >= 3) ohess[o] = make_double2((double)he[q].x, (double)he[q].y);
        }
    }
    __syncwarp();
}

// One warp per leaf with points of a set that wants outputs.
template <int CH, int PGH, bool MIXED>
__global__ void __launch_bounds__(kFarWarps * 32) far_leaf_kernel(
    int nb, const int *__restrict__ nchild, FarArgs fa, const int2 *__restrict__ sse,
    PointSet sset, PointSet tset, int ndc, int c0) {
    typedef typename Real<MIXED>::T2 R2;
    __shared__ R2 stage[kFarWarps][2 * (kLdc / 2 + 1) * CH];
    R2 *sm = stage[threadIdx.x >> 5];
    for (int b = warp_global(); b < nb; b += warp_count()) {
        if (nchild[b] != 0) continue;
        const int2 tr = tset.pgh > 0 ? tset.se[b] : make_int2(0, 0);
        const int2 sr0 = sset.pgh > 0 ? sset.se[b] : make_int2(0, 0);
        const int ntb = tr.y - tr.x, ntot = ntb + sr0.y - sr0.x;
        if (ntot == 0) continue;
        far_field_box<CH, PGH, MIXED>(b, ntb, tr, sr0, ntot, fa, sse, sset, tset, ndc, c0, sm);
    }
}

// LAPR: the two channels of a complex-Laplace density carry real charges
// and only the real part of each channel's potential is used
// (lfmm2d.f:141-157, 168-225), so the charge terms drop their imaginary
// halves and the potential keeps its real part only.  The results used are
// the same to the bit.
// One source's contribution to one target of the near field: pot += q
// log|z| + d/z, grad += q/z - d/z^2, hess += -q/z^2 + 2d/z^3 (z = t - s),
// with `st` the source's strengths (charges of the CH channels, then
// dipoles).  Pairs inside the threshold contribute exactly zero.
template <int CH, int PGH, bool IFC, bool IFD, bool MIXED, bool LAPR>
__device__ __forceinline__ void p2p_pair(const typename PosT<MIXED>::T &x,
                                         const typename PosT<MIXED>::T &sp,
                                         const typename Real<MIXED>::T2 *st,
                                         typename Real<MIXED>::T th2,
                                         typename Real<MIXED>::T2 *po,
                                         typename Real<MIXED>::T2 *gr,
                                         typename Real<MIXED>::T2 *he) {
    typedef typename Real<MIXED>::T R;
    typedef typename Real<MIXED>::T2 R2;
    R dx, dy;
    pos_diff(x, sp, dx, dy);
    const R rr = dx * dx + dy * dy;
    // skipped pairs contribute exactly zero, without a branch
    const bool skip = PGH == 1 ? (rr <= th2) : (rr < th2);
    const R rrs = skip ? (R)1 : rr;
    const R ri = skip ? (R)0 : rcp_pair(rrs);
    R2 zi;
    zi.x = dx * ri;
    zi.y = -dy * ri;
    R2 zi2 = mk2<R2>(0.0, 0.0), zi3 = mk2<R2>(0.0, 0.0);
    if (PGH >= 2 || IFD) zi2 = zmul(zi, zi);
    if (PGH >= 3 && IFD) zi3 = zmul(zi2, zi);
    R rl = 0;
    if (IFC) rl = skip ? (R)0 : half_ln_pair(rrs);
#pragma unroll
    for (int q = 0; q < CH; q++) {
        if (IFC) {
            const R2 qv = st[q];
            if (LAPR) {
                po[q].x = fma(rl, qv.x, po[q].x);
                if (PGH >= 2) {
                    gr[q].x = fma(zi.x, qv.x, gr[q].x);
                    gr[q].y = fma(zi.y, qv.x, gr[q].y);
                }
                if (PGH >= 3) {
                    he[q].x = fma(-zi2.x, qv.x, he[q].x);
                    he[q].y = fma(-zi2.y, qv.x, he[q].y);
                }
            } else {
                po[q].x = fma(rl, qv.x, po[q].x);
                po[q].y = fma(rl, qv.y, po[q].y);
                if (PGH >= 2) zfma(gr[q], zi, qv);
                if (PGH >= 3) zfma(he[q], zscal(zi2, (R)-1), qv);
            }
        }
        if (IFD) {
            const R2 dv = st[(IFC ? CH : 0) + q];
            if (LAPR) {
                po[q].x = fma(zi.x, dv.x, fma(-zi.y, dv.y, po[q].x));
            } else {
                zfma(po[q], zi, dv);
            }
            if (PGH >= 2) zfma(gr[q], zscal(zi2, (R)-1), dv);
            if (PGH >= 3) zfma(he[q], zscal(zi3, (R)2), dv);
        }
    }
}

// Strength slots per warp of p2p_kernel: the staged strengths, or the
// 32 lanes' group sums (3 CH values each) when those are more.
template <int CH, bool IFC, bool IFD>
constexpr int p2p_str_slots() {
    return kP2PStage * ((IFC ? CH : 0) + (IFD ? CH : 0)) > 32 * 3 * CH
               ? kP2PStage * ((IFC ? CH : 0) + (IFD ? CH : 0))
               : 32 * 3 * CH;
}

template <int CH, int PGH, bool IFC, bool IFD, bool MIXED, bool LAPR>
__global__ void __launch_bounds__(kP2PWarps * 32) p2p_kernel(
    int lo, int hi, const int *__restrict__ nlist1,
    const int *__restrict__ list1, const int *__restrict__ nchild,
    int leaves, const int2 *__restrict__ sse,
    const typename PosT<MIXED>::T *__restrict__ src,
    const typename Real<MIXED>::T2 *__restrict__ chg,
    const typename Real<MIXED>::T2 *__restrict__ dip, PointSet sset,
    PointSet tset, const typename PosT<MIXED>::T *__restrict__ spos,
    const typename PosT<MIXED>::T *__restrict__ tpos, int ndc, int c0,
    double th2d) {
    typedef typename Real<MIXED>::T R;
    typedef typename Real<MIXED>::T2 R2;
    typedef typename PosT<MIXED>::T PT;
    constexpr int kStr = (IFC ? CH : 0) + (IFD ? CH : 0);
    constexpr int kRed = 3 * CH;
    // the strengths' slots double as the 32 lanes' group sums (kRed values
    // each), so they hold the larger of the two
    constexpr int kStrSlots = p2p_str_slots<CH, IFC, IFD>();
    constexpr int kWarpBytes = kP2PStage * 16 + kStrSlots * (int)sizeof(R2);
    extern __shared__ __align__(16) unsigned char p2p_smem[];
    const int lane = lane_id(), wib = threadIdx.x >> 5;
    PT *s_pos = reinterpret_cast<PT *>(p2p_smem + (size_t)wib * kWarpBytes);
    R2 *s_str = reinterpret_cast<R2 *>(s_pos + kP2PStage);
    R2 *red = s_str;  // reused for the group sums
    // (the FP32 threshold is kept above zero so that coincident points are
    // skipped even when thresh^2 underflows)
    const R th2 = MIXED ? (R)fmax(th2d, 1.1754943508222875e-38) : (R)th2d;
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        const int n1 = nlist1[b];
        if (n1 == 0) continue;
        if ((nchild[b] == 0) != (leaves != 0)) continue;
        const int2 tr = tset.pgh > 0 ? tset.se[b] : make_int2(0, 0);
        const int2 sr0 = sset.pgh > 0 ? sset.se[b] : make_int2(0, 0);
        const int ntb = tr.y - tr.x, nsb = sr0.y - sr0.x, ntot = ntb + nsb;
        if (ntot == 0) continue;
        // list-1 source ranges and their running offsets
        int jstart = 0, jcount = 0;  // lane e < n1 holds entry e
        if (lane < n1) {
            const int2 r = sse[list1[kMaxList1 * b + lane]];
            jstart = r.x;
            jcount = r.y - r.x;
        }
        int jofs = jcount;  // inclusive prefix over entries
#pragma unroll
        for (int d = 1; d < 16; d <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, jofs, d);
            if (lane >= d) jofs += o;
        }
        const int nsrc = __shfl_sync(0xffffffffu, jofs, n1 - 1);
        jofs -= jcount;  // exclusive
        if (nsrc == 0) continue;
        // target chunking: c chunks of T = ceil(ntot / c) minimising the
        // lane sweeps c * ceil(min(nsrc, stage) / (32 / T))
        int best_c = (ntot + 31) / 32, best_cost = 1 << 30;
        const int ns_eff = min(nsrc, kP2PStage);
        for (int c = (ntot + 31) / 32; c <= (ntot + 31) / 32 + 3 && c <= ntot; c++) {
            const int Tc = (ntot + c - 1) / c;
            const int cost = c * ((ns_eff + 32 / Tc - 1) / (32 / Tc));
            if (cost < best_cost) {
                best_cost = cost;
                best_c = c;
            }
        }
        const int Tch = (ntot + best_c - 1) / best_c;
        for (int t0 = 0; t0 < ntot; t0 += Tch) {
            const int T = min(Tch, ntot - t0);
            const int G = 32 / T;
            const int g = lane / T, tl = lane - g * T;
            const bool act = g < G;
            const int it = t0 + tl;
            const bool is_t = it < ntb;
            PT x;
            if (act)
                x = is_t ? tpos[tr.x + it] : spos[sr0.x + it - ntb];
            else
                x = spos[sr0.x];  // any valid point; results discarded
            R2 po[CH], gr[CH], he[CH];
#pragma unroll
            for (int q = 0; q < CH; q++) po[q] = gr[q] = he[q] = mk2<R2>(0.0, 0.0);
            for (int s0 = 0; s0 < nsrc; s0 += kP2PStage) {
                const int nst = min(kP2PStage, nsrc - s0);
                __syncwarp();
                for (int i0 = 0; i0 < nst; i0 += 32) {  // warp-uniform trip count
                    // source i of the concatenated list-1 ranges
                    const int i = i0 + lane;
                    const int gi = s0 + i;
                    int e = 0;
                    for (int u = 1; u < n1; u++)
                        if (__shfl_sync(0xffffffffu, jofs, u) <= gi) e = u;
                    const int k = __shfl_sync(0xffffffffu, jstart, e) + gi -
                                  __shfl_sync(0xffffffffu, jofs, e);
                    if (i >= nst) continue;
                    s_pos[i] = src[k];
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        if (IFC) s_str[i * kStr + q] = chg[(size_t)k * ndc + c0 + q];
                        if (IFD) s_str[i * kStr + (IFC ? CH : 0) + q] = dip[(size_t)k * ndc + c0 + q];
                    }
                }
                __syncwarp();
                if (act) {
#pragma unroll 4
                    for (int kk = g; kk < nst; kk += G)
                        p2p_pair<CH, PGH, IFC, IFD, MIXED, LAPR>(x, s_pos[kk], s_str + kk * kStr,
                                                                 th2, po, gr, he);
                }
            }
            // sum the lane groups
            if (G > 1) {
                __syncwarp();
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    red[lane * kRed + q] = po[q];
                    if (PGH >= 2) red[lane * kRed + CH + q] = gr[q];
                    if (PGH >= 3) red[lane * kRed + 2 * CH + q] = he[q];
                }
                __syncwarp();
                if (act && g == 0) {
                    for (int gg = 1; gg < G; gg++) {
                        const int ol = gg * T + tl;
#pragma unroll
                        for (int q = 0; q < CH; q++) {
                            po[q] = zadd(po[q], red[ol * kRed + q]);
                            if (PGH >= 2) gr[q] = zadd(gr[q], red[ol * kRed + CH + q]);
                            if (PGH >= 3) he[q] = zadd(he[q], red[ol * kRed + 2 * CH + q]);
                        }
                    }
                }
            }
            if (act && g == 0) {
                const PointSet &S = is_t ? tset : sset;
                const int t = is_t ? tr.x + it : sr0.x + it - ntb;
                const int pg = S.pgh;
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    const size_t o = (size_t)t * ndc + c0 + q;
                    add_out(S.pot[o], po[q]);
                    if (PGH >= 2 && pg >= 2) add_out(S.grad[o], gr[q]);
                    if (PGH >= 3 && pg >= 3) add_out(S.hess[o], he[q]);
                }
            }
        }
    }
}

// Near field with the (target, source block) work flattened over the lanes.
// A warp takes up to 32 targets of a box at a time; the staged sources are
// cut into B blocks and the T * B (target, block) items are dealt to the
// lanes round by round, each item summing its block into registers and
// leaving the partial sums in shared memory, from where the target's lane
// adds the B partials in block order.  B is chosen per box to minimise the
// lane sweeps, so that a box of 19 targets keeps 30 of 32 lanes busy instead
// of 19.  Deterministic: every sum has a fixed order.
template <bool MIXED> struct FlatItems { static constexpr int value = MIXED ? 96 : 64; };

template <int CH, int PGH>
constexpr int flat_outputs() { return CH * (1 + (PGH >= 2 ? 1 : 0) + (PGH >= 3 ? 1 : 0)); }

template <int CH, int PGH, bool IFC, bool IFD, bool MIXED>
constexpr size_t p2p_flat_warp_bytes() {
    return (size_t)kP2PStage * (16 + ((IFC ? CH : 0) + (IFD ? CH : 0)) * sizeof(typename Real<MIXED>::T2)) +
           32 * 16 + (size_t)FlatItems<MIXED>::value * flat_outputs<CH, PGH>() *
                          sizeof(typename Real<MIXED>::T2);
}

template <int CH, int PGH, bool IFC, bool IFD, bool MIXED, bool LAPR>
__global__ void __launch_bounds__(kP2PWarps * 32) p2p_flat_kernel(
    int lo, int hi, const int *__restrict__ nlist1,
    const int *__restrict__ list1, const int *__restrict__ nchild,
    int leaves, const int2 *__restrict__ sse,
    const typename PosT<MIXED>::T *__restrict__ src,
    const typename Real<MIXED>::T2 *__restrict__ chg,
    const typename Real<MIXED>::T2 *__restrict__ dip, PointSet sset,
    PointSet tset, const typename PosT<MIXED>::T *__restrict__ spos,
    const typename PosT<MIXED>::T *__restrict__ tpos, int ndc, int c0,
    double th2d) {
    typedef typename Real<MIXED>::T R;
    typedef typename Real<MIXED>::T2 R2;
    typedef typename PosT<MIXED>::T PT;
    constexpr int kStr = (IFC ? CH : 0) + (IFD ? CH : 0);
    constexpr int kNo = flat_outputs<CH, PGH>();
    constexpr int kItems = FlatItems<MIXED>::value;
    constexpr size_t kWarpBytes = p2p_flat_warp_bytes<CH, PGH, IFC, IFD, MIXED>();
    extern __shared__ __align__(16) unsigned char p2p_smem[];
    const int lane = lane_id(), wib = threadIdx.x >> 5;
    PT *s_pos = reinterpret_cast<PT *>(p2p_smem + (size_t)wib * kWarpBytes);
    R2 *s_str = reinterpret_cast<R2 *>(s_pos + kP2PStage);
    PT *s_tgt = reinterpret_cast<PT *>(s_str + kP2PStage * kStr);
    R2 *part = reinterpret_cast<R2 *>(s_tgt + 32);
    const R th2 = MIXED ? (R)fmax(th2d, 1.1754943508222875e-38) : (R)th2d;
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        const int n1 = nlist1[b];
        if (n1 == 0) continue;
        if ((nchild[b] == 0) != (leaves != 0)) continue;
        const int2 tr = tset.pgh > 0 ? tset.se[b] : make_int2(0, 0);
        const int2 sr0 = sset.pgh > 0 ? sset.se[b] : make_int2(0, 0);
        const int ntb = tr.y - tr.x, nsb = sr0.y - sr0.x, ntot = ntb + nsb;
        if (ntot == 0) continue;
        int jstart = 0, jcount = 0;  // lane e < n1 holds list-1 entry e
        if (lane < n1) {
            const int2 r = sse[list1[kMaxList1 * b + lane]];
            jstart = r.x;
            jcount = r.y - r.x;
        }
        int jofs = jcount;
#pragma unroll
        for (int d = 1; d < 16; d <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, jofs, d);
            if (lane >= d) jofs += o;
        }
        const int nsrc = __shfl_sync(0xffffffffu, jofs, n1 - 1);
        jofs -= jcount;
        if (nsrc == 0) continue;
        // the targets and the sources as targets in chunks of at most 32
        // points (a chunk may hold both: measured on a B200, chunking each
        // set on its own made the near field of 10^7 + 10^7 points 45 %
        // slower, with more and smaller chunks per leaf)
        const int nchunk = (ntot + 31) / 32, T0 = (ntot + nchunk - 1) / nchunk;
        const int ns_eff = min(nsrc, kP2PStage);
        for (int t0 = 0; t0 < ntot; t0 += T0) {
            const int T = min(T0, ntot - t0);
            __syncwarp();
            if (lane < T) {
                const int it = t0 + lane;
                s_tgt[lane] = it < ntb ? tpos[tr.x + it] : spos[sr0.x + it - ntb];
            }
            int B = 1, best = 1 << 30;
            for (int bb = 1; bb * T <= kItems; bb++) {
                const int cost = ((T * bb + 31) >> 5) * ((ns_eff + bb - 1) / bb);
                if (cost < best) {
                    best = cost;
                    B = bb;
                }
            }
            const int nit = T * B;
            R2 po[CH], gr[CH], he[CH];
#pragma unroll
            for (int q = 0; q < CH; q++) po[q] = gr[q] = he[q] = mk2<R2>(0.0, 0.0);
            for (int s0 = 0; s0 < nsrc; s0 += kP2PStage) {
                const int nst = min(kP2PStage, nsrc - s0);
                __syncwarp();
                for (int i0 = 0; i0 < nst; i0 += 32) {  // warp-uniform trip count
                    const int i = i0 + lane;
                    const int gi = s0 + i;
                    int e = 0;
                    for (int u = 1; u < n1; u++)
                        if (__shfl_sync(0xffffffffu, jofs, u) <= gi) e = u;
                    const int k = __shfl_sync(0xffffffffu, jstart, e) + gi -
                                  __shfl_sync(0xffffffffu, jofs, e);
                    if (i >= nst) continue;
                    s_pos[i] = src[k];
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        if (IFC) s_str[i * kStr + q] = chg[(size_t)k * ndc + c0 + q];
                        if (IFD) s_str[i * kStr + (IFC ? CH : 0) + q] = dip[(size_t)k * ndc + c0 + q];
                    }
                }
                __syncwarp();
                const int sb = (nst + B - 1) / B;
                for (int i = lane; i < nit; i += 32) {
                    const int t = i % T, blk = i / T;
                    const PT x = s_tgt[t];
                    R2 apo[CH], agr[CH], ahe[CH];
#pragma unroll
                    for (int q = 0; q < CH; q++) apo[q] = agr[q] = ahe[q] = mk2<R2>(0.0, 0.0);
                    const int j0 = blk * sb, j1 = min(nst, j0 + sb);
#pragma unroll 4
                    for (int kk = j0; kk < j1; kk++)
                        p2p_pair<CH, PGH, IFC, IFD, MIXED, LAPR>(x, s_pos[kk], s_str + kk * kStr,
                                                                 th2, apo, agr, ahe);
                    R2 *pp = part + (size_t)i * kNo;
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        pp[q] = apo[q];
                        if (PGH >= 2) pp[CH + q] = agr[q];
                        if (PGH >= 3) pp[2 * CH + q] = ahe[q];
                    }
                }
                __syncwarp();
                if (lane < T) {
                    for (int blk = 0; blk < B; blk++) {
                        const R2 *pp = part + (size_t)(lane + blk * T) * kNo;
#pragma unroll
                        for (int q = 0; q < CH; q++) {
                            po[q] = zadd(po[q], pp[q]);
                            if (PGH >= 2) gr[q] = zadd(gr[q], pp[CH + q]);
                            if (PGH >= 3) he[q] = zadd(he[q], pp[2 * CH + q]);
                        }
                    }
                }
            }
            if (lane < T) {
                const int it = t0 + lane;
                const bool is_t = it < ntb;
                const int t = is_t ? tr.x + it : sr0.x + it - ntb;
                const int pg = is_t ? tset.pgh : sset.pgh;
                double2 *opot = is_t ? tset.pot : sset.pot;
                double2 *ograd = is_t ? tset.grad : sset.grad;
                double2 *ohess = is_t ? tset.hess : sset.hess;
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    const size_t o = (size_t)t * ndc + c0 + q;
                    add_out(opot[o], po[q]);
                    if (PGH >= 2 && pg >= 2) add_out(ograd[o], gr[q]);
                    if (PGH >= 3 && pg >= 3) add_out(ohess[o], he[q]);
                }
            }
        }
    }
}

template <int CH, bool IFC, bool IFD, bool MIXED>
constexpr size_t p2p_smem_bytes() {
    return (size_t)kP2PWarps * ((size_t)kP2PStage * 16 +
                                (size_t)p2p_str_slots<CH, IFC, IFD>() * sizeof(typename Real<MIXED>::T2));
}

int grid_for(int nwarps) {
    int blocks = (nwarps + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks > kNumSM * 16) blocks = kNumSM * 16;
    return blocks < 1 ? 1 : blocks;
}

template <int CH, int PGH, bool MIXED, bool LAPR>
void launch_p2p_t(const Tree &T, const CauchyProblem &P, int c0, double th2,
                  int lo, int hi, int leaves, cudaStream_t s) {
    typedef typename Real<MIXED>::T2 R2;
    const int g = std::max(1, std::min((hi - lo + kP2PWarps - 1) / kP2PWarps, kNumSM * 16));
    const int *n1 = T.nlist1.get(), *l1 = T.list1.get(), *nc = T.nchild.get();
    const int2 *sse = T.srcse.get();
    typedef typename PosT<MIXED>::T PT;
    const R2 *chg = MIXED ? (const R2 *)P.charge32 : (const R2 *)P.charge;
    const R2 *dip = MIXED ? (const R2 *)P.dipstr32 : (const R2 *)P.dipstr;
    const PT *spos = MIXED ? (const PT *)P.src_hl : (const PT *)P.src;
    const PT *tpos = MIXED ? (const PT *)P.trg_hl : (const PT *)P.tset.pos;
    // Flattened items in the mixed mode, equal lane groups in FP64: measured
    // on a B200 (10^7 + 10^7 uniform points, lfmm2d_st_cd_g) 5.56 against
    // 5.75 ms mixed, 19.1 against 17.1 ms FP64, where the flattened form's
    // larger register and shared-memory footprint costs occupancy.
    // FMM2D_B200_P2P=flat / group overrides.
    const char *mode = getenv("FMM2D_B200_P2P");
    const bool flat = mode ? !strcmp(mode, "flat") : MIXED;
#define FMM_P2P_CASE(IFC, IFD)                                                  \
    do {                                                                        \
        if (flat) {                                                             \
            constexpr size_t sm =                                               \
                kP2PWarps * p2p_flat_warp_bytes<CH, PGH, IFC, IFD, MIXED>();    \
            auto kern = p2p_flat_kernel<CH, PGH, IFC, IFD, MIXED, LAPR>;        \
            raise_smem_limit(kern, sm);                                         \
            kern<<<g, kP2PWarps * 32, sm, s>>>(lo, hi, n1, l1, nc, leaves, sse, \
                                              spos, chg, dip, P.sset, P.tset,   \
                                              spos, tpos, P.ndc, c0, th2);      \
        } else {                                                                \
            constexpr size_t sm = p2p_smem_bytes<CH, IFC, IFD, MIXED>();        \
            auto kern = p2p_kernel<CH, PGH, IFC, IFD, MIXED, LAPR>;             \
            raise_smem_limit(kern, sm);                                         \
            kern<<<g, kP2PWarps * 32, sm, s>>>(lo, hi, n1, l1, nc, leaves, sse, \
                                              spos, chg, dip, P.sset, P.tset,   \
                                              spos, tpos, P.ndc, c0, th2);      \
        }                                                                       \
    } while (0)
    if (P.ifcharge && P.ifdipole)
        FMM_P2P_CASE(true, true);
    else if (P.ifcharge)
        FMM_P2P_CASE(true, false);
    else
        FMM_P2P_CASE(false, true);
#undef FMM_P2P_CASE
    FMM_CHECK_LAUNCH();
}

// P2P for both point sets over boxes [lo, hi): leaves, or the non-leaf
// boxes that hold list-1 entries (a second launch, so that no two warps
// write the same point).
template <int CH>
void launch_p2p(const Tree &T, const CauchyProblem &P, int c0, double th2,
                int lo, int hi, int leaves, cudaStream_t s) {
    const int pgh = std::max(P.sset.n > 0 ? P.sset.pgh : 0, P.tset.n > 0 ? P.tset.pgh : 0);
#define FMM_P2P_PGH(PG)                                                         \
    if (CH == 2 && P.real_charge) {                                             \
        if (P.mixed)                                                            \
            launch_p2p_t<CH, PG, true, true>(T, P, c0, th2, lo, hi, leaves, s); \
        else                                                                    \
            launch_p2p_t<CH, PG, false, true>(T, P, c0, th2, lo, hi, leaves, s); \
    } else if (P.mixed)                                                         \
        launch_p2p_t<CH, PG, true, false>(T, P, c0, th2, lo, hi, leaves, s);    \
    else                                                                        \
        launch_p2p_t<CH, PG, false, false>(T, P, c0, th2, lo, hi, leaves, s);
    switch (pgh) {
        case 1: FMM_P2P_PGH(1) break;
        case 2: FMM_P2P_PGH(2) break;
        case 3: FMM_P2P_PGH(3) break;
        default: break;
    }
#undef FMM_P2P_PGH
}

template <int CH>
void launch_eval_far(const Tree &T, const CauchyProblem &P, const PointSet &set,
                     const int *leaf, int c0, const double2 *mp,
                     const double2 *loc, const float2 *mp32, const float2 *loc32,
                     cudaStream_t s) {
    const int blocks = std::max(1, std::min((set.n + 255) / 256, kNumSM * 8));
#define FMM_EVAL_CASE(PG, MX)                                                   \
    eval_far_points_kernel<CH, PG, MX><<<blocks, 256, 0, s>>>(                  \
        set.n, leaf, T.level.get(), T.centers.get(), T.d_boxsize.get(),         \
        T.nlist3.get(), T.list3.get(), T.srcse.get(), set, P.ndc, c0, P.p,      \
        T.nlevels, mp, loc, mp32, loc32)
    if (P.mixed) {
        if (set.pgh == 1) FMM_EVAL_CASE(1, true);
        if (set.pgh == 2) FMM_EVAL_CASE(2, true);
        if (set.pgh == 3) FMM_EVAL_CASE(3, true);
    } else {
        if (set.pgh == 1) FMM_EVAL_CASE(1, false);
        if (set.pgh == 2) FMM_EVAL_CASE(2, false);
        if (set.pgh == 3) FMM_EVAL_CASE(3, false);
    }
#undef FMM_EVAL_CASE
    FMM_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Expansion operators with one thread per (box, coefficient): every thread
// owns one coefficient of one box for the chunk's channels, so lanes are
// never idle on short expansions and no warp shuffles are needed.
// ---------------------------------------------------------------------------

// Step 1, P2M (l2dformmpc/d/cd, laprouts2d.c:41-190) at the leaves of levels
// >= 2 with sources:  M_0 += q,  M_k += -q z^k / k,  M_k += d z^(k-1) / r,
// z = (x - c) / r.
template <int CH>
__global__ void __launch_bounds__(256) p2m_coef_kernel(
    int lo, int hi, int p, const int *__restrict__ nchild,
    const double2 *__restrict__ centers, const int *__restrict__ level,
    const double *__restrict__ bs, const int2 *__restrict__ sse,
    const double2 *__restrict__ src, const double2 *__restrict__ chg,
    const double2 *__restrict__ dip, int ifc, int ifd, int ndc, int c0,
    double2 *__restrict__ mp) {
    const int np1 = p + 1, stride = np1 * ndc;
    const int64_t n = (int64_t)(hi - lo) * np1;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = lo + (int)(t / np1), k = (int)(t % np1);
        if (nchild[b] != 0) continue;
        const int2 rg = sse[b];
        if (rg.y <= rg.x) continue;
        const double2 c = centers[b];
        const double r = bs[level[b]], rinv = 1.0 / r;
        double2 acc[CH];
#pragma unroll
        for (int q = 0; q < CH; q++) acc[q] = make_double2(0.0, 0.0);
        const double ck = k > 0 ? -1.0 / k : 0.0;
        for (int j = rg.x; j < rg.y; j++) {
            const double2 x = src[j];
            const double2 z = make_double2((x.x - c.x) / r, (x.y - c.y) / r);
            const double2 zk1 = k > 0 ? zpow_int(z, k - 1) : make_double2(0.0, 0.0);
            const double2 zk = k > 0 ? cmul(zk1, z) : make_double2(1.0, 0.0);
#pragma unroll
            for (int q = 0; q < CH; q++) {
                if (ifc) {
                    const double2 qq = chg[(size_t)j * ndc + c0 + q];
                    if (k == 0)
                        acc[q] = cadd(acc[q], qq);
                    else
                        cfma(acc[q], qq, cscal(zk, ck));
                }
                if (ifd && k > 0) cfma(acc[q], dip[(size_t)j * ndc + c0 + q], cscal(zk1, rinv));
            }
        }
#pragma unroll
        for (int q = 0; q < CH; q++) mp[(size_t)b * stride + (size_t)k * ndc + c0 + q] = acc[q];
    }
}

// Step 2, P2L from list 4 (l2dformtac/d/cd, laprouts2d.c:358-505):
//   L_0 += q log|z|,  L_k += -q (r/z)^k / k,  L_k += -d (r/z)^k / z.
template <int CH>
__global__ void __launch_bounds__(256) p2l_coef_kernel(
    int lo, int hi, int p, EvalCounts ec, const int *__restrict__ nlist4,
    const int *__restrict__ list4, const double2 *__restrict__ centers,
    const int *__restrict__ level, const double *__restrict__ bs,
    const double2 *__restrict__ src, const double2 *__restrict__ chg,
    const double2 *__restrict__ dip, int ifc, int ifd, int ndc, int c0,
    double2 *__restrict__ loc) {
    const int np1 = p + 1, stride = np1 * ndc;
    const int64_t n = (int64_t)(hi - lo) * np1;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = lo + (int)(t / np1), k = (int)(t % np1);
        const int n4 = nlist4[b];
        if (n4 == 0 || ec.npts(b) <= 0) continue;
        const double2 c = centers[b];
        const double r = bs[level[b]];
        const double ck = k > 0 ? -1.0 / k : 0.0;
        double2 acc[CH];
#pragma unroll
        for (int q = 0; q < CH; q++) acc[q] = make_double2(0.0, 0.0);
        for (int e = 0; e < n4; e++) {
            const int2 rg = ec.sse[list4[kMaxList4 * b + e]];
            for (int j = rg.x; j < rg.y; j++) {
                const double2 x = src[j];
                const double2 z0 = make_double2(x.x - c.x, x.y - c.y);
                const double2 zi = cinv(z0);
                const double2 wk = zpow_int(cscal(zi, r), k);  // (r/z)^k
                const double lz = k == 0 ? 0.5 * log(z0.x * z0.x + z0.y * z0.y) : 0.0;
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    if (ifc) {
                        const double2 qq = chg[(size_t)j * ndc + c0 + q];
                        if (k == 0)
                            cfma(acc[q], qq, make_double2(lz, 0.0));
                        else
                            cfma(acc[q], qq, cscal(wk, ck));
                    }
                    if (ifd) cfma(acc[q], dip[(size_t)j * ndc + c0 + q], cscal(cmul(wk, zi), -1.0));
                }
            }
        }
#pragma unroll
        for (int q = 0; q < CH; q++) {
            double2 &o = loc[(size_t)b * stride + (size_t)k * ndc + c0 + q];
            o = cadd(o, acc[q]);
        }
    }
}

// Child position (0..3) of box b in its parent.
__device__ __forceinline__ int child_pos(const int *__restrict__ child, int pb, int b) {
    int c = 0;
#pragma unroll
    for (int j = 1; j < 4; j++)
        if (child[4 * pb + j] == b) c = j;
    return c;
}

// Step 3, M2M (l2dmpmp, laprouts2d.c:666-775) for the parents of one level:
//   H_i = sum over children with sources of sum_j A[cpos][i][j] M_j,
// with the fixed shift matrices A of the four child positions.
template <int CH>
__global__ void __launch_bounds__(256) m2m_coef_kernel(
    int lo, int hi, int p, const int *__restrict__ nchild,
    const int *__restrict__ child, const int2 *__restrict__ sse,
    const double2 *__restrict__ A, int ndc, int c0, double2 *__restrict__ mp) {
    const int np1 = p + 1, stride = np1 * ndc;
    const int64_t n = (int64_t)(hi - lo) * np1;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = lo + (int)(t / np1), i = (int)(t % np1);
        if (nchild[b] == 0) continue;
        double2 acc[CH];
#pragma unroll
        for (int q = 0; q < CH; q++) acc[q] = make_double2(0.0, 0.0);
        for (int cp = 0; cp < 4; cp++) {
            const int cb = child[4 * b + cp];
            if (count(sse, cb) <= 0) continue;
            const double2 *Arow = A + ((size_t)cp * np1 + i) * np1;
            const double2 *M = mp + (size_t)cb * stride + c0;
            for (int j = 0; j <= i; j++) {
                const double2 a = Arow[j];
#pragma unroll
                for (int q = 0; q < CH; q++) cfma(acc[q], a, M[(size_t)j * ndc + q]);
            }
        }
#pragma unroll
        for (int q = 0; q < CH; q++) mp[(size_t)b * stride + (size_t)i * ndc + c0 + q] = acc[q];
    }
}

// Step 5, L2L (l2dlocloc, laprouts2d.c:777-884) for the children of one
// level whose parent holds points:  L_i += sum_{j>=i} A[cpos][i][j] Lp_j.
template <int CH>
__global__ void __launch_bounds__(256) l2l_coef_kernel(
    int lo, int hi, int p, EvalCounts ec, const int *__restrict__ parent,
    const int *__restrict__ child, const double2 *__restrict__ A, int ndc,
    int c0, double2 *__restrict__ loc) {
    const int np1 = p + 1, stride = np1 * ndc;
    const int64_t n = (int64_t)(hi - lo) * np1;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = lo + (int)(t / np1), i = (int)(t % np1);
        const int pb = parent[b];
        if (ec.npts(pb) <= 0) continue;
        const int cp = child_pos(child, pb, b);
        const double2 *Arow = A + ((size_t)cp * np1 + i) * np1;
        const double2 *Lp = loc + (size_t)pb * stride + c0;
        double2 acc[CH];
#pragma unroll
        for (int q = 0; q < CH; q++) acc[q] = make_double2(0.0, 0.0);
        for (int j = i; j <= p; j++) {
            const double2 a = Arow[j];
#pragma unroll
            for (int q = 0; q < CH; q++) cfma(acc[q], a, Lp[(size_t)j * ndc + q]);
        }
#pragma unroll
        for (int q = 0; q < CH; q++) {
            double2 &o = loc[(size_t)b * stride + (size_t)i * ndc + c0 + q];
            o = cadd(o, acc[q]);
        }
    }
}

// Fixed M2M / L2L shift matrices of the four child positions, in scaled
// form (level independent): a child's center is its parent's +/- r_c / 2
// in x and y (r_c the child's box size), so with s = sx + i sy, sx, sy = +-1,
//   M2M: z0/r_child = s/2, z0/r_parent = s/4;  L2L: z0/r_parent = s/4,
//   r_child/z0 = 2/s,
// all exact in binary.  Layout [cpos][i][j], (p+1)^2 per position.
const double2 *shift_tables(int p, bool m2m, cudaStream_t s) {
    static std::mutex mu;
    static std::vector<std::pair<long, const double2 *>> cache;
    int dev;
    FMM_CUDA(cudaGetDevice(&dev));
    const long key = ((long)dev << 20) | ((long)p << 1) | (m2m ? 1 : 0);
    std::lock_guard<std::mutex> g(mu);
    for (auto &e : cache)
        if (e.first == key) return e.second;
    const int n = p + 1;
    // exact binomials by the Pascal recurrence
    std::vector<double> C((size_t)(2 * n + 1) * (2 * n + 1), 0.0);
    const int nc = 2 * n + 1;
    for (int l = 0; l < nc; l++) {
        C[(size_t)l * nc] = 1.0;
        C[(size_t)l * nc + l] = 1.0;
        for (int m = 1; m < l; m++)
            C[(size_t)l * nc + m] = C[(size_t)(l - 1) * nc + m - 1] + C[(size_t)(l - 1) * nc + m];
    }
    auto binom = [&](int l, int m) { return (m < 0 || m > l) ? 0.0 : C[(size_t)l * nc + m]; };
    typedef std::complex<double> cd;
    std::vector<double2> h((size_t)4 * n * n, make_double2(0.0, 0.0));
    for (int cp = 0; cp < 4; cp++) {
        const cd sgn((cp & 1) ? 1.0 : -1.0, (cp & 2) ? 1.0 : -1.0);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                cd v(0.0, 0.0);
                if (m2m) {
                    const cd z_par = sgn / 4.0, rz_ch = 2.0 / sgn;  // z0/r2, r1/z0
                    if (i == 0)
                        v = (j == 0) ? cd(1.0, 0.0) : cd(0.0, 0.0);
                    else if (j == 0)
                        v = std::pow(z_par, i) * (-1.0 / i);
                    else if (j <= i)
                        v = std::pow(z_par, i) * binom(i - 1, j - 1) * std::pow(rz_ch, j);
                } else {
                    const cd z_par = sgn / 4.0, rz_ch = 2.0 / sgn;  // z0/r1, r2/z0
                    if (j >= i) v = std::pow(rz_ch, i) * binom(j, i) * std::pow(z_par, j);
                }
                h[((size_t)cp * n + i) * n + j] = make_double2(v.real(), v.imag());
            }
    }
    double2 *d = nullptr;
    FMM_CUDA(cudaMalloc(&d, h.size() * sizeof(double2)));
    FMM_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaStreamSynchronize(s));
    cache.push_back({key, d});
    return d;
}


// ---------------------------------------------------------------------------
// M2M and L2L as Pascal-triangle passes, without shift matrices.  With the
// child center at c_parent + d r_parent, d = (+-1 +- i) / 4, the entries of
// the scaled shifts (the matrices of shift_tables above) give
//   L2L: L'_i = 2^-i sum_{j>=i} C(j, i) d^(j-i) L_j
//        = 2^-i d^-i e_i,  e_j = d^j L_j after the passes e_j += e_(j+1)
//   M2M: M_i = d^i (sum_{j=1..i} C(i-1, j-1) (2d)^-j M'_j - M'_0 / i),
//        the sum being f_i after the passes f_m += f_(m-1), f_j = (2d)^-j M'_j
// so each (box, channel) costs p^2 / 2 complex additions and O(p) complex
// products, all in registers.  L2L takes one thread per (child, channel);
// M2M one per (parent, channel, child), the four children's parts summed
// over adjacent lanes with shuffles.  FP64 throughout.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 child_offset(int cs) {
    return make_double2((cs & 1) ? 0.25 : -0.25, (cs & 2) ? 0.25 : -0.25);
}

// The boxes visited come from a BoxList (the level's boxes with evaluation
// points, whose parents then have points too), or, with ids null, are all
// boxes of [lo, hi) whose parent has points.
template <int PMAX>
__global__ void __launch_bounds__(128) l2l_pascal_kernel(
    int lo, int hi, int p, EvalCounts ec, const int *__restrict__ ids,
    const int *__restrict__ nids, const int *__restrict__ parent,
    const int *__restrict__ child, int ndc, int c0, int nch, double2 *__restrict__ loc,
    float2 *__restrict__ loc32) {
    const int stride = (p + 1) * ndc;
    const int64_t total = (int64_t)(ids ? *nids : hi - lo) * nch;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t / nch), q = c0 + (int)(t % nch);
        const int b = ids ? ids[k] : lo + k;
        const int pb = parent[b];
        if (!ids && ec.npts(pb) <= 0) continue;
        const double2 d = child_offset(child_pos(child, pb, b));
        const double2 *Lp = loc + (size_t)pb * stride + q;
        double2 e[PMAX];
        double2 w = make_double2(1.0, 0.0);
#pragma unroll
        for (int j = 0; j < PMAX; j++) {
            e[j] = j <= p ? cmul(w, Lp[(size_t)j * ndc]) : make_double2(0.0, 0.0);
            w = cmul(w, d);
        }
#pragma unroll
        for (int k = 0; k < PMAX - 1; k++)
#pragma unroll
            for (int j = PMAX - 2; j >= k; j--) e[j] = cadd(e[j], e[j + 1]);
        // (d / 2)^-i
        const double2 h = cinv(cscal(d, 2.0));
        double2 v = make_double2(1.0, 0.0);
        double2 *Lc = loc + (size_t)b * stride + q;
#pragma unroll
        for (int i = 0; i < PMAX; i++) {
            if (i > p) break;
            const double2 r = cadd(Lc[(size_t)i * ndc], cmul(v, e[i]));
            Lc[(size_t)i * ndc] = r;
            // (the box's local expansion is final here: FP32 copy for the
            // mixed-mode evaluation at the points)
            if (loc32) loc32[(size_t)b * stride + (size_t)i * ndc + q] = make_float2((float)r.x, (float)r.y);
            v = cmul(v, h);
        }
    }
}

// The parents visited come from a BoxList (the level's parents with
// sources), or, with ids null, are all boxes of [lo, hi) with children.
template <int PMAX>
__global__ void __launch_bounds__(128) m2m_pascal_kernel(
    int lo, int hi, int p, const int *__restrict__ ids, const int *__restrict__ nids,
    const int *__restrict__ nchild, const int *__restrict__ child,
    const int2 *__restrict__ sse, int ndc, int c0, int nch, double2 *__restrict__ mp) {
    const int stride = (p + 1) * ndc;
    const int64_t total = (int64_t)(ids ? *nids : hi - lo) * nch * 4;
    // warp-uniform trip count: the lanes of a parent meet in the shuffles
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < total;
         base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = base + threadIdx.x;
        const bool valid = t < total;
        const int64_t tt = valid ? t : 0;
        const int b = ids ? ids[(int)(tt / (4 * nch))] : lo + (int)(tt / (4 * nch));
        const int q = c0 + (int)((tt / 4) % nch), cs = (int)(tt % 4);
        const bool par = valid && nchild[b] > 0;
        const double2 d = child_offset(cs);
        double2 f[PMAX];
#pragma unroll
        for (int j = 0; j < PMAX; j++) f[j] = make_double2(0.0, 0.0);
        double2 a0 = make_double2(0.0, 0.0);
        const int cb = par ? child[4 * b + cs] : -1;
        if (cb >= 0 && count(sse, cb) > 0) {
            const double2 *M = mp + (size_t)cb * stride + q;
            a0 = M[0];
            // f_j = (2d)^-j M'_j
            const double2 r2 = cinv(cscal(d, 2.0));
            double2 w = r2;
#pragma unroll
            for (int j = 1; j < PMAX; j++) {
                if (j <= p) f[j] = cmul(w, M[(size_t)j * ndc]);
                w = cmul(w, r2);
            }
        }
#pragma unroll
        for (int k = 1; k < PMAX - 1; k++)
#pragma unroll
            for (int m = PMAX - 1; m > k; m--) f[m] = cadd(f[m], f[m - 1]);
        // M_i = d^i (f_i - a0 / i), M_0 = a0; summed over the four children
        double2 w = d;
        f[0] = a0;
#pragma unroll
        for (int i = 1; i < PMAX; i++) {
            f[i] = cmul(w, csub(f[i], cscal(a0, 1.0 / i)));
            w = cmul(w, d);
        }
#pragma unroll
        for (int i = 0; i < PMAX; i++) {
            if (i > p) break;
            double2 v = f[i];
            v.x += __shfl_xor_sync(0xffffffffu, v.x, 1);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, 1);
            v.x += __shfl_xor_sync(0xffffffffu, v.x, 2);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, 2);
            if (par && cs == 0) mp[(size_t)b * stride + (size_t)i * ndc + q] = v;
        }
    }
}

// The boxes the Pascal M2M and L2L, the FP32 P2M and the P2L visit, made in
// one launch.  List i holds the boxes with bit i of sel(b): lists 0 and 1
// (M2M, L2L) in one segment per level, level l's at ids[i][ls[l] ..
// ls[l] + cnt[i][l]) (the level's box range bounds it), lists 2 and 3
// (P2M, P2L) in one segment, ids[i][0 .. cnt[i][0]).  Slots come from
// warp-aggregated atomic counters, so the order within a segment is not
// box order; every visited box's work is independent of the others', so
// the results do not depend on it.
struct LevelStarts {
    int v[kMaxLevels + 2];
};
struct BoxLists {
    DevBuf<int> ids[4], cnt;
    int L = 0;
    // list i's count for level l (lists 0, 1) or all (2, 3)
    const int *count(int i, int l) const { return cnt.get() + i * (L + 1) + (i < 2 ? l : 0); }
};

template <class Sel>
void make_box_lists(const Tree &T, const LevelStarts &ls, Sel sel, BoxLists &B, cudaStream_t s) {
    const int nb = T.nboxes, L = T.nlevels;
    B.L = L;
    for (int i = 0; i < 4; i++) B.ids[i].alloc(std::max(nb, 1), s);
    B.cnt.alloc((size_t)4 * (L + 1), s);
    B.cnt.zero(s);
    int *i0 = B.ids[0].get(), *i1 = B.ids[1].get(), *i2 = B.ids[2].get(), *i3 = B.ids[3].get();
    int *cn = B.cnt.get();
    const int *lev = T.level.get();
    for_each(nb, s, [=] __device__(int64_t t) {
        const int b = (int)t, l = lev[b];
        const unsigned m = sel(b);
        const unsigned am = __activemask();
        const int lane = (int)(threadIdx.x & 31);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int key = ((m >> i) & 1u) ? (i < 2 ? l : 0) : -1;
            const unsigned peers = __match_any_sync(am, key);
            const int leader = __ffs(peers) - 1;
            int base = 0;
            if (key >= 0 && lane == leader)
                base = atomicAdd(cn + i * (L + 1) + key, __popc(peers));
            base = __shfl_sync(peers, base, leader);
            if (key >= 0) {
                int *ids = i == 0 ? i0 : (i == 1 ? i1 : (i == 2 ? i2 : i3));
                const int rank = __popc(peers & ((1u << lane) - 1u));
                ids[(i < 2 ? ls.v[l] : 0) + base + rank] = b;
            }
        }
    });
}

inline int pascal_grid(int64_t nthreads) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((nthreads + 127) / 128, kNumSM * 16));
}

// ---------------------------------------------------------------------------
// P2M (leaves of levels >= 2 with sources) and P2L (list 4) with one warp
// per box.  Sources go in chunks of kPowSrc: the chunk's lanes build each
// source's powers b^k (b = (x - c) / r for P2M, r / (x - c) for P2L) by
// the same recurrence as the per-box form and stage them with the
// strengths; then lane k sums coefficient k over the chunk.  P2M stores the
// multipoles (their first writer), P2L adds to the locals.
//   P2M: M_0 += q,  M_k += -q z^k / k + (d / r) z^(k-1)
//   P2L: L_0 += q log|z0| - d / z0,  L_k += -q w^k / k - (d / z0) w^k
// ---------------------------------------------------------------------------
constexpr int kPowSrc = 16;
constexpr int kPowWarps = 8;

inline size_t pow_warp_smem(int p, int CH) {
    // per warp: powers [kPowSrc][P], strengths [kPowSrc][2 CH], log|z0| [kPowSrc]
    return (size_t)kPowWarps * ((size_t)kPowSrc * (p + 1 + 2 * CH) * sizeof(double2) +
                                (size_t)kPowSrc * sizeof(double));
}

// Strengths as the passes read them: FP64, or the FP32 copies of the mixed
// mode (widened on load).
__device__ __forceinline__ double2 str_d2(double2 v) { return v; }
__device__ __forceinline__ double2 str_d2(float2 v) { return make_double2(v.x, v.y); }

template <int CH, bool P2L, class S>
__device__ __forceinline__ void pow_warp_box(int b, int p, int lane, double2 *sPw, double2 *sSt,
                                             double *sLz, const double2 c, const double r,
                                             const int2 *rgs, int nrg,
                                             const double2 *__restrict__ src,
                                             const S *__restrict__ chg,
                                             const S *__restrict__ dip, int ifc, int ifd,
                                             int ndc, int c0, double2 (&acc)[2][CH]) {
    const int P = p + 1;
    for (int g = 0; g < nrg; g++) {
        const int2 rg = rgs[g];
        for (int j0 = rg.x; j0 < rg.y; j0 += kPowSrc) {
            const int n = min(kPowSrc, rg.y - j0);
            __syncwarp();
            if (lane < n) {
                const int j = j0 + lane;
                const double2 x = src[j];
                double2 base;
                double2 dv[CH];
                if (P2L) {
                    const double2 z0 = make_double2(x.x - c.x, x.y - c.y);
                    const double2 zi = cinv(z0);
                    base = cscal(zi, r);  // r / z0
                    sLz[lane] = 0.5 * log(z0.x * z0.x + z0.y * z0.y);
#pragma unroll
                    for (int q = 0; q < CH; q++)
                        dv[q] = ifd ? cscal(cmul(str_d2(dip[(size_t)j * ndc + c0 + q]), zi), -1.0)
                                    : make_double2(0.0, 0.0);
                } else {
                    base = make_double2((x.x - c.x) / r, (x.y - c.y) / r);
                    const double rinv = 1.0 / r;
#pragma unroll
                    for (int q = 0; q < CH; q++)
                        dv[q] = ifd ? cscal(str_d2(dip[(size_t)j * ndc + c0 + q]), rinv)
                                    : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    sSt[lane * 2 * CH + q] =
                        ifc ? str_d2(chg[(size_t)j * ndc + c0 + q]) : make_double2(0.0, 0.0);
                    sSt[lane * 2 * CH + CH + q] = dv[q];
                }
                double2 w = make_double2(1.0, 0.0);
                for (int k = 0; k < P; k++) {
                    sPw[lane * P + k] = w;
                    w = cmul(w, base);
                }
            }
            __syncwarp();
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int k = lane + 32 * h;
                if (k >= P) break;
                const double ik = k > 0 ? -1.0 / k : 0.0;
                for (int s = 0; s < n; s++) {
                    const double2 pk = sPw[s * P + k];
                    // P2M: the dipole term takes z^(k-1); P2L takes w^k
                    const double2 pd = P2L ? pk : (k > 0 ? sPw[s * P + k - 1] : make_double2(0.0, 0.0));
                    const double lz = P2L ? sLz[s] : 0.0;
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        const double2 qv = sSt[s * 2 * CH + q], dv = sSt[s * 2 * CH + CH + q];
                        if (k == 0)
                            acc[h][q] = cadd(acc[h][q], P2L ? cscal(qv, lz) : qv);
                        else
                            cfma(acc[h][q], qv, cscal(pk, ik));
                        cfma(acc[h][q], dv, pd);
                    }
                }
            }
        }
    }
}

template <int CH>
__global__ void __launch_bounds__(kPowWarps * 32) p2m_warp_kernel(
    int lo, int hi, int p, const int *__restrict__ nchild, const double2 *__restrict__ centers,
    const int *__restrict__ level, const double *__restrict__ bs, const int2 *__restrict__ sse,
    const double2 *__restrict__ src, const double2 *__restrict__ chg,
    const double2 *__restrict__ dip, int ifc, int ifd, int ndc, int c0,
    double2 *__restrict__ mp) {
    extern __shared__ double2 pow_smem[];
    const int P = p + 1, stride = P * ndc;
    const int lane = lane_id(), wib = threadIdx.x >> 5;
    double2 *sPw = pow_smem + (size_t)wib * kPowSrc * (P + 2 * CH);
    double2 *sSt = sPw + kPowSrc * P;
    double *sLz = reinterpret_cast<double *>(pow_smem + (size_t)kPowWarps * kPowSrc * (P + 2 * CH)) +
                  wib * kPowSrc;
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        if (nchild[b] != 0) continue;
        const int2 rg = sse[b];
        if (rg.y <= rg.x) continue;
        double2 acc[2][CH];
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
            for (int q = 0; q < CH; q++) acc[h][q] = make_double2(0.0, 0.0);
        pow_warp_box<CH, false, double2>(b, p, lane, sPw, sSt, sLz, centers[b], bs[level[b]], &rg, 1, src,
                                chg, dip, ifc, ifd, ndc, c0, acc);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = lane + 32 * h;
            if (k >= P) break;
#pragma unroll
            for (int q = 0; q < CH; q++) mp[(size_t)b * stride + (size_t)k * ndc + c0 + q] = acc[h][q];
        }
    }
}

// P2M of the mixed mode: the same scheme with the power series and its
// sums in FP32 (the multipoles feed the FP32 / TF32 M2L, which reads them
// rounded to FP32), from FP32 charges; the scaled offsets (x - c) / r and
// d / r are formed in FP64 before the conversion.  A chunk holds up to 32
// sources (a leaf's sources in one chunk: every lane builds one source's
// powers), a source's strengths are read back as 16-byte pairs, and with
// real charges (LAPR: lfmm2d's channels, imaginary parts exactly 0) the
// charge terms drop their zero halves (the same sums to the bit).
constexpr int kPow32Src = 32;

inline size_t pow32_warp_smem(int p, int CH) {
    return (size_t)kPowWarps * kPow32Src * (p + 1 + 2 * CH) * sizeof(float2);
}

// S: the dipole strengths' type (FP64, or the mixed mode's FP32 copies).
// ids / off (optional): the leaves with sources in box order, entries
// ids[off[lo] .. off[hi]) (only those are visited).
template <int CH, class S, bool LAPR>
__global__ void __launch_bounds__(kPowWarps * 32) p2m_warp32_kernel(
    int lo, int hi, const int *__restrict__ ids, const int *__restrict__ nids, int p,
    const int *__restrict__ nchild, const double2 *__restrict__ centers,
    const int *__restrict__ level, const double *__restrict__ bs, const int2 *__restrict__ sse,
    const double2 *__restrict__ src, const float2 *__restrict__ chg32,
    const S *__restrict__ dip, int ifc, int ifd, int ndc, int c0,
    double2 *__restrict__ mp) {
    extern __shared__ float2 pow32_smem[];
    const int P = p + 1, stride = P * ndc;
    const int lane = lane_id(), wib = threadIdx.x >> 5;
    float2 *sPw = pow32_smem + (size_t)wib * kPow32Src * (P + 2 * CH);
    // strengths of source s: [q_0 .. q_CH-1, d_0 .. d_CH-1] at sSt + s * 2 CH
    // (16-byte aligned: the power table holds kPow32Src * P float2)
    float2 *sSt = sPw + kPow32Src * P;
    const float2 z0 = make_float2(0.f, 0.f);
    const int k0 = ids ? 0 : lo, k1 = ids ? *nids : hi;
    for (int kb = k0 + warp_global(); kb < k1; kb += warp_count()) {
        const int b = ids ? ids[kb] : kb;
        if (!ids && nchild[b] != 0) continue;
        const int2 rg = sse[b];
        if (rg.y <= rg.x) continue;
        const double2 c = centers[b];
        const double rinv = 1.0 / bs[level[b]];
        float2 acc[2][CH];
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
            for (int q = 0; q < CH; q++) acc[h][q] = z0;
        for (int j0 = rg.x; j0 < rg.y; j0 += kPow32Src) {
            const int n = min(kPow32Src, rg.y - j0);
            __syncwarp();
            if (lane < n) {
                const int j = j0 + lane;
                const double2 x = src[j];
                const float2 base = make_float2((float)((x.x - c.x) * rinv), (float)((x.y - c.y) * rinv));
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    sSt[lane * 2 * CH + q] = ifc ? chg32[(size_t)j * ndc + c0 + q] : z0;
                    const double2 d = ifd ? str_d2(dip[(size_t)j * ndc + c0 + q]) : make_double2(0.0, 0.0);
                    sSt[lane * 2 * CH + CH + q] = make_float2((float)(d.x * rinv), (float)(d.y * rinv));
                }
                float2 w = make_float2(1.f, 0.f);
                for (int k = 0; k < P; k++) {
                    sPw[lane * P + k] = w;
                    w = zmul(w, base);
                }
            }
            __syncwarp();
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int k = lane + 32 * h;
                if (k >= P) break;
                const float ik = k > 0 ? -1.f / (float)k : 0.f;
                for (int s = 0; s < n; s++) {
                    const float2 pk = sPw[s * P + k];
                    const float2 pd = k > 0 ? sPw[s * P + k - 1] : z0;  // z^(k-1) for the dipole
                    float2 qv[CH], dv[CH];
                    if constexpr (CH == 2) {
                        const float4 *st4 = reinterpret_cast<const float4 *>(sSt + s * 4);
                        const float4 a = st4[0], d4 = st4[1];
                        qv[0] = make_float2(a.x, a.y);
                        qv[1] = make_float2(a.z, a.w);
                        dv[0] = make_float2(d4.x, d4.y);
                        dv[1] = make_float2(d4.z, d4.w);
                    } else {
#pragma unroll
                        for (int q = 0; q < CH; q++) {
                            qv[q] = sSt[s * 2 * CH + q];
                            dv[q] = sSt[s * 2 * CH + CH + q];
                        }
                    }
                    const float2 pks = zscal(pk, ik);
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        if (k == 0) {
                            acc[h][q] = zadd(acc[h][q], qv[q]);
                        } else if (LAPR) {
                            acc[h][q].x = fmaf(qv[q].x, pks.x, acc[h][q].x);
                            acc[h][q].y = fmaf(qv[q].x, pks.y, acc[h][q].y);
                        } else {
                            zfma(acc[h][q], qv[q], pks);
                        }
                        zfma(acc[h][q], dv[q], pd);
                    }
                }
            }
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = lane + 32 * h;
            if (k >= P) break;
#pragma unroll
            for (int q = 0; q < CH; q++)
                mp[(size_t)b * stride + (size_t)k * ndc + c0 + q] =
                    make_double2((double)acc[h][q].x, (double)acc[h][q].y);
        }
    }
}

// S: the strengths' type (FP64, or the mixed mode's FP32 copies).
// ids / off (optional): the boxes with list-4 entries and evaluation
// points in box order, entries ids[off[lo] .. off[hi]) (only those are
// visited).
template <int CH, class S>
__global__ void __launch_bounds__(kPowWarps * 32) p2l_warp_kernel(
    int lo, int hi, const int *__restrict__ ids, const int *__restrict__ nids, int p,
    EvalCounts ec, const int *__restrict__ nlist4,
    const int *__restrict__ list4, const double2 *__restrict__ centers,
    const int *__restrict__ level, const double *__restrict__ bs,
    const double2 *__restrict__ src, const S *__restrict__ chg,
    const S *__restrict__ dip, int ifc, int ifd, int ndc, int c0,
    double2 *__restrict__ loc) {
    extern __shared__ double2 pow_smem[];
    const int P = p + 1, stride = P * ndc;
    const int lane = lane_id(), wib = threadIdx.x >> 5;
    double2 *sPw = pow_smem + (size_t)wib * kPowSrc * (P + 2 * CH);
    double2 *sSt = sPw + kPowSrc * P;
    double *sLz = reinterpret_cast<double *>(pow_smem + (size_t)kPowWarps * kPowSrc * (P + 2 * CH)) +
                  wib * kPowSrc;
    const int k0 = ids ? 0 : lo, k1 = ids ? *nids : hi;
    for (int kb = k0 + warp_global(); kb < k1; kb += warp_count()) {
        const int b = ids ? ids[kb] : kb;
        const int n4 = nlist4[b];
        if (n4 == 0 || ec.npts(b) <= 0) continue;
        int2 rgs[kMaxList4];
        for (int e = 0; e < n4; e++) rgs[e] = ec.sse[list4[kMaxList4 * b + e]];
        double2 acc[2][CH];
#pragma unroll
        for (int h = 0; h < 2; h++)
#pragma unroll
            for (int q = 0; q < CH; q++) acc[h][q] = make_double2(0.0, 0.0);
        pow_warp_box<CH, true, S>(b, p, lane, sPw, sSt, sLz, centers[b], bs[level[b]], rgs, n4,
                                  src, chg, dip, ifc, ifd, ndc, c0, acc);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = lane + 32 * h;
            if (k >= P) break;
#pragma unroll
            for (int q = 0; q < CH; q++) {
                double2 &o = loc[(size_t)b * stride + (size_t)k * ndc + c0 + q];
                o = cadd(o, acc[h][q]);
            }
        }
    }
}

inline int pow_grid(int nbox) {
    return std::max(1, std::min((nbox + kPowWarps - 1) / kPowWarps, kNumSM * 8));
}

// Upward pass for channels [c0, c0 + CH): P2M at the leaves of levels >= 2,
// then M2M from the finest parents up.
template <int CH>
void upward_chunk(const Tree &T, const CauchyProblem &P, int c0,
                  const double *binom, double2 *mp, cudaStream_t s) {
    (void)binom;
    const int L = T.nlevels, p = P.p, nb = T.nboxes;
    const double *bs = T.d_boxsize.get();
    auto blocks = [&](int nbox) {
        const int64_t n = (int64_t)nbox * (p + 1);
        return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, kNumSM * 8));
    };
    // warp-per-box kernels while their shared tables fit (p + 1 <= 40)
    const bool warpk = p + 1 <= 40;
    if (L >= 2) {
        const int lo = T.lstart[2];
        if (warpk && P.mixed && (P.charge32 || !P.ifcharge)) {
            // FP32 dipoles when there are (the FP64 ones may be absent)
            const bool d32 = P.dipstr32 || !P.ifdipole;
            const size_t sm = pow32_warp_smem(p, CH);
            auto launch = [&](auto kern, const auto *dip) {
                raise_smem_limit(kern, (int)sm);
                kern<<<pow_grid(nb - lo), kPowWarps * 32, sm, s>>>(
                    lo, nb, P.p2m_ids, P.p2m_cnt, p, T.nchild.get(), T.centers.get(), T.level.get(), bs,
                    T.srcse.get(), P.src, P.charge32, dip, P.ifcharge, P.ifdipole, P.ndc, c0, mp);
            };
            if (d32 && P.real_charge)
                launch(p2m_warp32_kernel<CH, float2, true>, P.dipstr32);
            else if (d32)
                launch(p2m_warp32_kernel<CH, float2, false>, P.dipstr32);
            else if (P.real_charge)
                launch(p2m_warp32_kernel<CH, double2, true>, P.dipstr);
            else
                launch(p2m_warp32_kernel<CH, double2, false>, P.dipstr);
        } else if (warpk) {
            const size_t sm = pow_warp_smem(p, CH);
            raise_smem_limit(p2m_warp_kernel<CH>, (int)sm);
            p2m_warp_kernel<CH><<<pow_grid(nb - lo), kPowWarps * 32, sm, s>>>(
                lo, nb, p, T.nchild.get(), T.centers.get(), T.level.get(), bs,
                T.srcse.get(), P.src, P.charge, P.dipstr, P.ifcharge, P.ifdipole,
                P.ndc, c0, mp);
        } else
            p2m_coef_kernel<CH><<<blocks(nb - lo), 256, 0, s>>>(
                lo, nb, p, T.nchild.get(), T.centers.get(), T.level.get(), bs,
                T.srcse.get(), P.src, P.charge, P.dipstr, P.ifcharge, P.ifdipole,
                P.ndc, c0, mp);
        FMM_CHECK_LAUNCH();
    }
    prof_mark("p2m", s);
    const double2 *A = shift_tables(p, true, s);
    for (int l = L - 1; l >= 1; l--) {
        const int lo = T.lstart[l], hi = T.lend[l];
        const int64_t nt = (int64_t)(hi - lo) * CH * 4;
        const int *ids = P.m2m_ids ? P.m2m_ids + lo : nullptr;
        const int *nid = P.m2m_ids ? P.m2m_cnt + l : nullptr;
        if (p + 1 <= 20)
            m2m_pascal_kernel<20><<<pascal_grid(nt), 128, 0, s>>>(
                lo, hi, p, ids, nid, T.nchild.get(), T.child.get(), T.srcse.get(),
                P.ndc, c0, CH, mp);
        else if (p + 1 <= 32)
            m2m_pascal_kernel<32><<<pascal_grid(nt), 128, 0, s>>>(
                lo, hi, p, ids, nid, T.nchild.get(), T.child.get(), T.srcse.get(),
                P.ndc, c0, CH, mp);
        else if (p + 1 <= 40)
            m2m_pascal_kernel<40><<<pascal_grid(nt), 128, 0, s>>>(
                lo, hi, p, ids, nid, T.nchild.get(), T.child.get(), T.srcse.get(),
                P.ndc, c0, CH, mp);
        else
            m2m_coef_kernel<CH><<<blocks(hi - lo), 256, 0, s>>>(
                lo, hi, p, T.nchild.get(), T.child.get(), T.srcse.get(), A, P.ndc,
                c0, mp);
        FMM_CHECK_LAUNCH();
    }
    prof_mark("m2m", s);
}

// M2L with the per-box kernel, levels 2..L, channels [c0, c0 + CH).
template <int CH>
void m2l_chunk(const Tree &T, const CauchyProblem &P, int c0,
               const double *binom, const double2 *mp, double2 *loc,
               cudaStream_t s) {
    const int L = T.nlevels, p = P.p;
    const EvalCounts ec{T.srcse.get(), T.trgse.get(), P.sset.pgh, P.tset.pgh};
    const size_t sh_exp = (size_t)kWarpsPerBlock * (p + 1) * CH * sizeof(double2);
    const size_t sh_m2l = (size_t)(((p + 1) * (p + 1) + 1) & ~1) * sizeof(double) + sh_exp;
    raise_smem_limit(m2l_kernel<CH>, (int)sh_m2l);
    for (int l = 2; l <= L; l++) {
        const int lo = T.lstart[l], hi = T.lend[l];
        m2l_kernel<CH><<<grid_for(hi - lo), kBlock, sh_m2l, s>>>(
            lo, hi, ec, T.nlist2.get(), T.list2.get(), T.centers.get(),
            T.boxsize[l], P.ndc, c0, p, binom, mp, loc);
        FMM_CHECK_LAUNCH();
    }
}

// Downward pass for channels [c0, c0 + CH): P2L, L2L.
template <int CH>
void downward_chunk(const Tree &T, const CauchyProblem &P, int c0,
                    const double *binom, const double2 *mp, double2 *loc,
                    const float2 *mp32, float2 *loc32, cudaStream_t s) {
    const int L = T.nlevels, p = P.p, nb = T.nboxes;
    const double *bs = T.d_boxsize.get();
    const EvalCounts ec{T.srcse.get(), T.trgse.get(), P.sset.pgh, P.tset.pgh};
    const size_t sh_exp = (size_t)kWarpsPerBlock * (p + 1) * CH * sizeof(double2);
    (void)sh_exp;
    (void)binom;
    auto blocks = [&](int nbox) {
        const int64_t n = (int64_t)nbox * (p + 1);
        return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, kNumSM * 8));
    };
    // step 2: P2L from list 4 (after M2L, which initialises the locals)
    const bool warpk = p + 1 <= 40;
    if (L >= 2) {
        const int lo = T.lstart[2];
        if (warpk && P.mixed && (P.charge32 || !P.ifcharge) && (P.dipstr32 || !P.ifdipole)) {
            // the FP32 copies of the strengths (the FP64 ones may be absent)
            const size_t sm = pow_warp_smem(p, CH);
            raise_smem_limit(p2l_warp_kernel<CH, float2>, (int)sm);
            p2l_warp_kernel<CH, float2><<<pow_grid(nb - lo), kPowWarps * 32, sm, s>>>(
                lo, nb, P.p2l_ids, P.p2l_cnt, p, ec, T.nlist4.get(), T.list4.get(), T.centers.get(),
                T.level.get(), bs, P.src, P.charge32, P.dipstr32, P.ifcharge,
                P.ifdipole, P.ndc, c0, loc);
        } else if (warpk) {
            const size_t sm = pow_warp_smem(p, CH);
            raise_smem_limit(p2l_warp_kernel<CH, double2>, (int)sm);
            p2l_warp_kernel<CH, double2><<<pow_grid(nb - lo), kPowWarps * 32, sm, s>>>(
                lo, nb, P.p2l_ids, P.p2l_cnt, p, ec, T.nlist4.get(), T.list4.get(), T.centers.get(),
                T.level.get(), bs, P.src, P.charge, P.dipstr, P.ifcharge,
                P.ifdipole, P.ndc, c0, loc);
        } else
            p2l_coef_kernel<CH><<<blocks(nb - lo), 256, 0, s>>>(
                lo, nb, p, ec, T.nlist4.get(), T.list4.get(), T.centers.get(),
                T.level.get(), bs, P.src, P.charge, P.dipstr, P.ifcharge,
                P.ifdipole, P.ndc, c0, loc);
        FMM_CHECK_LAUNCH();
    }
    prof_mark("p2l", s);
    // step 5: L2L, coarsest parents first
    const double2 *A = shift_tables(p, false, s);
    for (int l = 1; l <= L - 1; l++) {
        const int lo = T.lstart[l + 1], hi = T.lend[l + 1];
        const int64_t nt = (int64_t)(hi - lo) * CH;
        const int *ids = P.l2l_ids ? P.l2l_ids + lo : nullptr;
        const int *nid = P.l2l_ids ? P.l2l_cnt + l + 1 : nullptr;
        if (p + 1 <= 20)
            l2l_pascal_kernel<20><<<pascal_grid(nt), 128, 0, s>>>(
                lo, hi, p, ec, ids, nid, T.parent.get(), T.child.get(), P.ndc, c0,
                CH, loc, loc32);
        else if (p + 1 <= 32)
            l2l_pascal_kernel<32><<<pascal_grid(nt), 128, 0, s>>>(
                lo, hi, p, ec, ids, nid, T.parent.get(), T.child.get(), P.ndc, c0,
                CH, loc, loc32);
        else if (p + 1 <= 40)
            l2l_pascal_kernel<40><<<pascal_grid(nt), 128, 0, s>>>(
                lo, hi, p, ec, ids, nid, T.parent.get(), T.child.get(), P.ndc, c0,
                CH, loc, loc32);
        else
            l2l_coef_kernel<CH><<<blocks(hi - lo), 256, 0, s>>>(
                lo, hi, p, ec, T.parent.get(), T.child.get(), A, P.ndc, c0, loc);
        FMM_CHECK_LAUNCH();
    }
    prof_mark("l2l", s);
}

// Steps 6-8 at the points of P.sset and P.tset (a set with pgh = 0 is left
// out): list-3 multipoles and local expansions, then the near field.
template <int CH>
void evaluate_chunk(const Tree &T, const CauchyProblem &P, int c0, const double2 *mp,
                    const double2 *loc, const float2 *mp32, const float2 *loc32, cudaStream_t s) {
    const int L = T.nlevels, p = P.p, nb = T.nboxes;
    const double *bs = T.d_boxsize.get();
    // steps 6-7: list-3 multipoles and local expansions at the points, in
    // the near-field pass over the leaves when there is one
    FarArgs fa;
    fa.p = p;
    fa.nlevels = L;
    fa.level = T.level.get();
    fa.centers = T.centers.get();
    fa.bs = bs;
    fa.nlist3 = T.nlist3.get();
    fa.list3 = T.list3.get();
    fa.mp = mp;
    fa.loc = loc;
    if (far_per_leaf(P)) {
        const int pgh = std::max(P.sset.n > 0 ? P.sset.pgh : 0, P.tset.n > 0 ? P.tset.pgh : 0);
        const int g = std::max(1, std::min((nb + kFarWarps - 1) / kFarWarps, kNumSM * 16));
#define FMM_FAR_CASE(PG)                                                                 \
    if (P.mixed)                                                                         \
        far_leaf_kernel<CH, PG, true><<<g, kFarWarps * 32, 0, s>>>(                      \
            nb, T.nchild.get(), fa, T.srcse.get(), P.sset, P.tset, P.ndc, c0);           \
    else                                                                                 \
        far_leaf_kernel<CH, PG, false><<<g, kFarWarps * 32, 0, s>>>(                     \
            nb, T.nchild.get(), fa, T.srcse.get(), P.sset, P.tset, P.ndc, c0);
        if (pgh == 1) { FMM_FAR_CASE(1) }
        if (pgh == 2) { FMM_FAR_CASE(2) }
        if (pgh == 3) { FMM_FAR_CASE(3) }
#undef FMM_FAR_CASE
        if (pgh > 0) FMM_CHECK_LAUNCH();
    } else {
        for (const PointSet *set : {&P.tset, &P.sset}) {
            if (set->pgh <= 0 || set->n <= 0) continue;
            launch_eval_far<CH>(T, P, *set, set == &P.tset ? P.tleaf : P.sleaf, c0,
                                mp, loc, mp32, loc32, s);
        }
    }
    prof_mark("m2p_l2p", s);
    // step 8: near field over list 1 (leaves, then any non-leaf box that
    // holds list-1 entries, so that no two warps write the same point)
    if (P.ifnear) {
        const double th2 = P.thresh * P.thresh;
        launch_p2p<CH>(T, P, c0, th2, 0, nb, 1, s);
        launch_p2p<CH>(T, P, c0, th2, 0, nb, 0, s);
    }
    prof_mark("p2p", s);
}

// Work counts of one evaluation for the roofline: list-2 pairs translated
// (boxes passing the step-4 test) and near-field point pairs.
__global__ void count_work_kernel(int nb, EvalCounts ec, const int *__restrict__ lev,
                                  const int *__restrict__ n1, const int *__restrict__ l1,
                                  const int *__restrict__ n2,
                                  unsigned long long *__restrict__ c) {
    unsigned long long a0 = 0, a1 = 0, a2 = 0;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        if (lev[b] >= 2 && ec.npts(b) > 0) a0 += (unsigned long long)n2[b];
        if (n1[b] > 0) {
            unsigned long long ns_ = 0;
            for (int e = 0; e < n1[b]; e++) ns_ += count(ec.sse, l1[kMaxList1 * b + e]);
            if (ec.spgh > 0) a1 += ns_ * (unsigned long long)count(ec.sse, b);
            if (ec.tpgh > 0) a2 += ns_ * (unsigned long long)count(ec.tse, b);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&c[0], a0);
        atomicAdd(&c[1], a1);
        atomicAdd(&c[2], a2);
    }
}

void count_work(const Tree &T, const CauchyProblem &P, cudaStream_t s) {
    DevBuf<unsigned long long> cnt(3, s);
    cnt.zero(s);
    const EvalCounts ec{T.srcse.get(), T.trgse.get(), P.sset.pgh, P.tset.pgh};
    count_work_kernel<<<kNumSM * 2, 256, 0, s>>>(T.nboxes, ec, T.level.get(), T.nlist1.get(),
                                                 T.list1.get(), T.nlist2.get(), cnt.get());
    FMM_CHECK_LAUNCH();
    unsigned long long h[3];
    read_small(h, cnt.get(), sizeof(h), s);
    prof_set_count("m2l_pairs", (double)h[0]);
    prof_set_count("p2p_pairs_src", (double)h[1]);
    prof_set_count("p2p_pairs_targ", (double)h[2]);
    prof_set_count("nterms", (double)P.p);
    prof_set_count("nboxes", (double)T.nboxes);
    prof_set_count("nlevels", (double)T.nlevels);
    prof_set_count("ndc", (double)P.ndc);
}

}  // namespace

const double *device_binomials(cudaStream_t s) {
    static std::mutex mu;
    static const double *tab[64] = {nullptr};
    int dev;
    FMM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(mu);
    if (!tab[dev]) {
        const int n = kLdc + 1;
        std::vector<double> h((size_t)n * n, 0.0);
        // Pascal recurrence of init_carray (fmmcommon2d.c:110-129)
        for (int l = 0; l < n; l++) h[(size_t)l * n + 0] = 1.0;
        for (int m = 1; m < n; m++) {
            h[(size_t)m * n + m] = 1.0;
            for (int l = m + 1; l < n; l++)
                h[(size_t)l * n + m] = h[(size_t)(l - 1) * n + m] + h[(size_t)(l - 1) * n + (m - 1)];
        }
        double *d = nullptr;
        FMM_CUDA(cudaMalloc(&d, h.size() * sizeof(double)));
        FMM_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
        FMM_CUDA(cudaStreamSynchronize(s));
        tab[dev] = d;
    }
    return tab[dev];
}

void cauchy_fmm(const Tree &T, const CauchyProblem &P0, cudaStream_t s) {
    // (the work counts synchronise the stream: not inside a graph capture)
    if (profiling_enabled() && !(P0.m2l_cache && P0.m2l_cache->deferred)) count_work(T, P0, s);
    CauchyProblem P = P0;
    // leaf of every sorted point, for the per-point far-field evaluation
    DevBuf<int> sleaf(std::max(P.sset.n, 1), s), tleaf(std::max(P.tset.n, 1), s);
    if (!far_per_leaf(P)) {
        const int blocks = std::max(1, std::min((T.nboxes + 255) / 256, kNumSM * 8));
        if (P.sset.pgh > 0 && P.sset.n > 0) {
            leaf_of_kernel<<<blocks, 256, 0, s>>>(T.nboxes, T.nchild.get(), T.srcse.get(), sleaf.get());
            FMM_CHECK_LAUNCH();
        }
        if (P.tset.pgh > 0 && P.tset.n > 0) {
            leaf_of_kernel<<<blocks, 256, 0, s>>>(T.nboxes, T.nchild.get(), T.trgse.get(), tleaf.get());
            FMM_CHECK_LAUNCH();
        }
        P.sleaf = sleaf.get();
        P.tleaf = tleaf.get();
    }
    // FP32 copies of the strengths for the mixed-precision near field
    DevBuf<float2> chg32, dip32;
    if (P.mixed && !P.charge32 && !P.dipstr32) {
        const size_t nv = (size_t)P.sset.n * P.ndc;
        auto conv = [&](const double2 *in, DevBuf<float2> &out) {
            if (!in || !nv) return;
            out.alloc(nv, s);
            float2 *o = out.get();
            for_each((int64_t)nv, s, [=] __device__(int64_t i) {
                o[i] = make_float2((float)in[i].x, (float)in[i].y);
            });
        };
        conv(P.charge, chg32);
        conv(P.dipstr, dip32);
        P.charge32 = chg32.get();
        P.dipstr32 = dip32.get();
    }
    // hi/lo FP32 positions for the mixed near field
    DevBuf<float4> shl, thl;
    if (P.mixed && !P.src_hl) {
        auto split = [&](const double2 *in, int n, DevBuf<float4> &out) {
            out.alloc(std::max(n, 1), s);
            float4 *o = out.get();
            for_each(n, s, [=] __device__(int64_t i) { o[i] = split_pos(in[i]); });
        };
        split(P.src, P.sset.n, shl);
        split(P.tset.pos, P.tset.n, thl);
        P.src_hl = shl.get();
        P.trg_hl = thl.get();
    }
    if (2 * P.p > kLdc)
        throw FmmError(4, "expansion order above the supported maximum (64)");
    const double *binom = device_binomials(s);
    const size_t nexp = (size_t)T.nboxes * (P.p + 1) * P.ndc;
    DevBuf<double2> mp(nexp, s), loc(nexp, s);
    // Expansions are written before they are read (P2M / M2M store the
    // multipoles of every box that has sources, M2L stores the locals of
    // every box of level >= 2 with points), except the locals of levels 0
    // and 1, which receive no M2L and start at zero.
    const int nlow = T.nlevels >= 1 ? T.lend[1] : T.lend[0];
    FMM_CUDA(cudaMemsetAsync(loc.get(), 0,
                             (size_t)nlow * (P.p + 1) * P.ndc * sizeof(double2), s));
    // the boxes the Pascal M2M and L2L visit (in adaptive trees most boxes
    // of the deep levels are leaves or empty)
    BoxLists lists;
    if (T.nlevels >= 2 && P.p + 1 <= 40) {
        const int *nchp = T.nchild.get(), *n4p = T.nlist4.get();
        const int2 *sse = T.srcse.get();
        const EvalCounts ec{T.srcse.get(), T.trgse.get(), P.sset.pgh, P.tset.pgh};
        LevelStarts ls{};
        for (int l = 0; l <= T.nlevels; l++) ls.v[l] = T.lstart[l];
        const bool mixed = P.mixed;
        make_box_lists(T, ls, [=] __device__(int b) -> unsigned {
            const bool src = count(sse, b) > 0, pts = ec.npts(b) > 0, leaf = nchp[b] == 0;
            return (!leaf && src ? 1u : 0u) | (pts ? 2u : 0u) | (mixed && leaf && src ? 4u : 0u) |
                   (n4p[b] > 0 && pts ? 8u : 0u);
        }, lists, s);
        P.m2m_ids = lists.ids[0].get();
        P.l2l_ids = lists.ids[1].get();
        P.m2m_cnt = lists.count(0, 0);
        P.l2l_cnt = lists.count(1, 0);
        if (mixed) {
            P.p2m_ids = lists.ids[2].get();
            P.p2m_cnt = lists.count(2, 0);
        }
        P.p2l_ids = lists.ids[3].get();
        P.p2l_cnt = lists.count(3, 0);
    }
    prof_mark("fmm_setup", s);
    auto per_chunk = [&](auto f2, auto f1) {
        for (int c0 = 0; c0 < P.ndc; c0 += 2) {
            if (P.ndc - c0 >= 2)
                f2(c0);
            else
                f1(c0);
        }
    };
    per_chunk([&](int c0) { upward_chunk<2>(T, P, c0, binom, mp.get(), s); },
              [&](int c0) { upward_chunk<1>(T, P, c0, binom, mp.get(), s); });
    const char *mode = getenv("FMM2D_B200_M2L");
    const bool simple = mode && !strcmp(mode, "simple");
    const bool fp32 = P.mixed && !(mode && !strcmp(mode, "fp64"));
    // Mixed mode with the per-point far field: FP32 copies of the
    // multipoles (made for the M2L) and of the final locals (written by
    // L2L) feed the evaluation at the points, which then loads half the
    // bytes and converts nothing.
    const bool copies = fp32 && !simple && !far_per_leaf(P) && T.nlevels >= 2 && P.p + 1 <= 20;
    DevBuf<float2> mp32, loc32;
    if (copies) {
        mp32.alloc(nexp, s);
        loc32.alloc(nexp, s);
        FMM_CUDA(cudaMemsetAsync(loc32.get(), 0,
                                 (size_t)nlow * (P.p + 1) * P.ndc * sizeof(float2), s));
    }
    if (simple || !((fp32 && m2l_fp32(T, P, mp.get(), loc.get(), s, mp32.get())) ||
                    (P.split && !P.mixed && m2l_split_fp64(T, P, mp.get(), loc.get(), s)) ||
                    m2l_tensor_fp64(T, P, mp.get(), loc.get(), s)))
        per_chunk([&](int c0) { m2l_chunk<2>(T, P, c0, binom, mp.get(), loc.get(), s); },
                  [&](int c0) { m2l_chunk<1>(T, P, c0, binom, mp.get(), loc.get(), s); });
    prof_mark("m2l", s);
    per_chunk([&](int c0) { downward_chunk<2>(T, P, c0, binom, mp.get(), loc.get(), mp32.get(),
                                              loc32.get(), s); },
              [&](int c0) { downward_chunk<1>(T, P, c0, binom, mp.get(), loc.get(), mp32.get(),
                                              loc32.get(), s); });
    per_chunk([&](int c0) { evaluate_chunk<2>(T, P, c0, mp.get(), loc.get(), mp32.get(),
                                              loc32.get(), s); },
              [&](int c0) { evaluate_chunk<1>(T, P, c0, mp.get(), loc.get(), mp32.get(),
                                              loc32.get(), s); });
}

}  // namespace fmm2d
