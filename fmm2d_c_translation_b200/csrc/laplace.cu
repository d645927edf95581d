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
__device__ __forceinline__ double2 shfl2(double2 v, int l) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, l),
                        __shfl_sync(0xffffffffu, v.y, l));
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
// Step 1, P2M (l2dformmpc/d/cd, laprouts2d.c:41-190):
//   M_0 += q,  M_n += -q (z/r)^n / n,  M_n += d z^(n-1) / r^n,  z = x - c.
// ---------------------------------------------------------------------------
template <int CH>
__global__ void __launch_bounds__(kBlock) p2m_kernel(
    int lo, int hi, const int *__restrict__ nchild,
    const double2 *__restrict__ centers, const int *__restrict__ level,
    const double *__restrict__ bs, const int2 *__restrict__ sse,
    const double2 *__restrict__ src, const double2 *__restrict__ chg,
    const double2 *__restrict__ dip, int ifc, int ifd, int ndc, int c0, int p,
    double2 *__restrict__ mp) {
    const int lane = lane_id();
    const int stride = (p + 1) * ndc;
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        if (nchild[b] != 0) continue;
        const int2 r_ = sse[b];
        if (r_.y <= r_.x) continue;
        const double2 c = centers[b];
        const double r = bs[level[b]], rinv = 1.0 / r;
        for (int kb = 0; kb <= p; kb += 32) {
            const int k = kb + lane;
            double2 acc[CH];
#pragma unroll
            for (int q = 0; q < CH; q++) acc[q] = make_double2(0.0, 0.0);
            for (int j = r_.x; j < r_.y; j++) {
                const double2 x = src[j];
                const double2 z = make_double2((x.x - c.x) / r, (x.y - c.y) / r);
                const double2 pw = warp_powers(z);
                const double2 zk = chunk_power(pw, z, kb);  // z^k
                double2 zk1 = shfl_up2(zk, 1);               // z^(k-1)
                if (lane == 0) zk1 = kb == 0 ? make_double2(0.0, 0.0) : zpow_int(z, kb - 1);
                if (k <= p) {
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        if (ifc) {
                            const double2 qq = chg[(size_t)j * ndc + c0 + q];
                            if (k == 0)
                                acc[q] = cadd(acc[q], qq);
                            else
                                cfma(acc[q], qq, cscal(zk, -1.0 / k));
                        }
                        if (ifd && k >= 1) {
                            const double2 dd = dip[(size_t)j * ndc + c0 + q];
                            cfma(acc[q], dd, cscal(zk1, rinv));
                        }
                    }
                }
            }
            if (k <= p) {
#pragma unroll
                for (int q = 0; q < CH; q++)
                    mp[(size_t)b * stride + (size_t)k * ndc + c0 + q] = acc[q];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Step 2, P2L from list 4 (l2dformtac/d/cd, laprouts2d.c:358-505):
//   L_0 += q log|z|,  L_n += -q (r/z)^n / n,  L_n += -d (r/z)^n / z.
// ---------------------------------------------------------------------------
template <int CH>
__global__ void __launch_bounds__(kBlock) p2l_kernel(
    int lo, int hi, EvalCounts ec, const int *__restrict__ nlist4,
    const int *__restrict__ list4, const double2 *__restrict__ centers,
    const int *__restrict__ level, const double *__restrict__ bs,
    const double2 *__restrict__ src, const double2 *__restrict__ chg,
    const double2 *__restrict__ dip, int ifc, int ifd, int ndc, int c0, int p,
    double2 *__restrict__ loc) {
    const int lane = lane_id();
    const int stride = (p + 1) * ndc;
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        const int n4 = nlist4[b];
        if (n4 == 0 || ec.npts(b) <= 0) continue;
        const double2 c = centers[b];
        const double r = bs[level[b]];
        for (int kb = 0; kb <= p; kb += 32) {
            const int k = kb + lane;
            double2 acc[CH];
#pragma unroll
            for (int q = 0; q < CH; q++) acc[q] = make_double2(0.0, 0.0);
            for (int e = 0; e < n4; e++) {
                const int jb = list4[kMaxList4 * b + e];
                const int2 r_ = ec.sse[jb];
                for (int j = r_.x; j < r_.y; j++) {
                    const double2 x = src[j];
                    const double2 z0 = make_double2(x.x - c.x, x.y - c.y);
                    const double2 zi = cinv(z0);
                    const double2 w = cscal(zi, r);                     // r/z
                    const double2 wk = chunk_power(warp_powers(w), w, kb);  // (r/z)^k
                    const double lz = 0.5 * log(z0.x * z0.x + z0.y * z0.y);
                    if (k <= p) {
#pragma unroll
                        for (int q = 0; q < CH; q++) {
                            if (ifc) {
                                const double2 qq = chg[(size_t)j * ndc + c0 + q];
                                if (k == 0)
                                    cfma(acc[q], qq, make_double2(lz, 0.0));
                                else
                                    cfma(acc[q], qq, cscal(wk, -1.0 / k));
                            }
                            if (ifd) {
                                const double2 dd = dip[(size_t)j * ndc + c0 + q];
                                cfma(acc[q], dd, cscal(cmul(wk, zi), -1.0));
                            }
                        }
                    }
                }
            }
            if (k <= p) {
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    double2 &o = loc[(size_t)b * stride + (size_t)k * ndc + c0 + q];
                    o = cadd(o, acc[q]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Step 3, M2M (l2dmpmp, laprouts2d.c:666-775), child c1 -> parent c2:
//   h~_j = h_j (r1/z0)^j,  z0 = c1 - c2
//   H_0 += h_0,  H_i += [-h~_0/i + sum_{j=1..i} C(i-1,j-1) h~_j] (z0/r2)^i
// ---------------------------------------------------------------------------
template <int CH>
__global__ void __launch_bounds__(kBlock) m2m_kernel(
    int lo, int hi, const int *__restrict__ nchild,
    const int *__restrict__ child, const double2 *__restrict__ centers,
    double r1, double r2, const int2 *__restrict__ sse, int ndc, int c0,
    int p, const double *__restrict__ binom, double2 *__restrict__ mp) {
    extern __shared__ double2 sh_m2m[];
    const int lane = lane_id();
    const int wib = threadIdx.x >> 5;
    double2 *ht = sh_m2m + (size_t)wib * (p + 1) * CH;
    const int stride = (p + 1) * ndc;
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        if (nchild[b] == 0) continue;
        const double2 c2 = centers[b];
        for (int kb = 0; kb <= p; kb += 32) {
            const int i = kb + lane;
            double2 acc[CH];
#pragma unroll
            for (int q = 0; q < CH; q++) acc[q] = make_double2(0.0, 0.0);
            for (int ch = 0; ch < 4; ch++) {
                const int cb = child[4 * b + ch];
                if (count(sse, cb) <= 0) continue;
                const double2 c1 = centers[cb];
                const double2 z0 = make_double2(c1.x - c2.x, c1.y - c2.y);
                const double2 w1 = cinv(make_double2(z0.x / r1, z0.y / r1));
                const double2 w2 = make_double2(z0.x / r2, z0.y / r2);
                const double2 pw1 = warp_powers(w1);
                for (int jb = 0; jb <= p; jb += 32) {
                    const int j = jb + lane;
                    const double2 wj = chunk_power(pw1, w1, jb);
                    if (j <= p)
#pragma unroll
                        for (int q = 0; q < CH; q++)
                            ht[j * CH + q] = cmul(mp[(size_t)cb * stride + (size_t)j * ndc + c0 + q], wj);
                }
                __syncwarp();
                const double2 wi = chunk_power(warp_powers(w2), w2, kb);
                if (i <= p) {
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        double2 t;
                        if (i == 0) {
                            t = ht[q];
                        } else {
                            t = cscal(ht[q], -1.0 / i);
                            const double *brow = binom + (size_t)(i - 1) * (kLdc + 1);
                            for (int j = 1; j <= i; j++) {
                                const double cb_ = brow[j - 1];
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
            if (i <= p) {
#pragma unroll
                for (int q = 0; q < CH; q++)
                    mp[(size_t)b * stride + (size_t)i * ndc + c0 + q] = acc[q];
            }
        }
    }
}

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
// Step 5, L2L (l2dlocloc, laprouts2d.c:777-884), parent c1 -> child c2:
//   J~_j = J_j (z0/r1)^j,  z0 = c2 - c1
//   L_i += [sum_{j>=i} C(j, i) J~_j] (r2/z0)^i
// ---------------------------------------------------------------------------
template <int CH>
__global__ void __launch_bounds__(kBlock) l2l_kernel(
    int lo, int hi, EvalCounts ec, const int *__restrict__ parent,
    const double2 *__restrict__ centers, double r1, double r2, int ndc,
    int c0, int p, const double *__restrict__ binom,
    double2 *__restrict__ loc) {
    extern __shared__ double2 sh_l2l[];
    const int lane = lane_id();
    const int wib = threadIdx.x >> 5;
    double2 *jt = sh_l2l + (size_t)wib * (p + 1) * CH;
    const int stride = (p + 1) * ndc;
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        const int pb = parent[b];
        if (ec.npts(pb) <= 0) continue;
        const double2 c1 = centers[pb], c2 = centers[b];
        const double2 z0 = make_double2(c2.x - c1.x, c2.y - c1.y);
        const double2 w1 = make_double2(z0.x / r1, z0.y / r1);
        const double2 w2 = cinv(make_double2(z0.x / r2, z0.y / r2));
        const double2 pw1 = warp_powers(w1);
        for (int jb = 0; jb <= p; jb += 32) {
            const int j = jb + lane;
            const double2 wj = chunk_power(pw1, w1, jb);
            if (j <= p)
#pragma unroll
                for (int q = 0; q < CH; q++)
                    jt[j * CH + q] = cmul(loc[(size_t)pb * stride + (size_t)j * ndc + c0 + q], wj);
        }
        __syncwarp();
        const double2 pw2 = warp_powers(w2);
        for (int kb = 0; kb <= p; kb += 32) {
            const int i = kb + lane;
            const double2 wi = chunk_power(pw2, w2, kb);
            if (i <= p) {
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    double2 t = make_double2(0.0, 0.0);
                    for (int j = i; j <= p; j++) {
                        const double cb_ = binom[(size_t)j * (kLdc + 1) + i];
                        t.x = fma(cb_, jt[j * CH + q].x, t.x);
                        t.y = fma(cb_, jt[j * CH + q].y, t.y);
                    }
                    double2 &o = loc[(size_t)b * stride + (size_t)i * ndc + c0 + q];
                    o = cadd(o, cmul(t, wi));
                }
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Steps 6 and 7 for one point set: M2P over list 3 (l2dmpevalp/g/h,
// laprouts2d.c:193-356) and L2P at leaves (l2dtaevalp/g/h, :508-664).
// Lanes run over the box's points; series by Horner's rule.
// ---------------------------------------------------------------------------
template <int CH>
__global__ void __launch_bounds__(kBlock) eval_far_kernel(
    int lo, int hi, const int *__restrict__ nchild,
    const int *__restrict__ level, const double2 *__restrict__ centers,
    const double *__restrict__ bs, const int *__restrict__ nlist3,
    const int *__restrict__ list3, const int2 *__restrict__ sse, PointSet set,
    int ndc, int c0, int p, int nlevels, const double2 *__restrict__ mp,
    const double2 *__restrict__ loc) {
    const int lane = lane_id();
    const int stride = (p + 1) * ndc;
    const int pgh = set.pgh;
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        if (nchild[b] != 0) continue;
        const int2 rg = set.se[b];
        if (rg.y <= rg.x) continue;
        const int lb = level[b];
        const double2 cb = centers[b];
        const double rb = bs[lb];
        const int n3 = (lb >= 1 && lb <= nlevels - 1) ? nlist3[b] : 0;
        for (int t0 = rg.x; t0 < rg.y; t0 += 32) {
            const int t = t0 + lane;
            const bool act = t < rg.y;
            const double2 x = act ? set.pos[t] : cb;
            double2 po[CH], gr[CH], he[CH];
#pragma unroll
            for (int q = 0; q < CH; q++)
                po[q] = gr[q] = he[q] = make_double2(0.0, 0.0);
            // list 3: multipoles of the finer separated boxes
            for (int e = 0; e < n3; e++) {
                const int jb = list3[kMaxList3 * b + e];
                if (sse[jb].y <= sse[jb].x) continue;  // no multipole
                const double2 cj = centers[jb];
                const double r = bs[level[jb]];
                double2 z = make_double2(x.x - cj.x, x.y - cj.y);
                if (!act) z = make_double2(r, 0.0);
                const double2 zi = cinv(z);
                const double2 w = cscal(zi, r);
                const double lz = 0.5 * log(z.x * z.x + z.y * z.y);
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    const double2 *M = mp + (size_t)jb * stride + c0 + q;
                    double2 q0 = M[(size_t)p * ndc], q1 = make_double2(0.0, 0.0),
                            q2 = make_double2(0.0, 0.0);
                    for (int n = p - 1; n >= 0; n--) {
                        const double2 Mn = n >= 1 ? M[(size_t)n * ndc] : make_double2(0.0, 0.0);
                        q2 = cadd(cmul(q2, w), q1);
                        q1 = cadd(cmul(q1, w), q0);
                        q0 = cadd(cmul(q0, w), Mn);
                    }
                    const double2 M0 = M[0];
                    po[q] = cadd(po[q], cadd(cscal(M0, lz), q0));
                    if (pgh >= 2) {
                        const double2 w2 = cmul(w, w);
                        const double2 g = csub(cmul(M0, zi), cscal(cmul(q1, w2), 1.0 / r));
                        gr[q] = cadd(gr[q], g);
                        if (pgh >= 3) {
                            const double2 w3 = cmul(w2, w), w4 = cmul(w2, w2);
                            double2 h = cscal(cmul(M0, cmul(zi, zi)), -1.0);
                            h = cadd(h, cscal(cmul(q2, w4), 2.0 / (r * r)));
                            h = cadd(h, cscal(cmul(q1, w3), 2.0 / (r * r)));
                            he[q] = cadd(he[q], h);
                        }
                    }
                }
            }
            // local expansion of the leaf
            {
                const double2 z = make_double2((x.x - cb.x) / rb, (x.y - cb.y) / rb);
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    const double2 *Lc = loc + (size_t)b * stride + c0 + q;
                    double2 q0 = Lc[(size_t)p * ndc], q1 = make_double2(0.0, 0.0),
                            q2 = make_double2(0.0, 0.0);
                    for (int n = p - 1; n >= 0; n--) {
                        q2 = cadd(cmul(q2, z), q1);
                        q1 = cadd(cmul(q1, z), q0);
                        q0 = cadd(cmul(q0, z), Lc[(size_t)n * ndc]);
                    }
                    po[q] = cadd(po[q], q0);
                    if (pgh >= 2) gr[q] = cadd(gr[q], cscal(q1, 1.0 / rb));
                    if (pgh >= 3) he[q] = cadd(he[q], cscal(q2, 2.0 / (rb * rb)));
                }
            }
            if (act) {
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    const size_t o = (size_t)t * ndc + c0 + q;
                    set.pot[o] = cadd(set.pot[o], po[q]);
                    if (pgh >= 2) set.grad[o] = cadd(set.grad[o], gr[q]);
                    if (pgh >= 3) set.hess[o] = cadd(set.hess[o], he[q]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Step 8, P2P over list 1 (c2d_direct*, cauchykernels2d.c:31-442):
//   pot += q log|z| + d/z,  grad += q/z - d/z^2,  hess += -q/z^2 + 2d/z^3,
// z = t - s; pairs with |z|^2 <= thresh^2 (pot only) or < thresh^2 skipped.
// A warp takes up to 32 targets of one box; when the box has fewer, lane
// groups split the sources and are summed at the end.
// ---------------------------------------------------------------------------
constexpr int kP2PStage = 64;

template <int CH, int PGH, bool IFC, bool IFD>
__device__ __forceinline__ void p2p_pair(double2 x, double2 s, const double2 *qv,
                                         const double2 *dv, double th2,
                                         double2 *po, double2 *gr, double2 *he) {
    const double dx = x.x - s.x, dy = x.y - s.y;
    const double rr = dx * dx + dy * dy;
    if (PGH == 1 ? (rr <= th2) : (rr < th2)) return;
    const double rinv2 = 1.0 / rr;
    const double2 zi = make_double2(dx * rinv2, -dy * rinv2);
    double rl = 0.0;
    if (IFC) rl = 0.5 * log(rr);
    double2 zi2 = make_double2(0.0, 0.0), zi3 = make_double2(0.0, 0.0);
    if (PGH >= 2 || IFD) zi2 = cmul(zi, zi);
    if (PGH >= 3 && IFD) zi3 = cmul(zi2, zi);
#pragma unroll
    for (int q = 0; q < CH; q++) {
        if (IFC) {
            po[q].x = fma(rl, qv[q].x, po[q].x);
            po[q].y = fma(rl, qv[q].y, po[q].y);
            if (PGH >= 2) cfma(gr[q], zi, qv[q]);
            if (PGH >= 3) cfma(he[q], cscal(zi2, -1.0), qv[q]);
        }
        if (IFD) {
            cfma(po[q], zi, dv[q]);
            if (PGH >= 2) cfma(gr[q], cscal(zi2, -1.0), dv[q]);
            if (PGH >= 3) cfma(he[q], cscal(zi3, 2.0), dv[q]);
        }
    }
}

template <int CH, int PGH, bool IFC, bool IFD>
__global__ void __launch_bounds__(kBlock) p2p_kernel(
    int lo, int hi, const int *__restrict__ nlist1,
    const int *__restrict__ list1, const int *__restrict__ nchild,
    int leaves, const int2 *__restrict__ sse, const double2 *__restrict__ src,
    const double2 *__restrict__ chg, const double2 *__restrict__ dip,
    PointSet set, int ndc, int c0, double th2) {
    // per-warp buffer: staged sources during the sweep, partial sums after
    constexpr int kStage = kP2PStage * (1 + (IFC ? CH : 0) + (IFD ? CH : 0));
    constexpr int kRed = 32 * 3 * CH;
    constexpr int kBuf = kStage > kRed ? kStage : kRed;
    __shared__ double2 s_buf[kWarpsPerBlock][kBuf];
    const int lane = lane_id(), wib = threadIdx.x >> 5;
    double2 *s_pos = s_buf[wib];
    double2 *s_q = s_pos + kP2PStage;
    double2 *s_d = s_q + (IFC ? kP2PStage * CH : 0);
    for (int b = lo + warp_global(); b < hi; b += warp_count()) {
        const int n1 = nlist1[b];
        if (n1 == 0) continue;
        if ((nchild[b] == 0) != (leaves != 0)) continue;
        const int2 rg = set.se[b];
        if (rg.y <= rg.x) continue;
        for (int t0 = rg.x; t0 < rg.y; t0 += 32) {
            const int T = min(32, rg.y - t0);
            const int G = 32 / T;
            const int g = lane / T, tl = lane - g * T;
            const bool act = g < G;
            const double2 x = act ? set.pos[t0 + tl] : make_double2(0.0, 0.0);
            double2 po[CH], gr[CH], he[CH];
#pragma unroll
            for (int q = 0; q < CH; q++)
                po[q] = gr[q] = he[q] = make_double2(0.0, 0.0);
            for (int e = 0; e < n1; e++) {
                const int jb = list1[kMaxList1 * b + e];
                const int2 sr = sse[jb];
                for (int s0 = sr.x; s0 < sr.y; s0 += kP2PStage) {
                    const int ns = min(kP2PStage, sr.y - s0);
                    for (int k = lane; k < ns; k += 32) {
                        s_pos[k] = src[s0 + k];
#pragma unroll
                        for (int q = 0; q < CH; q++) {
                            if (IFC) s_q[k * CH + q] = chg[(size_t)(s0 + k) * ndc + c0 + q];
                            if (IFD) s_d[k * CH + q] = dip[(size_t)(s0 + k) * ndc + c0 + q];
                        }
                    }
                    __syncwarp();
                    if (act) {
                        for (int k = g; k < ns; k += G) {
                            p2p_pair<CH, PGH, IFC, IFD>(
                                x, s_pos[k], IFC ? &s_q[k * CH] : nullptr,
                                IFD ? &s_d[k * CH] : nullptr, th2, po, gr, he);
                        }
                    }
                    __syncwarp();
                }
            }
            // sum the lane groups
            double2 *red = s_buf[wib];
#pragma unroll
            for (int q = 0; q < CH; q++) {
                red[(lane * 3 + 0) * CH + q] = po[q];
                red[(lane * 3 + 1) * CH + q] = gr[q];
                red[(lane * 3 + 2) * CH + q] = he[q];
            }
            __syncwarp();
            if (act && g == 0) {
                for (int gg = 1; gg < G; gg++) {
                    const int ol = gg * T + tl;
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        po[q] = cadd(po[q], red[(ol * 3 + 0) * CH + q]);
                        gr[q] = cadd(gr[q], red[(ol * 3 + 1) * CH + q]);
                        he[q] = cadd(he[q], red[(ol * 3 + 2) * CH + q]);
                    }
                }
                const int t = t0 + tl;
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    const size_t o = (size_t)t * ndc + c0 + q;
                    set.pot[o] = cadd(set.pot[o], po[q]);
                    if (PGH >= 2) set.grad[o] = cadd(set.grad[o], gr[q]);
                    if (PGH >= 3) set.hess[o] = cadd(set.hess[o], he[q]);
                }
            }
            __syncwarp();
        }
    }
}

int grid_for(int nwarps) {
    int blocks = (nwarps + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks > kNumSM * 16) blocks = kNumSM * 16;
    return blocks < 1 ? 1 : blocks;
}

template <int CH, int PGH>
void launch_p2p_t(const Tree &T, const CauchyProblem &P, const PointSet &set,
                  int c0, double th2, int lo, int hi, int leaves,
                  cudaStream_t s) {
    const int g = grid_for(hi - lo);
    const int *n1 = T.nlist1.get(), *l1 = T.list1.get(), *nc = T.nchild.get();
    const int2 *sse = T.srcse.get();
#define FMM_P2P_CASE(IFC, IFD)                                                  \
    p2p_kernel<CH, PGH, IFC, IFD><<<g, kBlock, 0, s>>>(                         \
        lo, hi, n1, l1, nc, leaves, sse, P.src, P.charge, P.dipstr, set,       \
        P.ndc, c0, th2)
    if (P.ifcharge && P.ifdipole)
        FMM_P2P_CASE(true, true);
    else if (P.ifcharge)
        FMM_P2P_CASE(true, false);
    else
        FMM_P2P_CASE(false, true);
#undef FMM_P2P_CASE
    FMM_CHECK_LAUNCH();
}

template <int CH>
void launch_p2p(const Tree &T, const CauchyProblem &P, const PointSet &set,
                int c0, double th2, int lo, int hi, int leaves, cudaStream_t s) {
    switch (set.pgh) {
        case 1: launch_p2p_t<CH, 1>(T, P, set, c0, th2, lo, hi, leaves, s); break;
        case 2: launch_p2p_t<CH, 2>(T, P, set, c0, th2, lo, hi, leaves, s); break;
        case 3: launch_p2p_t<CH, 3>(T, P, set, c0, th2, lo, hi, leaves, s); break;
        default: break;
    }
}

// Upward pass for channels [c0, c0 + CH): P2M at the leaves of levels >= 2,
// then M2M from the finest parents up.
template <int CH>
void upward_chunk(const Tree &T, const CauchyProblem &P, int c0,
                  const double *binom, double2 *mp, cudaStream_t s) {
    const int L = T.nlevels, p = P.p, nb = T.nboxes;
    const double *bs = T.d_boxsize.get();
    const size_t sh_exp = (size_t)kWarpsPerBlock * (p + 1) * CH * sizeof(double2);
    if (L >= 2) {
        const int lo = T.lstart[2];
        p2m_kernel<CH><<<grid_for(nb - lo), kBlock, 0, s>>>(
            lo, nb, T.nchild.get(), T.centers.get(), T.level.get(), bs,
            T.srcse.get(), P.src, P.charge, P.dipstr, P.ifcharge, P.ifdipole,
            P.ndc, c0, p, mp);
        FMM_CHECK_LAUNCH();
    }
    prof_mark("p2m", s);
    for (int l = L - 1; l >= 1; l--) {
        const int lo = T.lstart[l], hi = T.lend[l];
        m2m_kernel<CH><<<grid_for(hi - lo), kBlock, sh_exp, s>>>(
            lo, hi, T.nchild.get(), T.child.get(), T.centers.get(),
            T.boxsize[l + 1], T.boxsize[l], T.srcse.get(), P.ndc, c0, p,
            binom, mp);
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
    FMM_CUDA(cudaFuncSetAttribute(m2l_kernel<CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sh_m2l));
    for (int l = 2; l <= L; l++) {
        const int lo = T.lstart[l], hi = T.lend[l];
        m2l_kernel<CH><<<grid_for(hi - lo), kBlock, sh_m2l, s>>>(
            lo, hi, ec, T.nlist2.get(), T.list2.get(), T.centers.get(),
            T.boxsize[l], P.ndc, c0, p, binom, mp, loc);
        FMM_CHECK_LAUNCH();
    }
}

// Downward pass and evaluation for channels [c0, c0 + CH): P2L, L2L, M2P +
// L2P, P2P.
template <int CH>
void downward_chunk(const Tree &T, const CauchyProblem &P, int c0,
                    const double *binom, const double2 *mp, double2 *loc,
                    cudaStream_t s) {
    const int L = T.nlevels, p = P.p, nb = T.nboxes;
    const double *bs = T.d_boxsize.get();
    const EvalCounts ec{T.srcse.get(), T.trgse.get(), P.sset.pgh, P.tset.pgh};
    const size_t sh_exp = (size_t)kWarpsPerBlock * (p + 1) * CH * sizeof(double2);
    // step 2: P2L from list 4 (after M2L, which initialises the locals)
    if (L >= 2) {
        const int lo = T.lstart[2];
        p2l_kernel<CH><<<grid_for(nb - lo), kBlock, 0, s>>>(
            lo, nb, ec, T.nlist4.get(), T.list4.get(), T.centers.get(),
            T.level.get(), bs, P.src, P.charge, P.dipstr, P.ifcharge,
            P.ifdipole, P.ndc, c0, p, loc);
        FMM_CHECK_LAUNCH();
    }
    prof_mark("p2l", s);
    // step 5: L2L, coarsest parents first
    for (int l = 1; l <= L - 1; l++) {
        const int lo = T.lstart[l + 1], hi = T.lend[l + 1];
        l2l_kernel<CH><<<grid_for(hi - lo), kBlock, sh_exp, s>>>(
            lo, hi, ec, T.parent.get(), T.centers.get(), T.boxsize[l],
            T.boxsize[l + 1], P.ndc, c0, p, binom, loc);
        FMM_CHECK_LAUNCH();
    }
    prof_mark("l2l", s);
    // steps 6-7: list-3 multipoles and local expansions at the points
    for (const PointSet *set : {&P.tset, &P.sset}) {
        if (set->pgh <= 0 || set->n <= 0) continue;
        eval_far_kernel<CH><<<grid_for(nb), kBlock, 0, s>>>(
            0, nb, T.nchild.get(), T.level.get(), T.centers.get(), bs,
            T.nlist3.get(), T.list3.get(), T.srcse.get(), *set, P.ndc, c0, p,
            L, mp, loc);
        FMM_CHECK_LAUNCH();
    }
    prof_mark("m2p_l2p", s);
    // step 8: near field over list 1 (leaves, then any non-leaf box that
    // holds list-1 entries, so that no two warps write the same point)
    if (P.ifnear) {
        for (const PointSet *set : {&P.tset, &P.sset}) {
            if (set->pgh <= 0 || set->n <= 0) continue;
            const double th2 = P.thresh * P.thresh;
            launch_p2p<CH>(T, P, *set, c0, th2, 0, nb, 1, s);
            launch_p2p<CH>(T, P, *set, c0, th2, 0, nb, 0, s);
        }
    }
    prof_mark("p2p", s);
}

// Work counts of one evaluation for the roofline: list-2 pairs translated
// (boxes passing the step-4 test) and near-field point pairs.
void count_work(const Tree &T, const CauchyProblem &P, cudaStream_t s) {
    DevBuf<unsigned long long> cnt(3, s);
    cnt.zero(s);
    unsigned long long *c = cnt.get();
    const EvalCounts ec{T.srcse.get(), T.trgse.get(), P.sset.pgh, P.tset.pgh};
    const int *lev = T.level.get(), *n1 = T.nlist1.get(), *l1 = T.list1.get(),
              *n2 = T.nlist2.get();
    const int2 *sse = T.srcse.get(), *tse = T.trgse.get();
    const int spgh = P.sset.pgh, tpgh = P.tset.pgh;
    for_each(T.nboxes, s, [=] __device__(int64_t i) {
        const int b = (int)i;
        if (lev[b] >= 2 && ec.npts(b) > 0 && n2[b] > 0)
            atomicAdd(&c[0], (unsigned long long)n2[b]);
        if (n1[b] > 0) {
            unsigned long long ns_ = 0;
            for (int e = 0; e < n1[b]; e++) ns_ += count(sse, l1[kMaxList1 * b + e]);
            if (spgh > 0) atomicAdd(&c[1], ns_ * (unsigned long long)count(sse, b));
            if (tpgh > 0) atomicAdd(&c[2], ns_ * (unsigned long long)count(tse, b));
        }
    });
    unsigned long long h[3];
    FMM_CUDA(cudaMemcpyAsync(h, c, sizeof(h), cudaMemcpyDeviceToHost, s));
    FMM_CUDA(cudaStreamSynchronize(s));
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

void cauchy_fmm(const Tree &T, const CauchyProblem &P, cudaStream_t s) {
    if (profiling_enabled()) count_work(T, P, s);
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
    if (simple || !m2l_tensor_fp64(T, P, mp.get(), loc.get(), s))
        per_chunk([&](int c0) { m2l_chunk<2>(T, P, c0, binom, mp.get(), loc.get(), s); },
                  [&](int c0) { m2l_chunk<1>(T, P, c0, binom, mp.get(), loc.get(), s); });
    prof_mark("m2l", s);
    per_chunk([&](int c0) { downward_chunk<2>(T, P, c0, binom, mp.get(), loc.get(), s); },
              [&](int c0) { downward_chunk<1>(T, P, c0, binom, mp.get(), loc.get(), s); });
}

void cauchy_direct(const CauchyProblem &P, int ns, PointSet set,
                   cudaStream_t s) {
    (void)P; (void)ns; (void)set; (void)s;
    throw FmmError(4, "cauchy_direct: not implemented");
}

}  // namespace fmm2d
