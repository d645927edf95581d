// m2l_window.cu -- M2L of the mixed mode over runs of same-row boxes, on
// the tcgen05 tensor cores with shifted shared-memory windows.
//
// The list-2 sources of a box at level l are the children of its parent's
// colleagues that do not touch it (c_translation/src/tree_routs2d.c,
// computelists).  Take a run of TB consecutive parent boxes of one row of
// level l-1 (grid columns i0 .. i0+TB-1, row Y) and all their children:
// the sources of every child lie among the children of the parents in rows
// Y-1..Y+1, columns i0-1 .. i0+TB.  Split those by child row (6 rows of
// level l: 2Y-2 .. 2Y+3) and column parity (2): 12 "stages".  In stage
// (row y', parity q') the source seen by the child at parent column i0+t
// and child position c = (px, py) through shift jj in {-1, 0, 1} is the
// child of parent column i0+t+jj, at lattice offset
//     dx = 2 jj + q' - px,   dy = y' - 2Y - py,
// and it belongs to list 2 unless |dx| <= 1 and |dy| <= 1.  Every list-2
// pair of the run is exactly one (stage, jj, c) triple, 27 per child.
//
// So the window of a stage -- the stage's source multipoles in parent
// column order, CH channels per column -- is the A operand of an MMA whose
// 128 rows are (parent t, channel); shifting the operand's shared-memory
// descriptor by (jj + 1) * CH rows presents to row (t, ch) the source at
// column i0+t+jj.  The B operand stacks, along N, the real-form shift
// matrices of the four child positions for that (stage, jj): N = 4 x 2P'
// (P' = HALF >= p + 1), with zero blocks where the offset is not in list
// 2.  One run is 36 (stage, shift) steps of 2P'/8 x 3 MMAs (3 x TF32:
// x = hi + lo, D += A_hi B_hi + A_hi B_lo + A_lo B_hi) accumulated in
// tensor memory: D[(t, ch)][(c, output)] holds the locals of all 4 TB
// children of the run.
//
// With t = dx + i dy, the scaled shift of the reference (l2dmploc,
// c_translation/src/laprouts2d.c:886-994) factors as
//     T_ij = (-1)^j C(i+j-1, j-1) t^-(i+j) = a_i h_{i+j}(t) b_j,
// a_i = 1/i!, b_0 = -1, b_j = (-1)^j / (j-1)!, h_k(t) = (k-1)! t^-k, and
// T_0j = h_j b_j for j >= 1.  The window holds b_j M_j, the epilogue
// multiplies row i by a_i, so the B operand is the Hankel matrix h_{i+j}
// of each offset: a copy out of a 40-offset table already split into TF32
// hi / lo.  Row 0 (L_0, whose terms cancel across slots and reach the
// potential undamped) is summed on the CUDA cores in FP32 from the same
// windows, and the level's log(r) M_0 term is added in FP64, as in the
// slot-table kernels; from order kM2LExactFrom on so are rows 1-3 (1-5
// with Hessians), which carry most of the gradient at a leaf's points and
// need FP32's 24 bits rather than the 22 of a TF32 x 3 product.  The
// window's lo plane holds the exact FP32 residual v - hi, so hi + lo gives
// back the FP32 window value for those sums.
//
// Warp roles (416 threads, one block per SM): warps 0-7 convert the
// windows (FP32 multipoles -> b_j-scaled TF32 hi/lo in the operand
// layout) and copy the shift matrices; warp 12 issues the MMAs; warps
// 8-11, one thread per accumulator row, sum the leading rows from each
// window and at the end of a run read the accumulators back and store the
// locals.
// Windows, matrices and accumulators are double-buffered and handed over
// with mbarriers; every wait is bounded in time and a wait that runs out
// stops all roles of the block and sets *err.
#include "laplace.cuh"
#include "sort.cuh"
#include "tc_common.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <stdlib.h>
#include <string.h>
#include <vector>

namespace fmm2d {
namespace {

constexpr int kWinRows = 136;         // window rows: (TB + 2) x CH = 132 or 130, padded to 8
constexpr int kWinWorkers = 256;      // warps 0-7
constexpr int kWinEpi0 = 8;           // warps 8-11 read the accumulators
constexpr int kWinThreads = 13 * 32;  // warp 12 issues the MMAs
constexpr int kWinMaxParentLevel = 28;
constexpr uint64_t kWinWaitNs = 2000000000ull;
constexpr int kWinOffsets = 40;       // [-3, 3]^2 minus the 3 x 3 block

// Index in 0..39 of a lattice offset with |dx| >= 2 or |dy| >= 2.
__host__ __device__ __forceinline__ int win_offset_index(int dx, int dy) {
    const int row = dy + 3, col = dx + 3;
    int before = 0;
    if (row > 4)
        before = 9;
    else if (row >= 2)
        before = (row - 2) * 3 + (col > 4 ? 3 : (col >= 2 ? col - 2 : 0));
    return row * 7 + col - before;
}

// Offset of the source seen by child position c in stage s through shift
// jj; true when the pair is in list 2.
__host__ __device__ __forceinline__ bool win_slot(int s, int jj, int c, int &dx, int &dy) {
    const int r = (s >> 1) - 2, q = s & 1;
    dx = 2 * jj + q - (c & 1);
    dy = r - (c >> 1);
    return dx < -1 || dx > 1 || dy < -1 || dy > 1;
}

struct WinArgs {
    const int *wbox;   // [run][12][TB + 2] source box of each window column (-1: none)
    const int *tbox;   // [run][4][TB] target box per child position and column (-1: none)
    const int *rlev;   // [run] level of the targets
    int run0, nrun;
    const double *bs;  // box size per level
    int ndc, c0, p;
    const float *Bimg;  // [12 stages][3 shifts][hi | lo] the B operands in the operand layout
    const float *Bj;   // [HALF] b_j
    const double *Ai;  // [HALF] a_i = 1 / i!
    const float2 *Hf;  // [40][2 HALF] h_k(t) in FP32, with -log|t| at k = 0 (the rows
                       // summed on the CUDA cores over the window values)
    const float2 *mp32;
    double2 *loc;
    int *err;
    int stall;                   // fault injection: the issuer issues nothing
    unsigned long long wait_ns;  // limit of every bounded wait of the roles
};

// Packed FP32 FMA (two lanes per instruction): d = a * b + c per lane,
// round to nearest like fmaf.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    const uint64_t ua = (uint64_t)__float_as_uint(a.x) | ((uint64_t)__float_as_uint(a.y) << 32);
    const uint64_t ub = (uint64_t)__float_as_uint(b.x) | ((uint64_t)__float_as_uint(b.y) << 32);
    const uint64_t uc = (uint64_t)__float_as_uint(c.x) | ((uint64_t)__float_as_uint(c.y) << 32);
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(ua), "l"(ub), "l"(uc));
    return make_float2(__uint_as_float((uint32_t)d), __uint_as_float((uint32_t)(d >> 32)));
}

// Window values: hi = tf32(v) and lo = v - hi, the exact FP32 residual, so
// that hi + lo gives back v for the rows summed on the CUDA cores (the MMA
// reads lo at TF32 precision).
__device__ __forceinline__ void split_exact(float v, float &hi, float &lo) {
    hi = tc_tf32(v);
    lo = v - hi;
}

__device__ __forceinline__ void put4(float *hi, float *lo, int f, float a, float b, float c,
                                     float d) {
    float4 h, l;
    split_exact(a, h.x, l.x);
    split_exact(b, h.y, l.y);
    split_exact(c, h.z, l.z);
    split_exact(d, h.w, l.w);
    *reinterpret_cast<float4 *>(hi + f) = h;
    *reinterpret_cast<float4 *>(lo + f) = l;
}

// NR: the leading rows L_0 .. L_(NR-1) summed in FP32 on the CUDA cores by
// the epilogue warps (1: row 0 only).
template <int CH, int HALF, int NR>
__global__ void __launch_bounds__(kWinThreads, 1) m2l_win_kernel(WinArgs A) {
    constexpr int KP = 2 * HALF, NQ = HALF / 4, NOP = 4 * KP;
    constexpr int TB = 128 / CH, WP = TB + 2;
    constexpr int WSZ = kWinRows * KP, OSZ = NOP * KP, KH = 2 * HALF;
    constexpr int TCOLS = 2 * NOP <= 256 ? 256 : 512;
    constexpr uint32_t LBO_W = (kWinRows / 8) * 128, LBO_O = (NOP / 8) * 128, SBO = 128;
    constexpr uint32_t IDESC = tc_idesc_tf32(128, NOP);
    static_assert(WP * CH <= kWinRows, "window rows");
    static_assert(HALF % 4 == 0 && NOP % 16 == 0 && NOP <= 256, "operand shape");
    extern __shared__ __align__(1024) unsigned char win_smem[];
    float *sW = reinterpret_cast<float *>(win_smem);                 // [buf][hi, lo]
    float *sO = sW + 4 * WSZ;                                         // [buf][hi, lo]
    // h_k(t) expanded for the packed FP32 pipe: (Re, Re, -Im, Im)
    float4 *sHf = reinterpret_cast<float4 *>(sO + 4 * OSZ);           // [40][KH]
    double *sAi = reinterpret_cast<double *>(sHf + kWinOffsets * KH);  // [HALF]
    float *sBj = reinterpret_cast<float *>(sAi + HALF);               // [HALF]
    // barriers: 0-1 window full, 2-3 window free of MMAs, 4-5 window free
    // of row-0 reads, 6-7 matrices full, 8-9 matrices free, 10-11
    // accumulator full, 12-13 accumulator free, 14 final
    __shared__ __align__(8) uint64_t s_bar[15];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    volatile int *abort_flag = &s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t bar0 = smem_u32(&s_bar[0]);
#define WBAR(i) (bar0 + 8u * (uint32_t)(i))
    if (tid == 0) {
        for (int i = 0; i < 2; i++) {
            mbar_init(WBAR(0 + i), kWinWorkers);
            mbar_init(WBAR(2 + i), 1);
            mbar_init(WBAR(4 + i), 128);
            mbar_init(WBAR(6 + i), 1);  // (with the bulk copy's bytes)
            mbar_init(WBAR(8 + i), 1);
            mbar_init(WBAR(10 + i), 1);
            mbar_init(WBAR(12 + i), 128);
        }
        mbar_init(WBAR(14), 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int e = tid; e < kWinOffsets * KH; e += blockDim.x) {
        const float2 t = A.Hf[e];
        sHf[e] = make_float4(t.x, t.x, -t.y, t.y);
    }
    for (int e = tid; e < HALF; e += blockDim.x) {
        sAi[e] = A.Ai[e];
        sBj[e] = A.Bj[e];
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&s_tmem)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const int P = A.p + 1, stride = P * A.ndc;

    if (warp < kWinEpi0) {
        // ------------------------------------------------------------ workers
        const int wt = tid;
        constexpr int NTW = (WP * NQ + kWinWorkers - 1) / kWinWorkers;
        float2 pre[NTW][4][CH];
        // two channels of a box stored side by side at a 16-byte boundary
        const bool pair4 = A.ndc == 2 && A.c0 == 0 && (stride % 2) == 0;
        // the stage's window: column ps (fastest over threads), K chunk jq
        auto prefetch = [&](int run, int s) {
            const int *wrow = A.wbox + ((size_t)run * 12 + s) * WP;
#pragma unroll
            for (int a = 0; a < NTW; a++) {
                const int tau = wt + a * kWinWorkers;
                const int ps = tau % WP, jq = tau / WP;
                const int box = tau < WP * NQ ? __ldg(wrow + ps) : -1;
                const float2 *m = A.mp32 + (size_t)(box >= 0 ? box : 0) * stride + A.c0;
                if (CH == 2 && pair4) {
                    // both channels of coefficient j in one 16-byte load
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const int j = jq * 4 + e;
                        const float4 v = (box >= 0 && j < P)
                                             ? __ldg(reinterpret_cast<const float4 *>(m + (size_t)j * 2))
                                             : make_float4(0.f, 0.f, 0.f, 0.f);
                        pre[a][e][0] = make_float2(v.x, v.y);
                        pre[a][e][CH - 1] = make_float2(v.z, v.w);
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const int j = jq * 4 + e;
#pragma unroll
                        for (int c = 0; c < CH; c++)
                            pre[a][e][c] = (box >= 0 && j < P) ? __ldg(m + (size_t)j * A.ndc + c)
                                                               : make_float2(0.f, 0.f);
                    }
                }
            }
        };
        // window rows (ps, ch): [b_j Re M_j | b_j Im M_j], TF32 hi / lo
        auto store_window = [&](float *Whi, float *Wlo) {
#pragma unroll
            for (int a = 0; a < NTW; a++) {
                const int tau = wt + a * kWinWorkers;
                if (tau >= WP * NQ) continue;
                const int ps = tau % WP, jq = tau / WP;
                const float b0 = sBj[4 * jq], b1 = sBj[4 * jq + 1], b2 = sBj[4 * jq + 2],
                            b3 = sBj[4 * jq + 3];
#pragma unroll
                for (int c = 0; c < CH; c++) {
                    const int row = ps * CH + c;
                    put4(Whi, Wlo, tc_fidx(row, 4 * jq, kWinRows), b0 * pre[a][0][c].x,
                         b1 * pre[a][1][c].x, b2 * pre[a][2][c].x, b3 * pre[a][3][c].x);
                    put4(Whi, Wlo, tc_fidx(row, HALF + 4 * jq, kWinRows), b0 * pre[a][0][c].y,
                         b1 * pre[a][1][c].y, b2 * pre[a][2][c].y, b3 * pre[a][3][c].y);
                }
            }
        };
        int g = 0, u = 0;
        bool ok = true;
        if ((int)blockIdx.x < A.nrun) prefetch(A.run0 + blockIdx.x, 0);
        for (int run = blockIdx.x; ok && run < A.nrun; run += gridDim.x) {
            const int R = A.run0 + run;
            for (int s = 0; ok && s < 12; s++, g++) {
                const int b = g & 1;
                float *Whi = sW + (2 * b) * WSZ, *Wlo = Whi + WSZ;
                if (g >= 2) {
                    const uint32_t par = (uint32_t)(((g >> 1) - 1) & 1);
                    if (!mbar_wait_bounded(WBAR(2 + b), par, abort_flag, A.wait_ns) ||
                        !mbar_wait_bounded(WBAR(4 + b), par, abort_flag, A.wait_ns)) {
                        ok = false;
                        break;
                    }
                }
                store_window(Whi, Wlo);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive(WBAR(0 + b));
                // the next stage's inputs
                if (s < 11)
                    prefetch(R, s + 1);
                else if (run + (int)gridDim.x < A.nrun)
                    prefetch(R + gridDim.x, 0);
                // the stage's three B operands: bulk copies of the
                // precomputed images, each into the matrix buffer the MMAs
                // of two steps ago have released
                if (wt == 0) {
                    for (int j = 0; j < 3; j++, u++) {
                        const int ob = u & 1;
                        if (u >= 2 && !mbar_wait_bounded(WBAR(8 + ob), (uint32_t)(((u >> 1) - 1) & 1),
                                                         abort_flag, A.wait_ns)) {
                            ok = false;
                            break;
                        }
                        mbar_arrive_expect_tx(WBAR(6 + ob), 2u * OSZ * 4u);
                        bulk_g2s(smem_u32(sO + (2 * ob) * OSZ), A.Bimg + (size_t)(s * 3 + j) * 2 * OSZ,
                                 2u * OSZ * 4u, WBAR(6 + ob));
                    }
                }
            }
        }
        if (wt == 0) {
            // the last bulk copies have landed before the block exits (the
            // issuer has waited for them unless the block stopped early)
            int never = 0;
            for (int t = u - 2; t < u; t++)
                if (t >= 0) mbar_wait_bounded(WBAR(6 + (t & 1)), (uint32_t)((t >> 1) & 1), &never, kWinWaitNs);
        }
        if (!ok) *abort_flag = 1;
    } else if (warp < kWinEpi0 + 4) {
        // ------------------------------------- leading rows and epilogue
        // thread = accumulator row (t, ch) for all four child positions
        const int e = warp - kWinEpi0;  // tensor-memory lanes 32 e .. 32 e + 31
        const int rho = (e << 5) + lane, tcol = rho / CH, chn = rho - tcol * CH;
        int g = 0, kr = 0;
        bool ok = true;
        for (int run = blockIdx.x; ok && run < A.nrun; run += gridDim.x, kr++) {
            const int R = A.run0 + run;
            // L_i = a_i sum_slots sum_j h_(i+j)(t) W_j (i = 1 .. NR-1) and
            // L_0 = sum_slots (sum_(j>=1) h_j(t) W_j - log|t| W_0) in FP32
            // from the windows (window value W_j = b_j M_j, W_0 = -M_0)
            float2 lr_[4][NR], s0[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                s0[c] = make_float2(0.f, 0.f);
#pragma unroll
                for (int i = 0; i < NR; i++) lr_[c][i] = make_float2(0.f, 0.f);
            }
            for (int s = 0; ok && s < 12; s++, g++) {
                const int b = g & 1;
                if (!mbar_wait_bounded(WBAR(0 + b), (uint32_t)((g >> 1) & 1), abort_flag, A.wait_ns)) {
                    ok = false;
                    break;
                }
                const float *Whi = sW + (2 * b) * WSZ, *Wlo = Whi + WSZ;
#pragma unroll 1
                for (int j = 0; j < 3; j++) {
                    int dxs[4], dys[4];
                    bool v[4];
                    bool any = false;
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        v[c] = win_slot(s, j - 1, c, dxs[c], dys[c]);
                        any = any || v[c];
                    }
                    if (!any) continue;
                    const int row = rho + j * CH;
                    float mr[HALF], mi[HALF];
#pragma unroll
                    for (int q = 0; q < NQ; q++) {
                        const int fr = tc_fidx(row, 4 * q, kWinRows), fi = tc_fidx(row, HALF + 4 * q, kWinRows);
                        const float4 h1 = *reinterpret_cast<const float4 *>(Whi + fr);
                        const float4 l1 = *reinterpret_cast<const float4 *>(Wlo + fr);
                        const float4 h2 = *reinterpret_cast<const float4 *>(Whi + fi);
                        const float4 l2 = *reinterpret_cast<const float4 *>(Wlo + fi);
                        mr[4 * q + 0] = h1.x + l1.x;
                        mr[4 * q + 1] = h1.y + l1.y;
                        mr[4 * q + 2] = h1.z + l1.z;
                        mr[4 * q + 3] = h1.w + l1.w;
                        mi[4 * q + 0] = h2.x + l2.x;
                        mi[4 * q + 1] = h2.y + l2.y;
                        mi[4 * q + 2] = h2.z + l2.z;
                        mi[4 * q + 3] = h2.w + l2.w;
                    }
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        if (!v[c]) continue;
                        // (window values beyond the order are zero)
                        // acc_i += h_(i+jp) W_jp for the NR rows at once: the
                        // table entries h_jp .. h_(jp+NR-1) rotate through
                        // registers, one load per jp; each complex update is
                        // two packed FMAs, (Re, Im) += (-Im h, Im h) (Im W,
                        // Re W) then += (Re h, Re h) (Re W, Im W) -- the same
                        // operations in the same order as scalar FMAs
                        const float4 *hf = sHf + win_offset_index(dxs[c], dys[c]) * KH;
                        float4 w[NR];
#pragma unroll
                        for (int q = 0; q + 1 < NR; q++) w[q] = hf[q];
#pragma unroll
                        for (int jp = 0; jp < HALF; jp++) {
                            w[NR - 1] = hf[jp + NR - 1];
                            const float2 MI = make_float2(mi[jp], mr[jp]);
                            const float2 MR = make_float2(mr[jp], mi[jp]);
#pragma unroll
                            for (int i = 0; i < NR; i++) {
                                lr_[c][i] = fma2(make_float2(w[i].z, w[i].w), MI, lr_[c][i]);
                                lr_[c][i] = fma2(make_float2(w[i].x, w[i].y), MR, lr_[c][i]);
                            }
#pragma unroll
                            for (int q = 0; q + 1 < NR; q++) w[q] = w[q + 1];
                        }
                        s0[c].x -= mr[0];  // M_0 = -W_0
                        s0[c].y -= mi[0];
                    }
                }
                mbar_arrive(WBAR(4 + b));
            }
            if (!ok) break;
            // locals of the run's targets: L_0 + log(r) sum M_0 (FP64), a_i D_i
            const int b = kr & 1;
            // (tcgen05.ld is warp-collective: the warp decides as one)
            const bool got =
                mbar_wait_backoff(WBAR(10 + b), (uint32_t)((kr >> 1) & 1), abort_flag, A.wait_ns);
            if (!__all_sync(0xffffffffu, got)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t taddr = tmem + ((uint32_t)(e << 5) << 16) + (uint32_t)(b * (TCOLS / 2));
            const double lr = log(A.bs[A.rlev[R]]);
#pragma unroll 1
            for (int c = 0; c < 4; c++) {
                float d[KP];
#pragma unroll
                for (int q = 0; q < KP / 8; q++) {
                    float vv[8];
                    tc_ld8(taddr + (uint32_t)(c * KP + 8 * q), vv);
#pragma unroll
                    for (int i = 0; i < 8; i++) d[8 * q + i] = vv[i];
                }
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int box = A.tbox[((size_t)R * 4 + c) * TB + tcol];
                if (box >= 0) {
                    double2 *o = A.loc + (size_t)box * stride + A.c0 + chn;
                    o[0] = make_double2((double)lr_[c][0].x + lr * (double)s0[c].x,
                                        (double)lr_[c][0].y + lr * (double)s0[c].y);
#pragma unroll
                    for (int i = 1; i < HALF; i++)
                        if (i < P) {
                            const double re = i < NR ? (double)lr_[c][i < NR ? i : 0].x : (double)d[i];
                            const double im = i < NR ? (double)lr_[c][i < NR ? i : 0].y : (double)d[HALF + i];
                            o[(size_t)i * A.ndc] = make_double2(sAi[i] * re, sAi[i] * im);
                        }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(WBAR(12 + b));
        }
        if (!ok) *abort_flag = 1;
    } else {
        // ------------------------------------------------------------ issuer
        int g = 0, u = 0, kr = 0;
        bool ok = true, issued = false;
        // (fault injection: nothing is issued or committed, so the other
        // roles' bounded waits run out)
        for (int run = blockIdx.x; ok && !A.stall && run < A.nrun; run += gridDim.x, kr++) {
            const int b = kr & 1;
            const bool freed = kr < 2 || mbar_wait_bounded(WBAR(12 + b), (uint32_t)(((kr >> 1) - 1) & 1),
                                                           abort_flag, A.wait_ns);
            if (!__all_sync(0xffffffffu, freed)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t dt = tmem + (uint32_t)(b * (TCOLS / 2));
            uint32_t acc = 0u;
            for (int s = 0; ok && s < 12; s++, g++) {
                const int wb = g & 1;
                if (!__all_sync(0xffffffffu, mbar_wait_bounded(WBAR(0 + wb), (uint32_t)((g >> 1) & 1),
                                                               abort_flag, A.wait_ns))) {
                    ok = false;
                    break;
                }
                const uint32_t whi = smem_u32(sW + (2 * wb) * WSZ), wlo = whi + WSZ * 4;
                for (int j = 0; j < 3; j++, u++) {
                    const int ob = u & 1;
                    if (!__all_sync(0xffffffffu, mbar_wait_bounded(WBAR(6 + ob), (uint32_t)((u >> 1) & 1),
                                                                   abort_flag, A.wait_ns))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    if (lane == 0) {
                        const uint32_t ohi = smem_u32(sO + (2 * ob) * OSZ), olo = ohi + OSZ * 4;
                        const uint32_t sh = (uint32_t)(j * CH * 16);  // (jj + 1) CH rows
#pragma unroll
                        for (int ks = 0; ks < KP / 8; ks++) {
                            const uint32_t ao = sh + 2u * ks * LBO_W, bo = 2u * ks * LBO_O;
                            tc_mma(dt, tc_sdesc(whi + ao, LBO_W, SBO), tc_sdesc(ohi + bo, LBO_O, SBO),
                                   IDESC, acc);
                            tc_mma(dt, tc_sdesc(whi + ao, LBO_W, SBO), tc_sdesc(olo + bo, LBO_O, SBO),
                                   IDESC, 1u);
                            tc_mma(dt, tc_sdesc(wlo + ao, LBO_W, SBO), tc_sdesc(ohi + bo, LBO_O, SBO),
                                   IDESC, 1u);
                            acc = 1u;
                        }
                        tc_commit(WBAR(8 + ob));
                    }
                    __syncwarp();
                    issued = true;
                }
                if (!ok) break;
                if (lane == 0) tc_commit(WBAR(2 + wb));
                __syncwarp();
            }
            if (!ok) break;
            if (lane == 0) tc_commit(WBAR(10 + b));
            __syncwarp();
        }
        if (!ok) *abort_flag = 1;
        // the MMAs still in flight finish before the tensor memory is freed
        if (issued && lane == 0) {
            int never = 0;
            tc_commit(WBAR(14));
            mbar_wait_bounded(WBAR(14), 0u, &never, kWinWaitNs);
        }
        __syncwarp();
    }
#undef WBAR
    __syncthreads();
    if (tid == 0 && s_abort) atomicExch(A.err, 1);
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS)
                     : "memory");
    }
}

template <int CH, int HALF>
constexpr size_t win_smem_bytes() {
    return (size_t)(4 * kWinRows * 2 * HALF + 4 * 8 * HALF * 2 * HALF) * sizeof(float) +
           (size_t)kWinOffsets * 2 * HALF * sizeof(float4) + (size_t)HALF * sizeof(double) +
           (size_t)HALF * sizeof(float);
}

// Tables of one (order, HALF): the B operand of every (stage, shift) step
// -- the real form of the Hankel matrices h_(i+j)(t) of the four child
// positions' offsets, rows i >= 1 (zero outside list 2 and beyond the
// order), TF32 hi then lo, in the operand layout --, h_k(t) in FP32 with
// -log|t| at k = 0 (the leading rows over the window values), b_j and a_i;
// cached per device.
struct WinTables {
    const float *Bimg = nullptr;  // [12][3][hi | lo][4 * 2 HALF * 2 HALF]
    const float2 *Hf = nullptr;
    const float *Bj = nullptr;
    const double *Ai = nullptr;
};

float tf32_host(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

// TF32 hi / lo of v: hi = tf32(v), lo = tf32(v - hi)
inline float2 tf32_split_host(double v) {
    const float h = tf32_host((float)v);
    return make_float2(h, tf32_host((float)(v - (double)h)));
}

WinTables win_tables(int p, int HALF, cudaStream_t s) {
    static std::mutex mu;
    static std::vector<std::pair<long, WinTables>> cache;
    int dev;
    FMM_CUDA(cudaGetDevice(&dev));
    const long key = ((long)dev << 20) | ((long)p << 8) | HALF;
    std::lock_guard<std::mutex> g(mu);
    for (auto &e : cache)
        if (e.first == key) return e.second;
    const int KH = 2 * HALF;
    std::vector<float4> H((size_t)kWinOffsets * KH, make_float4(0.f, 0.f, 0.f, 0.f));
    std::vector<float2> Hf((size_t)kWinOffsets * KH, make_float2(0.f, 0.f));
    for (int dy = -3; dy <= 3; dy++)
        for (int dx = -3; dx <= 3; dx++) {
            if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1) continue;
            const int o = win_offset_index(dx, dy);
            float4 *row = H.data() + (size_t)o * KH;
            float2 *hf = Hf.data() + (size_t)o * KH;
            hf[0] = make_float2((float)(-0.5 * std::log((double)(dx * dx + dy * dy))), 0.f);
            // h_1 = 1/t, h_{k+1} = h_k k / t
            const double2 ti = cinv(make_double2(dx, dy));
            double2 h = ti;
            for (int k = 1; k < KH; k++) {
                const float2 re = tf32_split_host(h.x), im = tf32_split_host(h.y);
                row[k] = make_float4(re.x, re.y, im.x, im.y);
                hf[k] = make_float2((float)h.x, (float)h.y);
                h = cscal(cmul(h, ti), (double)k);
            }
        }
    std::vector<float> Bj(HALF, 0.f);
    std::vector<double> Ai(HALF, 0.0);
    double fact = 1.0;  // (j - 1)! for j >= 1
    for (int j = 0; j < HALF; j++) {
        if (j == 0)
            Bj[j] = -1.f;
        else {
            if (j >= 2) fact *= (double)(j - 1);
            Bj[j] = (float)(((j & 1) ? -1.0 : 1.0) / fact);
        }
    }
    double fi = 1.0;
    for (int i = 0; i < HALF; i++) {
        if (i >= 1) fi *= (double)i;
        Ai[i] = 1.0 / fi;
    }
    // the B operands of the 36 steps (the layout the MMA reads: N = 4 KP
    // rows -- child position c, then [Re outputs | Im outputs] --, K = KP)
    const int KP = 2 * HALF, NOP = 4 * KP, NQ = HALF / 4, OSZ = NOP * KP;
    std::vector<float> img((size_t)36 * 2 * OSZ, 0.f);
    for (int st = 0; st < 12; st++)
        for (int j = 0; j < 3; j++) {
            float *Ohi = img.data() + (size_t)(st * 3 + j) * 2 * OSZ, *Olo = Ohi + OSZ;
            for (int c = 0; c < 4; c++) {
                int dx, dy;
                const bool in2 = win_slot(st, j - 1, c, dx, dy);
                for (int jq = 0; jq < NQ; jq++)
                    for (int i = 0; i < HALF; i++) {
                        float4 h[4];
                        for (int e = 0; e < 4; e++) h[e] = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (in2 && i >= 1 && i <= p) {
                            const float4 *hrow = H.data() + (size_t)win_offset_index(dx, dy) * KH + i + 4 * jq;
                            for (int e = 0; e < 4; e++)
                                if (4 * jq + e <= p) h[e] = hrow[e];
                        }
                        const int nre = c * KP + i, nim = nre + HALF;
                        const int f1 = tc_fidx(nre, 4 * jq, NOP), f2 = tc_fidx(nre, HALF + 4 * jq, NOP);
                        const int f3 = tc_fidx(nim, 4 * jq, NOP), f4 = tc_fidx(nim, HALF + 4 * jq, NOP);
                        for (int e = 0; e < 4; e++) {
                            Ohi[f1 + e] = h[e].x;   // Re h
                            Olo[f1 + e] = h[e].y;
                            Ohi[f2 + e] = -h[e].z;  // -Im h
                            Olo[f2 + e] = -h[e].w;
                            Ohi[f3 + e] = h[e].z;   // Im h
                            Olo[f3 + e] = h[e].w;
                            Ohi[f4 + e] = h[e].x;   // Re h
                            Olo[f4 + e] = h[e].y;
                        }
                    }
            }
        }
    WinTables t;
    float *dH = nullptr;
    float2 *dR = nullptr;
    float *dB = nullptr;
    double *dA = nullptr;
    FMM_CUDA(cudaMalloc(&dH, img.size() * sizeof(float)));
    FMM_CUDA(cudaMalloc(&dR, Hf.size() * sizeof(float2)));
    FMM_CUDA(cudaMalloc(&dB, Bj.size() * sizeof(float)));
    FMM_CUDA(cudaMalloc(&dA, Ai.size() * sizeof(double)));
    FMM_CUDA(cudaMemcpyAsync(dH, img.data(), img.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaMemcpyAsync(dR, Hf.data(), Hf.size() * sizeof(float2), cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaMemcpyAsync(dB, Bj.data(), Bj.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaMemcpyAsync(dA, Ai.data(), Ai.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaStreamSynchronize(s));
    t.Bimg = dH;
    t.Hf = dR;
    t.Bj = dB;
    t.Ai = dA;
    cache.push_back({key, t});
    return t;
}

// Runs of one evaluation: the parents of the targets, grouped by (level,
// row, column / TB) with a 64-bit key sorted in two stable 32-bit passes.
struct WinPlan {
    DevBuf<int> wbox, tbox, rlev;
    std::vector<std::pair<int, int>> ranges;  // [first run, count) per launch
    uint64_t levels = 0;                      // target levels covered
};

// the reference's "npts" of a box for the M2L step (points of the sets
// that are evaluated)
struct WinCounts {
    const int2 *sse, *tse;
    int spgh, tpgh;
    __device__ __forceinline__ int operator()(int b) const {
        int n = 0;
        if (tpgh > 0) n += tse[b].y - tse[b].x;
        if (spgh > 0) n += sse[b].y - sse[b].x;
        return n;
    }
};

bool win_plan(const Tree &T, const CauchyProblem &P, int CH, cudaStream_t s, WinPlan &W) {
    const int L = T.nlevels;
    if (L < 2 || L - 1 > kWinMaxParentLevel) return false;
    const int TB = 128 / CH, WP = TB + 2;
    const int nb = T.nboxes, lo1 = T.lstart[1], lo2 = T.lstart[2];
    const int npar = T.lend[L - 1] - lo1;
    if (npar <= 0) return false;
    const int2 *sse = T.srcse.get(), *tse = T.trgse.get();
    const int spgh = P.sset.pgh, tpgh = P.tset.pgh;
    const int *lev = T.level.get(), *par = T.parent.get(), *chi = T.child.get();
    const int *nnb = T.nnbors.get(), *nbr = T.nbors.get();
    const double2 *cen = T.centers.get();
    const double *bsd = T.d_boxsize.get();
    const WinCounts npts{sse, tse, spgh, tpgh};
    // parents of the boxes that receive an M2L
    DevBuf<int> flag(npar, s), pos(npar, s), total(1, s);
    flag.zero(s);
    {
        int *fl = flag.get();
        for_each(nb - lo2, s, [=] __device__(int64_t i) {
            const int b = lo2 + (int)i;
            if (npts(b) > 0) fl[par[b] - lo1] = 1;
        });
    }
    exclusive_scan_i32(flag.get(), pos.get(), npar, total.get(), s);
    const int m = read_scalar(total.get(), s);
    if (m == 0) return true;
    DevBuf<uint32_t> klo(m, s), khi(m, s), k0(m, s), k1(m, s), idx(m, s), ktmp(m, s), vtmp(m, s);
    DevBuf<int> pbox(m, s);
    {
        const int *fl = flag.get(), *ps = pos.get();
        uint32_t *kl = klo.get(), *kh = khi.get(), *a0 = k0.get(), *a1 = k1.get(), *ix = idx.get();
        int *pb = pbox.get();
        const int tb = TB;
        for_each(npar, s, [=] __device__(int64_t i) {
            if (!fl[i]) return;
            const int q = ps[i], b = lo1 + (int)i, lp = lev[b];
            const double bsl = bsd[lp], half = 0.5 * (double)((1ll << lp) - 1);
            const double2 c = cen[b], c0 = cen[0];
            const long long X = llrint((c.x - c0.x) / bsl + half);
            const long long Y = llrint((c.y - c0.y) / bsl + half);
            const uint64_t key = ((uint64_t)lp << 58) | ((uint64_t)Y << 29) | (uint64_t)(X / tb);
            kl[q] = (uint32_t)key;
            kh[q] = (uint32_t)(key >> 32);
            a0[q] = (uint32_t)key;
            a1[q] = (uint32_t)(key >> 32);
            ix[q] = (uint32_t)q;
            pb[q] = b;
        });
    }
    radix_sort_pairs(klo.get(), idx.get(), ktmp.get(), vtmp.get(), m, 32, s);
    {
        const uint32_t *ix = idx.get(), *a1 = k1.get();
        uint32_t *kh = khi.get();
        for_each(m, s, [=] __device__(int64_t q) { kh[q] = a1[ix[q]]; });
    }
    radix_sort_pairs(khi.get(), idx.get(), ktmp.get(), vtmp.get(), m, 32, s);
    // runs: a new run where the key changes
    DevBuf<int> head(m, s), rid(m, s), nrun_d(1, s);
    {
        const uint32_t *ix = idx.get(), *a0 = k0.get(), *a1 = k1.get();
        int *hd = head.get();
        for_each(m, s, [=] __device__(int64_t q) {
            const uint32_t i = ix[q];
            int h = 1;
            if (q > 0) {
                const uint32_t j = ix[q - 1];
                h = (a0[i] != a0[j] || a1[i] != a1[j]) ? 1 : 0;
            }
            hd[q] = h;
        });
    }
    exclusive_scan_i32(head.get(), rid.get(), m, nrun_d.get(), s);
    const int nrun = read_scalar(nrun_d.get(), s);
    W.wbox.alloc((size_t)nrun * 12 * WP, s);
    W.tbox.alloc((size_t)nrun * 4 * TB, s);
    W.rlev.alloc(nrun, s);
    FMM_CUDA(cudaMemsetAsync(W.wbox.get(), 0xff, (size_t)nrun * 12 * WP * sizeof(int), s));
    FMM_CUDA(cudaMemsetAsync(W.tbox.get(), 0xff, (size_t)nrun * 4 * TB * sizeof(int), s));
    DevBuf<int> cnt(128, s);
    cnt.zero(s);
    {
        const uint32_t *ix = idx.get();
        const int *pb = pbox.get(), *hd = head.get(), *rd = rid.get();
        int *wb = W.wbox.get(), *tbx = W.tbox.get(), *rl = W.rlev.get(), *ct = cnt.get();
        const int tb = TB, wp = WP;
        for_each(m, s, [=] __device__(int64_t q) {
            const int b = pb[ix[q]], run = rd[q] + hd[q] - 1;
            const int lp = lev[b];
            const double bsl = bsd[lp], half = 0.5 * (double)((1ll << lp) - 1);
            const double2 cb = cen[b], c0 = cen[0];
            const long long X = llrint((cb.x - c0.x) / bsl + half);
            const int t = (int)(X % tb);
            if (hd[q]) rl[run] = lp + 1;
            int ntq = 0;
            for (int c = 0; c < 4; c++) {
                const int kb = chi[4 * b + c];
                if (kb >= 0 && npts(kb) > 0) {
                    tbx[((size_t)run * 4 + c) * tb + t] = kb;
                    ntq++;
                }
            }
            // runs and targets per level, one atomic per group of lanes
            // of the same level (consecutive parents share levels)
            const unsigned am = __activemask();
            const unsigned peers = __match_any_sync(am, lp);
            const int nr = __reduce_add_sync(peers, hd[q] ? 1 : 0);
            const int nt = __reduce_add_sync(peers, ntq);
            if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) {
                if (nr) atomicAdd(&ct[lp + 1], nr);
                if (nt) atomicAdd(&ct[64 + lp + 1], nt);
            }
            for (int k = 0; k < nnb[b]; k++) {
                const int cb2 = nbr[9 * b + k];
                const double2 cc = cen[cb2];
                const int dX = (int)rint((cc.x - cb.x) / bsl), dY = (int)rint((cc.y - cb.y) / bsl);
                if (dX < -1 || dX > 1 || dY < -1 || dY > 1) continue;
                for (int st = 0; st < 12; st++) {
                    const int r = (st >> 1) - 2;
                    if ((r >> 1) != dY) continue;
                    const int kb = chi[4 * cb2 + (st & 1) + 2 * (r & 1)];
                    if (kb >= 0 && sse[kb].y > sse[kb].x)
                        wb[((size_t)run * 12 + st) * wp + t + dX + 1] = kb;
                }
            }
        });
    }
    std::vector<int> hc(128);
    read_small(hc.data(), cnt.get(), 128 * sizeof(int), s);
    // a level goes through the windows when its runs are at least 1/8 full
    int start = 0, open = -1;
    for (int l = 0; l <= L + 1 && l < 64; l++) {
        const int nr = hc[l], nt = hc[64 + l];
        const bool win = l >= 2 && l <= L && nr > 0 && (long long)nt * 8 >= (long long)nr * 4 * TB;
        if (win) {
            W.levels |= 1ull << l;
            if (open < 0) open = start;
        } else if (open >= 0) {
            W.ranges.push_back({open, start - open});
            open = -1;
        }
        start += nr;
    }
    if (open >= 0) W.ranges.push_back({open, start - open});
    return true;
}

template <int CH, int HALF>
void launch_win(const WinPlan &W, const WinTables &tb, const Tree &T, const CauchyProblem &P,
                int c0, const float2 *mp32, double2 *loc, int *err, cudaStream_t s) {
    constexpr size_t sm = win_smem_bytes<CH, HALF>();
    // The tensor-core kernel's TF32 x 3 products hold 22 of FP32's 24 bits;
    // from order kM2LExactFrom on, the leading coefficients -- which carry
    // most of the gradient (and, with six, the Hessian) at a leaf's points
    // -- are summed in FP32 on the CUDA cores from the same windows instead
    // (row 0 always is: its terms cancel across the slots).
    const bool hess = std::max(P.sset.n > 0 ? P.sset.pgh : 0, P.tset.n > 0 ? P.tset.pgh : 0) >= 3;
    const int nr = !m2l_exact_rows(P.p) ? 1 : (hess ? kM2LExactRowsHess : kM2LExactRows);
    auto kern = nr == 1 ? m2l_win_kernel<CH, HALF, 1>
                        : (nr == kM2LExactRows ? m2l_win_kernel<CH, HALF, kM2LExactRows>
                                               : m2l_win_kernel<CH, HALF, kM2LExactRowsHess>);
    raise_smem_limit(kern, (int)sm);
    for (const auto &r : W.ranges) {
        WinArgs a;
        a.wbox = W.wbox.get();
        a.tbox = W.tbox.get();
        a.rlev = W.rlev.get();
        a.run0 = r.first;
        a.nrun = r.second;
        a.bs = T.d_boxsize.get();
        a.ndc = P.ndc;
        a.c0 = c0;
        a.p = P.p;
        a.Bimg = tb.Bimg;
        a.Bj = tb.Bj;
        a.Ai = tb.Ai;
        a.Hf = tb.Hf;
        a.mp32 = mp32;
        a.loc = loc;
        a.err = err;
        a.stall = tc_stall_injected();
        a.wait_ns = tc_wait_limit_ns();
        const int grid = std::max(1, std::min(r.second, kNumSM));
        kern<<<grid, kWinThreads, sm, s>>>(a);
        FMM_CHECK_LAUNCH();
    }
}

template <int HALF>
void run_win(const WinPlan &W, const WinTables &tb, int CH, const Tree &T,
             const CauchyProblem &P, const float2 *mp32, double2 *loc, int *err, cudaStream_t s) {
    for (int c0 = 0; c0 < P.ndc; c0 += CH) {
        if (CH == 2)
            launch_win<2, HALF>(W, tb, T, P, c0, mp32, loc, err, s);
        else
            launch_win<1, HALF>(W, tb, T, P, c0, mp32, loc, err, s);
    }
}

}  // namespace

uint64_t m2l_window_fp32(const Tree &T, const CauchyProblem &P, const float2 *mp32, double2 *loc,
                         int *err, cudaStream_t s) {
    const int HALF = P.p + 1 <= 12 ? 12 : (P.p + 1 <= 16 ? 16 : (P.p + 1 <= 20 ? 20 : 0));
    if (HALF == 0) return 0;
    // (the runs are found from box positions, which the trees of a forest
    // share: forests use the slot tables)
    if (T.nroots > 1) return 0;
    const int CH = P.ndc % 2 == 0 ? 2 : 1;
    bool ok = false;
    const auto Wp = m2l_cached<WinPlan>(P.m2l_cache, ((uint64_t)2 << 56) | (uint64_t)CH, ok,
                                        [&](WinPlan &x) { return win_plan(T, P, CH, s, x); });
    const WinPlan &W = *Wp;
    if (!ok || W.ranges.empty()) return 0;
    const WinTables tb = win_tables(P.p, HALF, s);
    int nrun = 0;
    for (const auto &r : W.ranges) nrun += r.second;
    prof_set_count("m2l_window_levels", (double)__builtin_popcountll(W.levels));
    prof_set_count("m2l_window_runs", (double)nrun);
    if (HALF == 12)
        run_win<12>(W, tb, CH, T, P, mp32, loc, err, s);
    else if (HALF == 16)
        run_win<16>(W, tb, CH, T, P, mp32, loc, err, s);
    else
        run_win<20>(W, tb, CH, T, P, mp32, loc, err, s);
    return W.levels;
}

}  // namespace fmm2d
