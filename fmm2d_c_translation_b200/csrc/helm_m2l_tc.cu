// helm_m2l_tc.cu -- M2L of the Helmholtz FMM in the mixed mode, as batched
// complex contractions on the tcgen05 tensor cores (kind::tf32, FP32
// accumulation in tensor memory).
//
// The reference's multipole-to-local shift (h2dmploc,
// c_translation/src/helmrouts2d.c:937-1042) between two boxes of level l
// (same scale rs) is
//     L_i += sum_j B_ij M_j,   B_ij = T(i - j) w_ij,
// with T(q) the scaled Hankel table of the offset (H_|q|(k|d|) rs^|q| times
// the phase e^{-i q theta}, shift_table in helmholtz.cu) and w_ij = 1 when
// i j <= 0, rs^(2 min(|i|, |j|)) otherwise.  B depends only on the level
// and the lattice offset between the two boxes, and a target box at child
// position c sees exactly 27 possible offsets (the slot tables of m2l.cu).
// So for one level, one child position and one slot, the M2L of all target
// boxes is one real GEMM:
//     D[row][n] += sum_k A[row][k] Bop[n][k],
// rows = (target box, channel), A[row] = [Re M_-p..p | Im M_-p..p] of the
// row's source box for that slot (K = 2(2p+1), zero padded), and Bop the
// real form [[Re B, -Im B], [Im B, Re B]] (N = 2(2p+1), zero padded).  The
// 27 slots of a tile of 128 rows accumulate in one tensor-memory tile.
//
// Precision: operands are split into TF32 hi + lo (x = hi + lo, about 22
// significant bits), D += A_hi B_hi + A_hi B_lo + A_lo B_hi; Bop is scaled by
// a power of two so that its largest entry is about 1, and the epilogue
// undoes the scale and adds to the FP64 local expansions.  Levels whose
// order exceeds 23 (K > 96) or whose tables leave the FP32 range keep the
// FP64 CUDA-core M2L.
//
// Pipeline (one block per SM, persistent over the level's tiles): the K
// dimension of each slot is cut into chunks of 16, and every (slot, chunk)
// step stages A (128 x 16, hi and lo: gathered with cp.async from
// operand-ready rows built once per level) and Bop (N x 16, hi and lo: a
// contiguous block of the per-level images, also cp.async) into one of
// kHtStages shared-memory stages.  Warps 0-3 (one thread per A row) fill
// the stages, keeping kHtLag groups of copies in flight; warp 8 issues
// 3 x 2 MMAs per step and commits the stage back.  Each slot accumulates
// in a fresh tensor-memory tile (two alternate), and warps 4-7 add every
// slot's tile to FP64 sums in shared memory: the FP32 accumulation then
// spans one slot's K chunks (a few tens of MMAs) instead of all 27 slots,
// whose hundreds of FP32 roundings measured 4e-6 relative in the
// potential.  (A caller whose products are small beside the result -- the
// tail of the split-precision Laplace M2L -- accumulates a tile's slots in
// one tile and has it summed once, `group`.)  At the end of a tile the FP64 sums are added to the local
// expansions.  Levels with fewer tiles than SMs split the 27 slots over
// slices of blocks (grid rows), each writing FP64 partial sums that a
// second kernel adds in slice order.  Every wait is bounded in time; a wait that runs out
// stops all roles of the block, sets *err, and the block still frees its
// tensor memory after its MMAs have completed.
#include "helmholtz.cuh"
#include "laplace.cuh"
#include "tc_common.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>

namespace fmm2d {
namespace {

constexpr int kHtRows = 128;
constexpr int kHtStages = 4;
constexpr int kHtLag = 2;
constexpr int kHtEpi0 = 4;             // warps 4-7 read the accumulators
constexpr int kHtThreads = 9 * 32;     // warp 8 issues the MMAs
constexpr int kHtTmemCols = 256;       // two accumulators of up to 128 columns
constexpr uint64_t kHtWaitNs = 2000000000ull;
constexpr int kHtSlots = 27;
constexpr int kHtMaxOrder = 23;        // 2 (2p + 1) <= 96

struct HtArgs {
    int tb[5];     // tiles of the level's four segments: [tb[c], tb[c + 1])
    int start[4];  // first plan row of each segment
    int count[4];  // targets of each segment
    const int *boxes;  // target box of each plan row
    const int *slots;  // [plan row][27] source box, -1 when none
    int lstart;        // first box of the level
    int nd, tpt, W;    // channels, target boxes per tile, 2p + 1
    const float *arow;  // [level box][nd][hi KP | lo KP]
    const float *bimg;  // [cp][slot][chunk][hi NP x 16 | lo NP x 16], operand layout
    double2 *locl;      // the level's local expansions, [level box][2p + 1][nd]
    double oscale;      // 1 / (scale of Bop)
    int *err;
    int stall;                 // fault injection: the issuer issues nothing
    unsigned long long wait_ns;  // limit of every bounded wait
    // slot slices (levels with fewer tiles than SMs): block row y takes the
    // slots [27 y / gridDim.y, 27 (y + 1) / gridDim.y) and, with more than
    // one slice, writes its FP64 partial sums to part[y][plan row - q_lo][W][nd]
    double2 *part;
    int q_lo, nq;
    // consecutive slots that share one tensor-memory accumulator before the
    // epilogue adds it to the FP64 sums: 1 (every slot summed in FP64), or
    // 27 (one FP32 accumulation over the tile's slots, for products whose
    // FP32 accumulation error is far below the result's tolerance)
    int group;
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int KP, int NP>
__global__ void __launch_bounds__(kHtThreads, 1) slot_gemm_tc_kernel(HtArgs A) {
    constexpr int KC = KP / 16;                      // K chunks per slot
    constexpr uint32_t A_BYTES = kHtRows * 16 * 4;   // one of hi / lo
    constexpr uint32_t B_BYTES = NP * 16 * 4;
    constexpr uint32_t STAGE = 2 * A_BYTES + 2 * B_BYTES;
    constexpr uint32_t LBO_A = (kHtRows / 8) * 128, LBO_B = (NP / 8) * 128, SBO = 128;
    constexpr uint32_t IDESC = tc_idesc_tf32(kHtRows, NP);
    static_assert(KP % 16 == 0 && NP % 16 == 0 && NP <= 128, "operand shape");
    extern __shared__ __align__(1024) unsigned char ht_smem[];
    // FP64 sums of the slots' partial products, column-major [NP][128] (the
    // epilogue thread of row r owns column entries c * 128 + r)
    double *sSum = reinterpret_cast<double *>(ht_smem + (size_t)kHtStages * STAGE);
    // barriers: [0, S) stage full, [S, 2S) stage free, 2S + a accumulator a
    // full, 2S + 2 + a accumulator a free, 2S + 4 final
    __shared__ __align__(8) uint64_t s_bar[2 * kHtStages + 5];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    volatile int *abort_flag = &s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t bar0 = smem_u32(&s_bar[0]);
#define HBAR(i) (bar0 + 8u * (uint32_t)(i))
    if (tid == 0) {
        for (int i = 0; i < kHtStages; i++) {
            mbar_init(HBAR(i), kHtRows);
            mbar_init(HBAR(kHtStages + i), 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(HBAR(2 * kHtStages + a), 1);
            mbar_init(HBAR(2 * kHtStages + 2 + a), kHtRows);
        }
        mbar_init(HBAR(2 * kHtStages + 4), 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&s_tmem)),
                     "r"(kHtTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t sbase = smem_u32(ht_smem);
    const int ntiles = A.tb[4] - A.tb[0];
    const int k0 = (int)blockIdx.y * kHtSlots / (int)gridDim.y;
    const int k1 = ((int)blockIdx.y + 1) * kHtSlots / (int)gridDim.y;
    // segment (child position) and first plan row of a tile
    auto tile_seg = [&](int tile, int &cp, int &q0) {
        const int t = A.tb[0] + tile;
        cp = 0;
        while (cp < 3 && t >= A.tb[cp + 1]) cp++;
        q0 = A.start[cp] + (t - A.tb[cp]) * A.tpt;
    };

    if (warp < kHtEpi0) {
        // ------------------------------------------------------- producers
        const int r = tid;  // A row
        const int bx = r / A.nd, ch = r - bx * A.nd;
        const uint32_t aoff = (uint32_t)(((r >> 3) * 128) + ((r & 7) * 16));
        long long step = 0;
        bool ok = true;
        for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
            int cp, q0;
            tile_seg(tile, cp, q0);
            const int q = q0 + bx;
            const bool valid = bx < A.tpt && q < A.start[cp] + A.count[cp];
            const int *qs = A.slots + (size_t)(valid ? q : 0) * kHtSlots;
            for (int k = k0; ok && k < k1; k++) {
                const int sb = valid ? __ldg(qs + k) : -1;
                const float *src = A.arow + (sb >= 0 ? ((size_t)(sb - A.lstart) * A.nd + ch) * 2 * KP : 0);
                const uint32_t abytes = sb >= 0 ? 16u : 0u;  // 0: zero fill
                const float *bsrc = A.bimg + ((size_t)(cp * kHtSlots + k) * KC) * (2 * NP * 16);
                for (int kc = 0; kc < KC; kc++, step++) {
                    const int s = (int)(step % kHtStages);
                    const long long u = step / kHtStages;
                    if (u >= 1 &&
                        !mbar_wait_bounded(HBAR(kHtStages + s), (uint32_t)((u - 1) & 1), abort_flag,
                                           A.wait_ns)) {
                        ok = false;
                        break;
                    }
                    const uint32_t st = sbase + (uint32_t)s * STAGE;
#pragma unroll
                    for (int cc = 0; cc < 4; cc++) {
                        const int kk = 16 * kc + 4 * cc;
                        cp_async16(st + (uint32_t)cc * LBO_A + aoff, src + kk, abytes);
                        cp_async16(st + A_BYTES + (uint32_t)cc * LBO_A + aoff, src + KP + kk, abytes);
                    }
                    const float *bc = bsrc + (size_t)kc * (2 * NP * 16);
#pragma unroll
                    for (int e = r; e < NP * 8; e += kHtRows)
                        cp_async16(st + 2 * A_BYTES + 16u * (uint32_t)e, bc + 4 * e, 16u);
                    cp_async_commit();
                    if (step >= kHtLag) {
                        cp_async_wait<kHtLag>();
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        mbar_arrive(HBAR((int)((step - kHtLag) % kHtStages)));
                    }
                }
            }
        }
        cp_async_wait<0>();
        if (ok) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            for (long long t = step - kHtLag; t < step; t++)
                if (t >= 0) mbar_arrive(HBAR((int)(t % kHtStages)));
        } else {
            *abort_flag = 1;
        }
    } else if (warp < kHtEpi0 + 4) {
        // -------------------------------------------------------- epilogue
        // Each slot's products accumulate in a fresh tensor-memory tile
        // (two alternate between slots); this thread adds its row of every
        // slot's tile in FP64, so the FP32 accumulation spans only the
        // slot's own K chunks.
        const int e = warp - kHtEpi0;  // tensor-memory lanes 32 e .. 32 e + 31
        const int r = (e << 5) + lane;
        const int bx = r / A.nd, ch = r - bx * A.nd;
        long long g = 0;  // slots finished by this block
        bool ok = true;
        for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
#pragma unroll 4
            for (int c = 0; c < NP; c++) sSum[c * kHtRows + r] = 0.0;
            for (int k = k0; k < k1; k++) {
                if ((k - k0) % A.group != A.group - 1 && k != k1 - 1) continue;  // (not a group's end)
                const int a = (int)(g & 1);
                const bool got = mbar_wait_backoff(HBAR(2 * kHtStages + a), (uint32_t)((g >> 1) & 1),
                                                   abort_flag, A.wait_ns);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t taddr = tmem + ((uint32_t)(e << 5) << 16) + (uint32_t)(a * 128);
                float d[NP];
#pragma unroll
                for (int c8 = 0; c8 < NP / 8; c8++) {
                    float v[8];
                    tc_ld8(taddr + (uint32_t)(8 * c8), v);
#pragma unroll
                    for (int i = 0; i < 8; i++) d[8 * c8 + i] = v[i];
                }
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                mbar_arrive(HBAR(2 * kHtStages + 2 + a));
#pragma unroll
                for (int c = 0; c < NP; c++) sSum[c * kHtRows + r] += (double)d[c];
                g++;
            }
            if (!ok) break;
            int cp, q0;
            tile_seg(tile, cp, q0);
            const int q = q0 + bx;
            if (bx < A.tpt && q < A.start[cp] + A.count[cp]) {
                double *o;
                bool add = true;
                if (gridDim.y > 1) {  // this slice's partial sums
                    o = reinterpret_cast<double *>(
                        A.part + ((size_t)blockIdx.y * A.nq + (q - A.q_lo)) * A.W * A.nd + ch);
                    add = false;
                } else {
                    const int b = A.boxes[q];
                    o = reinterpret_cast<double *>(A.locl + (size_t)(b - A.lstart) * A.W * A.nd + ch);
                }
                const size_t st = 2 * (size_t)A.nd;
                // column c: Re L_(c - p) for c < W, Im L_(c - W - p) for W <= c < 2W
                for (int c = 0; c < 2 * A.W; c++) {
                    const double v = A.oscale * sSum[c * kHtRows + r];
                    double &dst = c < A.W ? o[(size_t)c * st] : o[(size_t)(c - A.W) * st + 1];
                    dst = add ? dst + v : v;
                }
            }
        }
        if (!ok) *abort_flag = 1;
    } else {
        // ---------------------------------------------------------- issuer
        long long step = 0, g = 0;
        bool ok = true, issued = false;
        // (fault injection: nothing is issued or committed, so the other
        // roles' bounded waits run out)
        for (int tile = blockIdx.x; ok && !A.stall && tile < ntiles; tile += gridDim.x) {
            uint32_t acc = 0u, dt = tmem;
            int a = 0;
            for (int k = k0; ok && k < k1; k++) {
                const bool gstart = (k - k0) % A.group == 0;
                const bool gend = (k - k0) % A.group == A.group - 1 || k == k1 - 1;
                if (gstart) {
                    // the group's accumulator tile, once the epilogue has
                    // read it two groups ago
                    a = (int)(g & 1);
                    const bool freed = g < 2 || mbar_wait_bounded(HBAR(2 * kHtStages + 2 + a),
                                                                  (uint32_t)(((g >> 1) - 1) & 1),
                                                                  abort_flag, A.wait_ns);
                    if (!__all_sync(0xffffffffu, freed)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    dt = tmem + (uint32_t)(a * 128);
                    acc = 0u;
                }
                for (int kc = 0; kc < KC; kc++, step++) {
                    const int s = (int)(step % kHtStages);
                    const long long u = step / kHtStages;
                    if (!__all_sync(0xffffffffu, mbar_wait_bounded(HBAR(s), (uint32_t)(u & 1),
                                                                   abort_flag, A.wait_ns))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    if (lane == 0) {
                        const uint32_t st = sbase + (uint32_t)s * STAGE;
                        const uint32_t ahi = st, alo = st + A_BYTES;
                        const uint32_t bhi = st + 2 * A_BYTES, blo = bhi + B_BYTES;
#pragma unroll
                        for (int ks = 0; ks < 2; ks++) {
                            const uint32_t ao = 2u * ks * LBO_A, bo = 2u * ks * LBO_B;
                            tc_mma(dt, tc_sdesc(ahi + ao, LBO_A, SBO), tc_sdesc(bhi + bo, LBO_B, SBO),
                                   IDESC, acc);
                            tc_mma(dt, tc_sdesc(ahi + ao, LBO_A, SBO), tc_sdesc(blo + bo, LBO_B, SBO),
                                   IDESC, 1u);
                            tc_mma(dt, tc_sdesc(alo + ao, LBO_A, SBO), tc_sdesc(bhi + bo, LBO_B, SBO),
                                   IDESC, 1u);
                            acc = 1u;
                        }
                        tc_commit(HBAR(kHtStages + s));
                    }
                    __syncwarp();
                    issued = true;
                }
                if (!ok) break;
                if (gend) {
                    if (lane == 0) tc_commit(HBAR(2 * kHtStages + a));
                    __syncwarp();
                    g++;
                }
            }
        }
        if (!ok) *abort_flag = 1;
        // the MMAs still in flight finish before the tensor memory is freed
        if (issued && lane == 0) {
            int never = 0;
            tc_commit(HBAR(2 * kHtStages + 4));
            mbar_wait_bounded(HBAR(2 * kHtStages + 4), 0u, &never, kHtWaitNs);
        }
        __syncwarp();
    }
#undef HBAR
    __syncthreads();
    if (tid == 0 && s_abort) atomicExch(A.err, 1);
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kHtTmemCols)
                     : "memory");
    }
}

template <int KP, int NP>
constexpr size_t ht_smem_bytes() {
    return (size_t)kHtStages * (2 * kHtRows * 16 * 4 + 2 * NP * 16 * 4) +
           (size_t)NP * kHtRows * sizeof(double);
}

// x rounded to TF32 (nearest, ties away from zero), as cvt.rna does.
__device__ __forceinline__ void ht_split(float v, float &hi, float &lo) {
    hi = tc_tf32(v);
    lo = tc_tf32(v - hi);
}

// Operand-ready A rows of the level's boxes: [box][ch][hi KP | lo KP] of
// [Re M_-p..p | Im M_-p..p | 0].
__global__ void __launch_bounds__(256) slot_rows_kernel(long long nrow, int nd, int W, int KP,
                                                          const double2 *__restrict__ mpl,
                                                          float *__restrict__ arow) {
    const long long n = nrow * KP;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const long long row = t / KP;
        const int k = (int)(t - row * KP);
        const long long b = row / nd;
        const int ch = (int)(row - b * nd);
        float v = 0.f;
        if (k < 2 * W) {
            const double2 m = mpl[((size_t)b * W + (k < W ? k : k - W)) * nd + ch];
            v = (float)(k < W ? m.x : m.y);
        }
        float hi, lo;
        ht_split(v, hi, lo);
        arow[row * 2 * KP + k] = hi;
        arow[row * 2 * KP + KP + k] = lo;
    }
}

// Bop images of the level: for child position cp, slot k (source offset
// dxy[cp][k] = source - target) and K chunk kc, the real form of
// B_ij = T(i - j) w_ij scaled by `scale`, TF32 hi then lo, each N x 16 in
// the K-major no-swizzle layout.
__global__ void __launch_bounds__(256) helm_tc_bimg_kernel(int p, int KP, int NP, double scale,
                                                          const int2 *__restrict__ dxy,
                                                          const double2 *__restrict__ Tl,
                                                          const double *__restrict__ pw,
                                                          float *__restrict__ bimg) {
    const int W = 2 * p + 1, N = 2 * p, tw = 2 * N + 1, KC = KP / 16;
    const long long n = (long long)4 * kHtSlots * NP * KP;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % KP);
        const int nn = (int)((t / KP) % NP);
        const int cs = (int)(t / ((long long)KP * NP));  // cp * 27 + slot
        double v = 0.0;
        if (nn < 2 * W && k < 2 * W) {
            const int i = (nn < W ? nn : nn - W) - p, j = (k < W ? k : k - W) - p;
            const int2 d = dxy[cs];
            const double2 *T0 = Tl + (size_t)((3 - d.y) * 7 + (3 - d.x)) * tw + N;
            double2 b = T0[i - j];
            if ((i > 0 && j > 0) || (i < 0 && j < 0)) {
                const double w = pw[2 * min(abs(i), abs(j))];
                b.x *= w;
                b.y *= w;
            }
            const bool re_out = nn < W, re_in = k < W;
            v = re_out ? (re_in ? b.x : -b.y) : (re_in ? b.y : b.x);
        }
        float hi, lo;
        ht_split((float)(v * scale), hi, lo);
        float *blk = bimg + (size_t)cs * KC * (2 * NP * 16) + slot_bimg_at(nn, k, NP);
        blk[0] = hi;
        blk[NP * 16] = lo;
    }
}

template <int KP, int NP>
void launch_ht(const HtArgs &a, int ntiles, int nslice, cudaStream_t s) {
    const size_t smem = ht_smem_bytes<KP, NP>();
    raise_smem_limit((const void *)slot_gemm_tc_kernel<KP, NP>, smem);
    const dim3 grid(std::max(1, std::min(ntiles, kNumSM)), nslice);
    slot_gemm_tc_kernel<KP, NP><<<grid, kHtThreads, smem, s>>>(a);
    FMM_CHECK_LAUNCH();
}

// The slices' partial sums, added in slice order to the local expansions
// of the level's plan rows.
__global__ void __launch_bounds__(256) helm_tc_slices_kernel(
    int nq, int wf, int nslice, const double2 *__restrict__ part, const int *__restrict__ boxes,
    int q_lo, int lstart, double2 *__restrict__ locl) {
    const long long n = (long long)nq * wf;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(t / wf), o = (int)(t - (long long)q * wf);
        double2 acc = make_double2(0.0, 0.0);
        for (int y = 0; y < nslice; y++) acc = cadd(acc, part[(size_t)y * n + t]);
        double2 *dst = locl + (size_t)(boxes[q_lo + q] - lstart) * wf + o;
        *dst = cadd(*dst, acc);
    }
}

}  // namespace

int helm_m2l_tc_max_order() { return kHtMaxOrder; }

int slot_gemm_kp(int W) {
    int KP = 32;
    while (KP < 2 * W) KP += 16;
    return KP <= 96 ? KP : 0;
}

void slot_gemm_rows(long long nrow, int nd, int W, int KP, const double2 *x, float *arow,
                    cudaStream_t s) {
    const long long n = nrow * KP;
    if (n <= 0) return;
    const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)kNumSM * 16);
    slot_rows_kernel<<<std::max(blocks, 1), 256, 0, s>>>(nrow, nd, W, KP, x, arow);
    FMM_CHECK_LAUNCH();
}

bool slot_gemm_tc_level(const SlotGemmLevel &g, const SlotPlan &spl, int *err, cudaStream_t s) {
    const int W = g.W, nd = g.nd, KP = g.KP;
    if (W < 1 || nd < 1 || nd > kHtRows || KP != slot_gemm_kp(W) || KP == 0) return false;
    const int g0 = 4 * (g.level - 2);
    if (g0 < 0 || g0 + 4 > spl.nseg) return false;
    HtArgs a;
    for (int c = 0; c <= 4; c++) a.tb[c] = spl.tile_base[g0 + c];
    for (int c = 0; c < 4; c++) {
        a.start[c] = spl.start[g0 + c];
        a.count[c] = spl.count[g0 + c];
    }
    const int ntiles = a.tb[4] - a.tb[0];
    if (ntiles == 0) return true;
    a.boxes = spl.boxes;
    a.slots = spl.slots;
    a.lstart = g.lstart;
    a.nd = nd;
    a.tpt = kHtRows / nd;
    a.W = W;
    a.arow = g.arow;
    a.bimg = g.bimg;
    a.locl = g.out;
    a.oscale = g.oscale;
    a.err = err;
    a.stall = tc_stall_injected();
    a.wait_ns = tc_wait_limit_ns();
    a.group = g.group >= 1 ? g.group : 1;
    // levels with fewer tiles than SMs (the coarse ones) split the 27 slots
    // over slices of blocks, whose FP64 partial sums are added in slice order
    const int nslice = ntiles < kNumSM ? std::min(kHtSlots, std::max(1, kNumSM / ntiles)) : 1;
    a.q_lo = a.start[0];
    a.nq = a.start[3] + a.count[3] - a.q_lo;
    DevBuf<double2> part(nslice > 1 ? (size_t)nslice * a.nq * W * nd : 0, s);
    a.part = part.get();
    switch (KP) {
        case 32: launch_ht<32, 32>(a, ntiles, nslice, s); break;
        case 48: launch_ht<48, 48>(a, ntiles, nslice, s); break;
        case 64: launch_ht<64, 64>(a, ntiles, nslice, s); break;
        case 80: launch_ht<80, 80>(a, ntiles, nslice, s); break;
        case 96: launch_ht<96, 96>(a, ntiles, nslice, s); break;
        default: return false;
    }
    if (nslice > 1) {
        const long long n = (long long)a.nq * W * nd;
        const int blocks = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, kNumSM * 8));
        helm_tc_slices_kernel<<<blocks, 256, 0, s>>>(a.nq, W * nd, nslice, part.get(), spl.boxes,
                                                     a.q_lo, g.lstart, g.out);
        FMM_CHECK_LAUNCH();
    }
    return true;
}

bool helm_m2l_tc_level(const HtLevel &lv, const SlotPlan &spl, const double2 *mp, double2 *loc,
                       int *err, cudaStream_t s) {
    const int p = lv.p, W = 2 * p + 1, nd = lv.nd;
    if (p > kHtMaxOrder || p < 1 || nd < 1 || nd > kHtRows) return false;
    if (!(lv.maxabs > 0.0) || !std::isfinite(lv.maxabs)) return false;
    // a power of two that brings the largest entry of Bop to about 1; the
    // level keeps the FP64 form if that scale or the entries leave the
    // FP32 range
    const int ex = (int)std::floor(std::log2(lv.maxabs));
    if (ex > 120 || ex < -120) return false;
    const double scale = std::ldexp(1.0, -ex);
    const int g0 = 4 * (lv.level - 2);
    if (g0 < 0 || g0 + 4 > spl.nseg) return false;
    if (spl.tile_base[g0 + 4] == spl.tile_base[g0]) return true;
    const int KP = slot_gemm_kp(W);
    if (KP == 0) return false;
    const int NP = KP;
    const long long nbox = lv.nbox;
    DevBuf<float> arow((size_t)nbox * nd * 2 * KP, s);
    DevBuf<float> bimg((size_t)4 * kHtSlots * 2 * NP * KP, s);
    slot_gemm_rows(nbox * nd, nd, W, KP, mp + lv.off, arow.get(), s);
    {
        const long long n = (long long)4 * kHtSlots * NP * KP;
        const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)kNumSM * 16);
        helm_tc_bimg_kernel<<<blocks, 256, 0, s>>>(p, KP, NP, scale, spl.dxy, lv.table, lv.pw,
                                                   bimg.get());
        FMM_CHECK_LAUNCH();
    }
    SlotGemmLevel g;
    g.level = lv.level;
    g.lstart = lv.lstart;
    g.nd = nd;
    g.W = W;
    g.KP = KP;
    g.arow = arow.get();
    g.bimg = bimg.get();
    g.out = loc + lv.off;
    g.oscale = 1.0 / scale;
    return slot_gemm_tc_level(g, spl, err, s);
}

}  // namespace fmm2d
