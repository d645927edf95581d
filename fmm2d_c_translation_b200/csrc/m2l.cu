// m2l.cu -- M2L over list 2 on the FP64 tensor cores (mma.sync m8n8k4 f64).
//
// The reference's multipole-to-local shift (l2dmploc,
// c_translation/src/laprouts2d.c:886-994) of a source box at c1 to a
// target box at c2 of the same level (box size r) factors as
//
//     L_i += w2^i [ B h~ ]_i  (+ log|z0| h~_0 for i = 0),  h~_j = w1^j M_j,
//
// with z0 = c1 - c2 = r t, w1 = -1/t, w2 = 1/t and the fixed real matrix
//     B_00 = 0,  B_0j = 1 (j >= 1),  B_i0 = -1/i,  B_ij = C(i+j-1, j-1).
// In a list-2 pair t is one of 40 lattice offsets, and the 8 target boxes
// of a tile that sit at the same position in their parents share the same
// 27 possible offsets.  A warp therefore owns 8 such boxes, walks the 27
// offsets, and for each one multiplies B (the A operand, fixed, staged in
// shared memory) by the 8 scaled source multipoles (the B operand, one
// column per box) with DMMA, then applies w2^i and accumulates the locals
// in registers.  Each box's local expansion has one writer (no atomics).
//
// Boxes are grouped into tiles by (level, child position) with one radix
// sort; the source of every (target, offset) slot is found once from
// list 2.  If any list-2 entry falls outside the 27 slots (not expected of
// the reference's trees) the caller falls back to the per-box kernel.
#include "laplace.cuh"
#include "sort.cuh"
#include "tc_common.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <stdlib.h>
#include <string.h>
#include <vector>

namespace fmm2d {

namespace {

constexpr int kSlots = 27;

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile(
        "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// The 27 lattice offsets (dx, dy) of list 2 for a box at child position
// cpos (bit 0: right half of the parent, bit 1: upper half), in a fixed
// order; slot_of maps (cpos, dx + 3, dy + 3) to the slot or -1.
struct SlotTables {
    int dx[4][kSlots], dy[4][kSlots];
    int slot_of[4][7][7];
};

SlotTables make_slot_tables() {
    SlotTables t;
    for (int c = 0; c < 4; c++) {
        for (int a = 0; a < 7; a++)
            for (int b = 0; b < 7; b++) t.slot_of[c][a][b] = -1;
        const int px = c & 1, py = (c >> 1) & 1;
        int k = 0;
        for (int dy = -2 - py; dy <= 3 - py; dy++)
            for (int dx = -2 - px; dx <= 3 - px; dx++) {
                if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1) continue;
                t.dx[c][k] = dx;
                t.dy[c][k] = dy;
                t.slot_of[c][dx + 3][dy + 3] = k;
                k++;
            }
    }
    return t;
}

__constant__ int c_slot_dx[4][kSlots];
__constant__ int c_slot_dy[4][kSlots];
__constant__ int c_slot_of[4][7][7];

// Segment = (level, child position); tiles of 8 boxes within a segment.
struct SegTable {
    const int *tile_base;  // nseg + 1
    const int *start;      // nseg, into the sorted box list
    const int *count;      // nseg
    const int *level;      // nseg
    const int *cpos;       // nseg
    int nseg;
};

// NT > 0: only the terms with i + j < NT (the leading triangle of the
// shift; the split-precision M2L adds the rest on the tensor cores), every
// row of the locals still stored.
template <int MT, int KS, int CH, int NT = 0>
__global__ void __launch_bounds__(128, 4) m2l_dmma_kernel(
    SegTable seg, const int *__restrict__ boxes, const int *__restrict__ slots,
    const double *__restrict__ bs, int ndc, int c0, int p,
    const double *__restrict__ binom, const double2 *__restrict__ mp,
    double2 *__restrict__ loc, int ntiles) {
    // A-operand fragments of B: [mt][ks][lane]
    __shared__ double s_a[MT * KS * 32];
    __shared__ int s_tb[257];
    // (mt, ks) tiles with a term of the triangle
    auto live = [](int mt, int ks) { return NT == 0 || mt * 8 + ks * 4 < NT; };
    for (int e = threadIdx.x; e < MT * KS * 32; e += blockDim.x) {
        const int l = e & 31, ks = (e >> 5) % KS, mt = (e >> 5) / KS;
        const int i = mt * 8 + (l >> 2), j = ks * 4 + (l & 3);
        double v = 0.0;
        if (i <= p && j <= p && (NT == 0 || i + j < NT)) {
            if (i == 0)
                v = j == 0 ? 0.0 : 1.0;
            else
                v = j == 0 ? -1.0 / i : binom[(size_t)(i + j - 1) * (kLdc + 1) + (j - 1)];
        }
        s_a[e] = v;
    }
    for (int e = threadIdx.x; e <= seg.nseg && e < 257; e += blockDim.x) s_tb[e] = seg.tile_base[e];
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    const int stride = (p + 1) * ndc;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < ntiles; tile += nwarps) {
        // segment of this tile
        int lo = 0, hi = seg.nseg;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_tb[mid] <= tile) lo = mid; else hi = mid;
        }
        const int sg = lo;
        const int q0 = seg.start[sg] + (tile - s_tb[sg]) * 8;
        const int qend = seg.start[sg] + seg.count[sg];
        const int cp = seg.cpos[sg];
        const double lr = log(bs[seg.level[sg]]);
        // this lane's B-operand column box (g) and C columns (2 tig, 2 tig + 1)
        const int qg = q0 + g;
        const bool has_g = qg < qend;
        double acc[CH][MT][2][2];  // [ch][mt][e][re/im]
#pragma unroll
        for (int c = 0; c < CH; c++)
#pragma unroll
            for (int mt = 0; mt < MT; mt++)
#pragma unroll
                for (int e = 0; e < 2; e++) acc[c][mt][e][0] = acc[c][mt][e][1] = 0.0;
        for (int k = 0; k < kSlots; k++) {
            const int sg_box = has_g ? slots[(size_t)qg * kSlots + k] : -1;
            // skip the offset when no box of the tile has a source there
            if (__ballot_sync(0xffffffffu, sg_box >= 0) == 0) continue;
            const double tx = (double)c_slot_dx[cp][k], ty = (double)c_slot_dy[cp][k];
            // w2 = 1/t, w1 = -1/t
            const double tn = 1.0 / (tx * tx + ty * ty);
            const double2 w2 = make_double2(tx * tn, -ty * tn);
            const double2 w1 = make_double2(-w2.x, -w2.y);
            const double lt = 0.5 * log(tx * tx + ty * ty);
            // w1^(tig) and w1^4 for the B fragments (j = 4 ks + tig)
            double2 w1p = make_double2(1.0, 0.0);
            for (int u = 0; u < tig; u++) w1p = cmul(w1p, w1);
            const double2 w1_2 = cmul(w1, w1), w1_4 = cmul(w1_2, w1_2);
            // w2^g and w2^8 for the C rows (i = 8 mt + g)
            double2 w2p = make_double2(1.0, 0.0);
            for (int u = 0; u < g; u++) w2p = cmul(w2p, w2);
            const double2 w2_2 = cmul(w2, w2), w2_4 = cmul(w2_2, w2_2), w2_8 = cmul(w2_4, w2_4);
            // sources of the C columns, for the log term of row 0
            const int sn0 = __shfl_sync(0xffffffffu, sg_box, (2 * tig) * 4);
            const int sn1 = __shfl_sync(0xffffffffu, sg_box, (2 * tig + 1) * 4);
#pragma unroll
            for (int c = 0; c < CH; c++) {
                double bre[KS], bim[KS];
                double2 wj = w1p;
#pragma unroll
                for (int ks = 0; ks < KS; ks++) {
                    const int j = ks * 4 + tig;
                    double2 h = make_double2(0.0, 0.0);
                    if (live(0, ks) && sg_box >= 0 && j <= p)
                        h = cmul(mp[(size_t)sg_box * stride + (size_t)j * ndc + c0 + c], wj);
                    bre[ks] = h.x;
                    bim[ks] = h.y;
                    wj = cmul(wj, w1_4);
                }
                double tre[MT][2], tim[MT][2];
#pragma unroll
                for (int mt = 0; mt < MT; mt++) {
                    tre[mt][0] = tre[mt][1] = tim[mt][0] = tim[mt][1] = 0.0;
#pragma unroll
                    for (int ks = 0; ks < KS; ks++) {
                        if (!live(mt, ks)) continue;
                        const double a = s_a[(mt * KS + ks) * 32 + lane];
                        dmma(tre[mt][0], tre[mt][1], a, bre[ks]);
                        dmma(tim[mt][0], tim[mt][1], a, bim[ks]);
                    }
                }
                double2 wi = w2p;
#pragma unroll
                for (int mt = 0; mt < MT; mt++) {
                    if (!live(mt, 0)) break;  // (rows of no triangle term stay zero)
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const double2 tt = make_double2(tre[mt][e], tim[mt][e]);
                        const double2 v = cmul(wi, tt);
                        acc[c][mt][e][0] += v.x;
                        acc[c][mt][e][1] += v.y;
                    }
                    wi = cmul(wi, w2_8);
                }
                if (g == 0) {  // row i = 0 of mt = 0: + log|z0| M_0
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const int sn = e == 0 ? sn0 : sn1;
                        if (sn >= 0) {
                            const double2 m0 = mp[(size_t)sn * stride + c0 + c];
                            acc[c][0][e][0] += (lr + lt) * m0.x;
                            acc[c][0][e][1] += (lr + lt) * m0.y;
                        }
                    }
                }
            }
        }
        // store: the first writer of these boxes' local expansions
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int q = q0 + 2 * tig + e;
            if (q >= qend) continue;
            const int b = boxes[q];
#pragma unroll
            for (int mt = 0; mt < MT; mt++) {
                const int i = mt * 8 + g;
                if (i > p) continue;
#pragma unroll
                for (int c = 0; c < CH; c++)
                    loc[(size_t)b * stride + (size_t)i * ndc + c0 + c] =
                        make_double2(acc[c][mt][e][0], acc[c][mt][e][1]);
            }
        }
    }
}

template <int MT, int KS, int NT = 0>
void launch_dmma(const SegTable &sg, const int *boxes, const int *slots,
                 const double *bs, int ndc, int p, const double *binom,
                 const double2 *mp, double2 *loc, int ntiles, cudaStream_t s) {
    const int blocks = std::max(1, std::min((ntiles + 3) / 4, kNumSM * 16));
    const char *e = getenv("FMM2D_B200_M2L_CH2");
    const bool ch2 = e && e[0] == '1';
    for (int c0 = 0; c0 < ndc;) {
        if (ch2 && ndc - c0 >= 2 && MT <= 5) {
            m2l_dmma_kernel<MT, KS, 2, NT><<<blocks, 128, 0, s>>>(
                sg, boxes, slots, bs, ndc, c0, p, binom, mp, loc, ntiles);
            c0 += 2;
        } else {
            m2l_dmma_kernel<MT, KS, 1, NT><<<blocks, 128, 0, s>>>(
                sg, boxes, slots, bs, ndc, c0, p, binom, mp, loc, ntiles);
            c0 += 1;
        }
        FMM_CHECK_LAUNCH();
    }
}


// The tiles of one M2L evaluation: target boxes of levels >= 2 that hold
// points, sorted by (level, child position) = segment, and the source box of
// every (target, slot).
struct M2LWork {
    DevBuf<uint32_t> keys, vals, kt, vt;
    DevBuf<int> segd, slots;
    std::vector<int> hseg;  // host copy of segd
    int nseg = 0, ntarg = 0, ntiles = 0;
    SegTable seg() const {
        const int *h = segd.get();
        return SegTable{h, h + nseg + 1, h + 2 * nseg + 1, h + 3 * nseg + 1, h + 4 * nseg + 1,
                        nseg};
    }
};

// Cache key of a planning object: its kind, tile size and skipped levels.
inline uint64_t m2l_key(int kind, int tile, uint64_t skip) {
    return ((uint64_t)kind << 56) | ((uint64_t)tile << 40) | (skip & ((1ull << 40) - 1));
}

void ensure_slot_tables(cudaStream_t s) {
    static std::mutex tables_mu;
    static bool tables_ready[64] = {false};
    int dev = 0;
    FMM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> tables_lock(tables_mu);
    if (!tables_ready[dev]) {
        const SlotTables st = make_slot_tables();
        FMM_CUDA(cudaMemcpyToSymbolAsync(c_slot_dx, st.dx, sizeof(st.dx), 0, cudaMemcpyHostToDevice, s));
        FMM_CUDA(cudaMemcpyToSymbolAsync(c_slot_dy, st.dy, sizeof(st.dy), 0, cudaMemcpyHostToDevice, s));
        FMM_CUDA(cudaMemcpyToSymbolAsync(c_slot_of, st.slot_of, sizeof(st.slot_of), 0, cudaMemcpyHostToDevice, s));
        FMM_CUDA(cudaStreamSynchronize(s));
        tables_ready[dev] = true;
    }
}

// Builds the segments (tiles of `tile` boxes) and the slot table, leaving
// out the target levels set in skip_levels; false when a list-2 entry
// falls outside the 27 slots or there are too many segments.
bool m2l_work(const Tree &T, const CauchyProblem &P, int tile, cudaStream_t s, M2LWork &w,
              uint64_t skip_levels = 0) {
    const int L = T.nlevels;
    ensure_slot_tables(s);
    const int lo = T.lstart[2], n = T.nboxes - lo;
    const int nseg = 4 * (L - 1);
    w.nseg = nseg;
    const int2 *sse = T.srcse.get(), *tse = T.trgse.get();
    const int spgh = P.sset.pgh, tpgh = P.tset.pgh;
    const int *lev = T.level.get(), *par = T.parent.get(), *chi = T.child.get();
    // ---- keys: (level - 2) * 4 + child position, or nseg when not a target
    w.keys.alloc(n, s);
    w.vals.alloc(n, s);
    w.kt.alloc(n, s);
    w.vt.alloc(n, s);
    DevBuf<int> cnt(nseg + 1, s);
    cnt.zero(s);
    uint32_t *kp = w.keys.get(), *vp = w.vals.get();
    int *cp = cnt.get();
    for_each(n, s, [=] __device__(int64_t i) {
        const int b = lo + (int)i;
        int np = 0;
        if (tpgh > 0) np += tse[b].y - tse[b].x;
        if (spgh > 0) np += sse[b].y - sse[b].x;
        int key = nseg;
        if (np > 0 && !((skip_levels >> lev[b]) & 1ull)) {
            const int pb = par[b];
            int c = 0;
            for (int j = 0; j < 4; j++)
                if (chi[4 * pb + j] == b) c = j;
            key = (lev[b] - 2) * 4 + c;
        }
        kp[i] = (uint32_t)key;
        vp[i] = (uint32_t)b;
        // one atomic per group of lanes with the same segment
        const unsigned am = __activemask();
        const unsigned peers = __match_any_sync(am, key);
        if (key < nseg && (int)(threadIdx.x & 31) == __ffs(peers) - 1)
            atomicAdd(&cp[key], __popc(peers));
    });
    int bits = 1;
    while ((1 << bits) <= nseg) bits++;
    radix_sort_pairs(kp, vp, w.kt.get(), w.vt.get(), n, bits, s);
    std::vector<int> hc(nseg + 1);
    read_small(hc.data(), cp, (nseg + 1) * sizeof(int), s);
    std::vector<int> h(5 * nseg + 1);
    int *tb = h.data(), *st = tb + nseg + 1, *ct = st + nseg, *lv = ct + nseg, *cpv = lv + nseg;
    int run = 0, start = 0;
    for (int k = 0; k < nseg; k++) {
        tb[k] = run;
        st[k] = start;
        ct[k] = hc[k];
        lv[k] = 2 + k / 4;
        cpv[k] = k % 4;
        run += (hc[k] + tile - 1) / tile;
        start += hc[k];
    }
    tb[nseg] = run;
    w.ntiles = run;
    w.ntarg = start;
    w.hseg = h;
    if (w.ntiles == 0) return true;
    if (nseg + 1 > 257) return false;
    w.segd.alloc(h.size(), s);
    FMM_CUDA(cudaMemcpyAsync(w.segd.get(), h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    // ---- the source box of every (target, slot), from list 2
    const int ntarg = w.ntarg;
    w.slots.alloc((size_t)ntarg * kSlots, s);
    DevBuf<int> err(1, s);
    FMM_CUDA(cudaMemsetAsync(w.slots.get(), 0xff, (size_t)ntarg * kSlots * sizeof(int), s));
    err.zero(s);
    {
        int *sl = w.slots.get(), *ep = err.get();
        const int *n2 = T.nlist2.get(), *l2 = T.list2.get();
        const double2 *cen = T.centers.get();
        const double *bsd = T.d_boxsize.get();
        const uint32_t *bx = vp;
        for_each(ntarg, s, [=] __device__(int64_t q) {
            const int b = (int)bx[q];
            const int pb = par[b];
            int c = 0;
            for (int j = 0; j < 4; j++)
                if (chi[4 * pb + j] == b) c = j;
            const double r = bsd[lev[b]];
            const double2 cb = cen[b];
            for (int e = 0; e < n2[b]; e++) {
                const int sb = l2[kMaxList2 * b + e];
                if (sse[sb].y <= sse[sb].x) continue;  // no multipole
                const double2 cs = cen[sb];
                const int dx = (int)rint((cs.x - cb.x) / r), dy = (int)rint((cs.y - cb.y) / r);
                const int k = (dx >= -3 && dx <= 3 && dy >= -3 && dy <= 3)
                                  ? c_slot_of[c][dx + 3][dy + 3] : -1;
                if (k < 0) {
                    atomicExch(ep, 1);
                    continue;
                }
                sl[q * kSlots + k] = sb;
            }
        });
    }
    return read_scalar(err.get(), s) == 0;
}

// ---------------------------------------------------------------------------
// FP32 M2L of the mixed-precision mode.  With t the slot offset in box
// units, the whole shift is one complex matrix per (child position, slot),
// level independent in the scaled form:
//     T_ij = w2^i B_ij w1^j  (T_00 = log|t|),
// and L_i += sum_slots sum_j T_ij M_j, plus log(r) M_0 in L_0.  One thread
// per target box, 128 boxes of one segment per block; the block stages
// each slot's matrix in shared memory (read as broadcasts) and every thread
// streams its source multipole (an FP32 copy) through the j loop, keeping
// the P1 x CH accumulators in registers (FP32 arithmetic, FP32
// accumulation over the 27 slots, stored as FP64).
// ---------------------------------------------------------------------------
// NR < P1: only the rows i < NR (the leading local coefficients) are
// computed and stored; the tensor-core forms use this to recompute the rows
// that carry most of the gradient in FP32 (see the end of m2l_fp32).
constexpr int kFp32Tile = 128;

template <int P1, int CH, int NR = P1>
__global__ void __launch_bounds__(kFp32Tile) m2l_fp32_kernel(
    SegTable seg, const int *__restrict__ boxes, const int *__restrict__ slots,
    const double *__restrict__ bs, int ndc, int c0, int p, const float2 *__restrict__ Tall,
    const float2 *__restrict__ mp32, double2 *__restrict__ loc, int ntiles) {
    __shared__ float2 sT[NR * P1];
    __shared__ int s_tb[257];
    for (int e = threadIdx.x; e <= seg.nseg && e < 257; e += blockDim.x) s_tb[e] = seg.tile_base[e];
    __syncthreads();
    const int stride = (p + 1) * ndc;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int lo = 0, hi = seg.nseg;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_tb[mid] <= tile) lo = mid; else hi = mid;
        }
        const int sg = lo;
        const int q = seg.start[sg] + (tile - s_tb[sg]) * kFp32Tile + threadIdx.x;
        const bool valid = q < seg.start[sg] + seg.count[sg];
        const int cp = seg.cpos[sg];
        const float lr = (float)log(bs[seg.level[sg]]);
        float2 acc[CH][NR];
        float2 s0[CH];
#pragma unroll
        for (int c = 0; c < CH; c++) {
            s0[c] = make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 0; i < NR; i++) acc[c][i] = make_float2(0.f, 0.f);
        }
        for (int k = 0; k < kSlots; k++) {
            __syncthreads();  // the previous slot's matrix is no longer read
            const float2 *Tk = Tall + ((size_t)cp * kSlots + k) * P1 * P1;
            for (int e = threadIdx.x; e < NR * P1; e += blockDim.x) sT[e] = Tk[e];
            __syncthreads();
            const int sb = valid ? slots[(size_t)q * kSlots + k] : -1;
            if (sb < 0) continue;
            const float2 *M = mp32 + (size_t)sb * stride + c0;
#pragma unroll
            for (int j = 0; j < P1; j++) {
                float2 m[CH];
#pragma unroll
                for (int c = 0; c < CH; c++)
                    m[c] = j <= p ? M[(size_t)j * ndc + c] : make_float2(0.f, 0.f);
                if (j == 0) {
#pragma unroll
                    for (int c = 0; c < CH; c++) {
                        s0[c].x += m[c].x;
                        s0[c].y += m[c].y;
                    }
                }
#pragma unroll
                for (int i = 0; i < NR; i++) {
                    const float2 t = sT[i * P1 + j];
#pragma unroll
                    for (int c = 0; c < CH; c++) {
                        acc[c][i].x = fmaf(t.x, m[c].x, fmaf(-t.y, m[c].y, acc[c][i].x));
                        acc[c][i].y = fmaf(t.x, m[c].y, fmaf(t.y, m[c].x, acc[c][i].y));
                    }
                }
            }
        }
        if (valid) {
            const int b = boxes[q];
#pragma unroll
            for (int c = 0; c < CH; c++) {
                acc[c][0].x += lr * s0[c].x;
                acc[c][0].y += lr * s0[c].y;
            }
#pragma unroll
            for (int i = 0; i < NR; i++) {
                if (i > p) break;
#pragma unroll
                for (int c = 0; c < CH; c++)
                    loc[(size_t)b * stride + (size_t)i * ndc + c0 + c] =
                        make_double2((double)acc[c][i].x, (double)acc[c][i].y);
            }
        }
    }
}

// T_ij = w2^i B_ij w1^j per (child position, slot), FP64 built, FP32
// stored, padded to P1 x P1; cached per device and order.
const float2 *fp32_tables(int p, int P1, cudaStream_t s) {
    static std::mutex mu;
    static std::vector<std::pair<long, const float2 *>> cache;
    int dev;
    FMM_CUDA(cudaGetDevice(&dev));
    const long key = ((long)dev << 20) | ((long)p << 8) | P1;
    std::lock_guard<std::mutex> g(mu);
    for (auto &e : cache)
        if (e.first == key) return e.second;
    const SlotTables st = make_slot_tables();
    // binomials C(l, m) for l <= 2 P1
    const int nc = 2 * P1 + 2;
    std::vector<double> C((size_t)nc * nc, 0.0);
    for (int l = 0; l < nc; l++) {
        C[(size_t)l * nc] = 1.0;
        for (int m = 1; m <= l; m++)
            C[(size_t)l * nc + m] = C[(size_t)(l - 1) * nc + m - 1] + (m < l ? C[(size_t)(l - 1) * nc + m] : 0.0);
    }
    std::vector<float2> h((size_t)4 * kSlots * P1 * P1, make_float2(0.f, 0.f));
    for (int c = 0; c < 4; c++)
        for (int k = 0; k < kSlots; k++) {
            const double tx = st.dx[c][k], ty = st.dy[c][k];
            const double tn = 1.0 / (tx * tx + ty * ty);
            const double2 w2 = make_double2(tx * tn, -ty * tn), w1 = make_double2(-w2.x, -w2.y);
            float2 *Tk = h.data() + ((size_t)c * kSlots + k) * P1 * P1;
            double2 w2i = make_double2(1.0, 0.0);
            for (int i = 0; i <= p; i++) {
                double2 w1j = make_double2(1.0, 0.0);
                for (int j = 0; j <= p; j++) {
                    double b;
                    if (i == 0)
                        b = j == 0 ? 0.0 : 1.0;
                    else
                        b = j == 0 ? -1.0 / i : C[(size_t)(i + j - 1) * nc + (j - 1)];
                    double2 v = cscal(cmul(w2i, w1j), b);
                    if (i == 0 && j == 0) v = make_double2(0.5 * std::log(tx * tx + ty * ty), 0.0);
                    Tk[i * P1 + j] = make_float2((float)v.x, (float)v.y);
                    w1j = cmul(w1j, w1);
                }
                w2i = cmul(w2i, w2);
            }
        }
    float2 *d = nullptr;
    FMM_CUDA(cudaMalloc(&d, h.size() * sizeof(float2)));
    FMM_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaStreamSynchronize(s));
    cache.push_back({key, d});
    return d;
}

template <int P1, int NR = P1>
void launch_fp32(const M2LWork &w, const Tree &T, const CauchyProblem &P, const float2 *Tab,
                 const float2 *mp32, double2 *loc, cudaStream_t s) {
    const int blocks = std::max(1, std::min(w.ntiles, kNumSM * 16));
    const SegTable sg = w.seg();
    const int *boxes = (const int *)w.vals.get();
    for (int c0 = 0; c0 < P.ndc;) {
        if (P.ndc - c0 >= 2) {
            m2l_fp32_kernel<P1, 2, NR><<<blocks, kFp32Tile, 0, s>>>(
                sg, boxes, w.slots.get(), T.d_boxsize.get(), P.ndc, c0, P.p, Tab, mp32, loc,
                w.ntiles);
            c0 += 2;
        } else {
            m2l_fp32_kernel<P1, 1, NR><<<blocks, kFp32Tile, 0, s>>>(
                sg, boxes, w.slots.get(), T.d_boxsize.get(), P.ndc, c0, P.p, Tab, mp32, loc,
                w.ntiles);
            c0 += 1;
        }
        FMM_CHECK_LAUNCH();
    }
}

// ---------------------------------------------------------------------------
// M2L of the mixed mode on the 5th-generation tensor cores (tcgen05, kind
// tf32, operands in shared memory, accumulator in tensor memory).
//
// In real form the slot operator is the 2P x 2P block matrix
// [[Re T, -Im T], [Im T, Re T]] (P = p + 1) acting on [Re M; Im M].  A tile
// is 128 rows = 128 / CH target boxes x CH channels of one segment; for each
// of the 27 slots the block gathers the rows' source multipoles (A, 128 x
// KP, KP = 2P rounded up to 8) and copies the slot's matrix (B, KP x KP,
// stored N-rows x K as the MMA's K-major B) into shared memory, and one
// thread issues D += A_hi B_hi + A_hi B_lo + A_lo B_hi (3 x TF32 split:
// x = hi + lo, both TF32-rounded; about 22 significant bits) accumulating
// all slots in the same tensor-memory tile.  The rows are read back with
// tcgen05.ld and stored as FP64.  Waits on the MMA-completion barrier are
// bounded; a wait that runs out sets *err and the kernel returns after
// releasing its tensor memory.
//
// Shared-memory operands use the no-swizzle K-major layout: 8-row x 16-byte
// core matrices, contiguous 128 bytes each; core matrix (row group g, K
// chunk c) at ((c * G + g) * 128) bytes, G = rows / 8.  So SBO (between row
// groups) = 128 bytes and LBO (between K chunks) = G * 128 bytes.
// ---------------------------------------------------------------------------
constexpr int kTcRows = 128;
constexpr int kTcMaxKP = 40;
// longest wait for an MMA-completion barrier (the MMAs of one slot take
// microseconds)
constexpr uint64_t kTcWaitNs = 2000000000ull;

// Bounded wait for the barrier phase with the given parity.
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
    int never = 0;
    return mbar_wait_bounded(mbar, parity, &never, kTcWaitNs);
}

// byte offset of element (row, k) in a K-major no-swizzle operand of
// `rows` rows
__host__ __device__ __forceinline__ int tc_off(int row, int k, int rows) { return tc_fidx(row, k, rows) << 2; }

template <int CH, int HALF>
__global__ void __launch_bounds__(kTcRows, 1) m2l_tc_kernel(
    SegTable seg, const int *__restrict__ boxes, const int *__restrict__ slots,
    const double *__restrict__ bs, int ndc, int c0, int p,
    const float *__restrict__ Bimg, const float2 *__restrict__ T0,
    const float2 *__restrict__ mp32, double2 *__restrict__ loc, int ntiles,
    int *__restrict__ err) {
    constexpr int KP = 2 * HALF;  // [Re 0..HALF-1 | Im 0..HALF-1]
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    float *sAhi = reinterpret_cast<float *>(tc_smem);
    float *sAlo = sAhi + kTcRows * KP;
    float *sBhi = sAlo + kTcRows * KP;  // followed by the lo image
    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_tb[257];
    __shared__ unsigned s_mask;
    __shared__ float2 s_t0[kSlots * (kTcMaxKP / 2)];
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int e = tid; e <= seg.nseg && e < 257; e += blockDim.x) s_tb[e] = seg.tile_base[e];
    if (tid == 0) s_mask = 0u;
    const uint32_t mbar = smem_u32(&s_mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&s_tmem)),
                     "r"(64)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const int TPT = kTcRows / CH;
    const int P = p + 1, stride = P * ndc;
    const int nB4 = (2 * KP * KP) / 4;  // float4s of the two B images
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(KP >> 3) << 17) |
                           (8u << 24);
    const uint32_t aLBO = (kTcRows / 8) * 128, bLBO = (KP / 8) * 128, SBO = 128;
    const uint32_t aHi = smem_u32(sAhi), aLo = smem_u32(sAlo);
    const uint32_t bHi = smem_u32(sBhi), bLo = bHi + KP * KP * 4;
    uint32_t ncommit = 0;
    bool failed = false;
    int cp_loaded = -1;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int lo = 0, hi = seg.nseg;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_tb[mid] <= tile) lo = mid; else hi = mid;
        }
        const int sg = lo;
        const int qend = seg.start[sg] + seg.count[sg];
        const int q = seg.start[sg] + (tile - s_tb[sg]) * TPT + tid / CH;
        const int c = c0 + tid % CH;
        const bool valid = q < qend;
        const int cp = seg.cpos[sg];
        // the source of every slot for this row, and the tile's slot mask
        const int *qslots = slots + (size_t)(valid ? q : 0) * kSlots;
        unsigned mymask = 0u;
#pragma unroll
        for (int k = 0; k < kSlots; k++)
            if (valid && qslots[k] >= 0) mymask |= 1u << k;
        if (mymask) atomicOr(&s_mask, mymask);
        if (cp != cp_loaded) {  // row 0 of this position's 27 matrices
            for (int e = tid; e < kSlots * P; e += blockDim.x)
                s_t0[(e / P) * (kTcMaxKP / 2) + e % P] = T0[((size_t)cp * kSlots + e / P) * P + e % P];
        }
        cp_loaded = cp;
        __syncthreads();
        unsigned mask = s_mask;
        __syncthreads();  // all have read the mask; it is cleared for the next tile
        if (tid == 0) s_mask = 0u;
        float l0x = 0.f, l0y = 0.f;  // row 0 (L_0) on the CUDA cores
        float s0x = 0.f, s0y = 0.f;
        // registers holding the next slot's row and matrix part
        float2 mrow[HALF];
        float4 breg[(2 * KP * KP / 4 + kTcRows - 1) / kTcRows];
        auto prefetch = [&](int k) {
            const int sb = valid ? qslots[k] : -1;
            const float2 *M = mp32 + (size_t)(sb >= 0 ? sb : 0) * stride + c;
#pragma unroll
            for (int j = 0; j < HALF; j++)
                mrow[j] = (sb >= 0 && j < P) ? M[(size_t)j * ndc] : make_float2(0.f, 0.f);
            const float4 *src = reinterpret_cast<const float4 *>(
                Bimg + ((size_t)cp * kSlots + k) * 2 * KP * KP);
#pragma unroll
            for (int u = 0; u < (int)(sizeof(breg) / sizeof(float4)); u++) {
                const int e = tid + u * kTcRows;
                breg[u] = e < nB4 ? src[e] : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        };
        bool issued = false;
        if (mask) prefetch(__ffs(mask) - 1);
        while (mask) {
            const int k = __ffs(mask) - 1;
            mask &= mask - 1;
            // the previous slot's MMAs read the operand buffers
            if (ncommit > 0 && !tc_wait(mbar, (ncommit - 1) & 1)) failed = true;
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            // A row `tid`: [Re M_0..HALF-1 | Im M_0..HALF-1] (zero beyond p),
            // split into TF32 hi / lo
#pragma unroll
            for (int kc = 0; kc < KP; kc += 4) {
                float4 vh, vl;
                float *ph = &vh.x, *pl = &vl.x;
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int kk = kc + u;
                    const float v = kk < HALF ? mrow[kk].x : mrow[kk - HALF].y;
                    const float h = tc_tf32(v);
                    ph[u] = h;
                    pl[u] = tc_tf32(v - h);
                }
                const int off = tc_off(tid, kc, kTcRows) >> 2;
                *reinterpret_cast<float4 *>(sAhi + off) = vh;
                *reinterpret_cast<float4 *>(sAlo + off) = vl;
            }
            {
                float4 *dst = reinterpret_cast<float4 *>(sBhi);
#pragma unroll
                for (int u = 0; u < (int)(sizeof(breg) / sizeof(float4)); u++) {
                    const int e = tid + u * kTcRows;
                    if (e < nB4) dst[e] = breg[u];
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int ks = 0; ks < KP / 8; ks++) {
                    const uint32_t ao = 2 * ks * aLBO, bo = 2 * ks * bLBO;
                    tc_mma(tmem, tc_sdesc(aHi + ao, aLBO, SBO), tc_sdesc(bHi + bo, bLBO, SBO),
                           idesc, (issued || ks > 0) ? 1u : 0u);
                    tc_mma(tmem, tc_sdesc(aHi + ao, aLBO, SBO), tc_sdesc(bLo + bo, bLBO, SBO),
                           idesc, 1u);
                    tc_mma(tmem, tc_sdesc(aLo + ao, aLBO, SBO), tc_sdesc(bHi + bo, bLBO, SBO),
                           idesc, 1u);
                }
                tc_commit(mbar);
            }
            ncommit++;
            issued = true;
            // row 0 on the CUDA cores while the MMAs run, then the next slot
            if (valid && qslots[k] >= 0) {
                const float2 *t0 = s_t0 + k * (kTcMaxKP / 2);
#pragma unroll
                for (int j = 0; j < HALF; j++) {
                    if (j < P) {
                        const float2 t = t0[j], m = mrow[j];
                        l0x = fmaf(t.x, m.x, fmaf(-t.y, m.y, l0x));
                        l0y = fmaf(t.x, m.y, fmaf(t.y, m.x, l0y));
                    }
                }
                s0x += mrow[0].x;
                s0y += mrow[0].y;
            }
            if (mask) prefetch(__ffs(mask) - 1);
        }
        if (failed) break;
        float d[KP];
#pragma unroll
        for (int i = 0; i < KP; i++) d[i] = 0.f;
        if (issued) {
            if (!tc_wait(mbar, (ncommit - 1) & 1)) failed = true;
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
            for (int c8 = 0; c8 < KP / 8; c8++) {
                float v[8];
                tc_ld8(taddr + c8 * 8, v);
#pragma unroll
                for (int u = 0; u < 8; u++) d[c8 * 8 + u] = v[u];
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        }
        if (valid) {
            const int b = boxes[q];
            const double lr = log(bs[seg.level[sg]]);
#pragma unroll
            for (int i = 0; i < HALF; i++) {
                if (i < P) {
                    double re, im;
                    if (i == 0) {
                        re = (double)l0x + lr * s0x;
                        im = (double)l0y + lr * s0y;
                    } else {
                        re = d[i];
                        im = d[HALF + i];
                    }
                    loc[(size_t)b * stride + (size_t)i * ndc + c] = make_double2(re, im);
                }
            }
        }
        // the next tile's MMAs overwrite the accumulator
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) atomicExch(err, 1);
        // let MMAs still in flight finish before the memory is released
        if (ncommit > 0) tc_wait(mbar, (ncommit - 1) & 1);
    }
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64)
                     : "memory");
    }
}

// B images per (child position, slot): the real form of T (rows = outputs
// i, K = inputs j), TF32 hi and lo, in the operand layout; cached per
// device and order.
float tf32_round_host(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

// Also returns (t0) row 0 of each matrix, P complex FP32 values per
// (child position, slot), for the CUDA-core L_0 sum.
const float *tc_tables(int p, int KP, cudaStream_t s, const float2 **t0out) {
    static std::mutex mu;
    static std::vector<std::pair<long, const float *>> cache;
    static std::vector<std::pair<long, const float2 *>> cache0;
    int dev;
    FMM_CUDA(cudaGetDevice(&dev));
    const long key = ((long)dev << 20) | ((long)p << 8) | KP;
    std::lock_guard<std::mutex> g(mu);
    for (size_t e = 0; e < cache.size(); e++)
        if (cache[e].first == key) {
            *t0out = cache0[e].second;
            return cache[e].second;
        }
    const int P = p + 1;
    const SlotTables st = make_slot_tables();
    std::vector<float2> t0h((size_t)4 * kSlots * P);
    const int nc = 2 * P + 2;
    std::vector<double> C((size_t)nc * nc, 0.0);
    for (int l = 0; l < nc; l++) {
        C[(size_t)l * nc] = 1.0;
        for (int m = 1; m <= l; m++)
            C[(size_t)l * nc + m] =
                C[(size_t)(l - 1) * nc + m - 1] + (m < l ? C[(size_t)(l - 1) * nc + m] : 0.0);
    }
    std::vector<float> h((size_t)4 * kSlots * 2 * KP * KP, 0.f);
    std::vector<double2> T((size_t)P * P);
    for (int cp = 0; cp < 4; cp++)
        for (int k = 0; k < kSlots; k++) {
            const double tx = st.dx[cp][k], ty = st.dy[cp][k];
            const double tn = 1.0 / (tx * tx + ty * ty);
            const double2 w2 = make_double2(tx * tn, -ty * tn), w1 = make_double2(-w2.x, -w2.y);
            double2 w2i = make_double2(1.0, 0.0);
            for (int i = 0; i < P; i++) {
                double2 w1j = make_double2(1.0, 0.0);
                for (int j = 0; j < P; j++) {
                    double b;
                    if (i == 0)
                        b = j == 0 ? 0.0 : 1.0;
                    else
                        b = j == 0 ? -1.0 / i : C[(size_t)(i + j - 1) * nc + (j - 1)];
                    double2 v = cscal(cmul(w2i, w1j), b);
                    if (i == 0 && j == 0) v = make_double2(0.5 * std::log(tx * tx + ty * ty), 0.0);
                    T[(size_t)i * P + j] = v;
                    w1j = cmul(w1j, w1);
                }
                w2i = cmul(w2i, w2);
            }
            float *hi = h.data() + ((size_t)cp * kSlots + k) * 2 * KP * KP;
            float *lo = hi + KP * KP;
            float2 *t0 = t0h.data() + ((size_t)cp * kSlots + k) * P;
            for (int j = 0; j < P; j++)
                t0[j] = make_float2((float)T[j].x, (float)T[j].y);
            // rows / columns [Re 0..HALF-1 | Im 0..HALF-1], zero beyond p;
            // row 0 (L_0) is summed on the CUDA cores: rows 0 and HALF stay zero
            const int HALF = KP / 2;
            for (int n = 0; n < KP; n++)
                for (int kk = 0; kk < KP; kk++) {
                    const int i = n < HALF ? n : n - HALF, j = kk < HALF ? kk : kk - HALF;
                    if (i == 0 || i >= P || j >= P) continue;
                    const double2 t = T[(size_t)i * P + j];
                    double v;
                    if (n < HALF) v = kk < HALF ? t.x : -t.y;
                    else v = kk < HALF ? t.y : t.x;
                    const float f = (float)v;
                    const float fh = tf32_round_host(f);
                    const int off = tc_off(n, kk, KP) >> 2;
                    hi[off] = fh;
                    lo[off] = tf32_round_host(f - fh);
                }
        }
    float *d = nullptr;
    float2 *d0 = nullptr;
    FMM_CUDA(cudaMalloc(&d, h.size() * sizeof(float)));
    FMM_CUDA(cudaMalloc(&d0, t0h.size() * sizeof(float2)));
    FMM_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaMemcpyAsync(d0, t0h.data(), t0h.size() * sizeof(float2), cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaStreamSynchronize(s));
    cache.push_back({key, d});
    cache0.push_back({key, d0});
    *t0out = d0;
    return d;
}

}  // namespace

bool m2l_tensor_fp64(const Tree &T, const CauchyProblem &P, const double2 *mp,
                     double2 *loc, cudaStream_t s) {
    const int L = T.nlevels, p = P.p;
    if (L < 2 || p > 63) return false;
    bool ok = false;
    const auto wp = m2l_cached<M2LWork>(P.m2l_cache, m2l_key(1, 8, 0), ok,
                                        [&](M2LWork &x) { return m2l_work(T, P, 8, s, x); });
    if (!ok) return false;
    const M2LWork &w = *wp;
    if (w.ntiles == 0) return true;
    const SegTable sg = w.seg();
    const int *boxes = (const int *)w.vals.get();
    const double *bs = T.d_boxsize.get();
    const double *binom = device_binomials(s);
    const int ntiles = w.ntiles;
    const int ks = (p + 1 + 3) / 4;
    const int mt = (p + 1 + 7) / 8;
#define FMM_M2L_CASE(MT_, KS_)                                                   \
    if (mt <= MT_ && ks <= KS_) {                                                \
        launch_dmma<MT_, KS_>(sg, boxes, w.slots.get(), bs, P.ndc, p, binom, mp, \
                              loc, ntiles, s);                                   \
        return true;                                                             \
    }
    FMM_M2L_CASE(2, 4)
    FMM_M2L_CASE(3, 5)
    FMM_M2L_CASE(3, 6)
    FMM_M2L_CASE(4, 8)
    FMM_M2L_CASE(5, 10)
    FMM_M2L_CASE(6, 12)
    FMM_M2L_CASE(8, 16)
#undef FMM_M2L_CASE
    return false;
}

// ---------------------------------------------------------------------------
// Split-precision M2L (eps below the mixed mode's range, all other passes
// FP64).  The scaled shift's terms T_ij M_j fall off with the total order
// n = i + j: for the nearest list-2 offsets (|t| = 2) and points at the
// box corners their share of the potential is about 0.707^n, and measured
// errors fall about 8x per 4 orders.  The leading triangle i + j < NT runs
// in FP64 on the DMMA kernel (the first writer of every local); the tail
// i + j >= NT runs as TF32 x 3 slot GEMMs on the tcgen05 tensor cores
// (slot_gemm_tc_level, about 2^-22 relative per product, one FP32
// accumulation over a tile's slots: the tail is small beside the result)
// and is added on top.  The tail's error falls about 0.59x per order of NT
// and eps about 0.47x per order of p, so NT grows faster than p:
// NT = 4 (p - 13) / 3 + 2 (rounded up to a multiple of 4) holds gradients
// and Hessians on clustered points within eps of the FP64 mode at 1e-9
// (p = 28, NT = 24) and 1e-10 (p = 31, NT = 28; 24 left Hessians 1.15e-10
// off).  At 1e-12 (p = 37) even NT = 32 left the Hessians of clustered
// points at 2e-11, twenty times the FP64 mode's error: orders above 31 keep
// the FP64 M2L.
// ---------------------------------------------------------------------------

// The tail images (i + j >= nt) of the 4 x 27 slot operators in real form,
// T_ij = w2^i B_ij w1^j (w2 = 1/t, w1 = -1/t, t the slot offset), TF32
// split; cached per device, order and nt.
const float *split_tail_tables(int p, int KP, int nt, cudaStream_t s) {
    static std::mutex mu;
    static std::vector<std::pair<long, const float *>> cache;
    int dev;
    FMM_CUDA(cudaGetDevice(&dev));
    const long key = ((long)dev << 24) | ((long)nt << 16) | ((long)p << 8) | KP;
    std::lock_guard<std::mutex> g(mu);
    for (auto &e : cache)
        if (e.first == key) return e.second;
    const int W = p + 1, nc = 2 * W + 2;
    std::vector<double> C((size_t)nc * nc, 0.0);
    for (int l = 0; l < nc; l++) {
        C[(size_t)l * nc] = 1.0;
        for (int m = 1; m <= l; m++)
            C[(size_t)l * nc + m] =
                C[(size_t)(l - 1) * nc + m - 1] + (m < l ? C[(size_t)(l - 1) * nc + m] : 0.0);
    }
    const SlotTables st = make_slot_tables();
    const size_t per = (size_t)(KP / 16) * 2 * KP * 16;  // floats per (position, slot)
    std::vector<float> h((size_t)4 * kSlots * per, 0.f);
    std::vector<double2> T((size_t)W * W);
    for (int cp = 0; cp < 4; cp++)
        for (int k = 0; k < kSlots; k++) {
            const double tx = st.dx[cp][k], ty = st.dy[cp][k];
            const double tn = 1.0 / (tx * tx + ty * ty);
            const double2 w2 = make_double2(tx * tn, -ty * tn), w1 = make_double2(-w2.x, -w2.y);
            double2 w2i = make_double2(1.0, 0.0);
            for (int i = 0; i < W; i++) {
                double2 w1j = make_double2(1.0, 0.0);
                for (int j = 0; j < W; j++) {
                    double b;
                    if (i == 0)
                        b = j == 0 ? 0.0 : 1.0;
                    else
                        b = j == 0 ? -1.0 / i : C[(size_t)(i + j - 1) * nc + (j - 1)];
                    T[(size_t)i * W + j] =
                        i + j >= nt ? cscal(cmul(w2i, w1j), b) : make_double2(0.0, 0.0);
                    w1j = cmul(w1j, w1);
                }
                w2i = cmul(w2i, w2);
            }
            float *img = h.data() + (size_t)(cp * kSlots + k) * per;
            for (int n = 0; n < 2 * W; n++)
                for (int kk = 0; kk < 2 * W; kk++) {
                    const double2 t = T[(size_t)(n < W ? n : n - W) * W + (kk < W ? kk : kk - W)];
                    const bool re_out = n < W, re_in = kk < W;
                    const double v = re_out ? (re_in ? t.x : -t.y) : (re_in ? t.y : t.x);
                    const float f = (float)v, fh = tf32_round_host(f);
                    const size_t at = slot_bimg_at(n, kk, KP);
                    img[at] = fh;
                    img[at + (size_t)KP * 16] = tf32_round_host(f - fh);
                }
        }
    float *d = nullptr;
    FMM_CUDA(cudaMalloc(&d, h.size() * sizeof(float)));
    FMM_CUDA(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaStreamSynchronize(s));
    cache.push_back({key, d});
    return d;
}

// The FP64 triangle on the DMMA kernel for the supported (MT, KS, NT).
template <int NT>
bool launch_split_triangle(const SegTable &sg, const int *boxes, const int *slots, const double *bs,
                           int ndc, int p, const double *binom, const double2 *mp, double2 *loc,
                           int ntiles, cudaStream_t s) {
    const int ks = (p + 1 + 3) / 4, mt = (p + 1 + 7) / 8;
#define FMM_SPLIT_CASE(MT_, KS_)                                                           \
    if (mt <= MT_ && ks <= KS_) {                                                          \
        launch_dmma<MT_, KS_, NT>(sg, boxes, slots, bs, ndc, p, binom, mp, loc, ntiles, s); \
        return true;                                                                       \
    }
    FMM_SPLIT_CASE(4, 8)
    FMM_SPLIT_CASE(5, 10)
    FMM_SPLIT_CASE(6, 12)
#undef FMM_SPLIT_CASE
    return false;
}

namespace {
struct SplitHold {
    SlotPlan spl;
};
}  // namespace

// 0: the order keeps the FP64 M2L
int split_triangle_order(int p) {
    const char *e = getenv("FMM2D_B200_SPLIT_NT");
    if (!e && p > 31) return 0;
    int nt = e ? atoi(e) : (4 * (p - 13) + 2) / 3 + 2;
    // the supported triangles: 8, 12, ..., 32
    if (nt < 8) nt = 8;
    nt = (nt + 3) / 4 * 4;
    return nt > 32 ? 0 : nt;
}

bool m2l_split_fp64(const Tree &T, const CauchyProblem &P, const double2 *mp, double2 *loc,
                    cudaStream_t s) {
    const int L = T.nlevels, p = P.p, W = p + 1;
    if (L < 2 || W < 20 || W > 48 || P.ndc > 128) return false;
    const int KP = slot_gemm_kp(W);
    const int nt = split_triangle_order(p);
    if (KP == 0 || nt == 0 || nt >= 2 * W - 1) return false;
    // planning first (nothing is launched when it fails)
    bool ok = false;
    const auto wp = m2l_cached<M2LWork>(P.m2l_cache, m2l_key(1, 8, 0), ok,
                                        [&](M2LWork &x) { return m2l_work(T, P, 8, s, x); });
    if (!ok) return false;
    bool ok2 = false;
    const int tpt = 128 / P.ndc;
    const auto hp = m2l_cached<SplitHold>(P.m2l_cache, m2l_key(6, tpt, 0), ok2, [&](SplitHold &x) {
        return plan_slots(T, P.sset.pgh, P.tset.pgh, tpt, s, x.spl);
    });
    if (!ok2) return false;
    const M2LWork &w = *wp;
    if (w.ntiles == 0) return true;
    const float *bimg = split_tail_tables(p, KP, nt, s);
    // 1. the FP64 triangle, storing every local of levels >= 2 with points
    const double *binom = device_binomials(s);
    const SegTable sg = w.seg();
    const int *boxes = (const int *)w.vals.get();
    const double *bs = T.d_boxsize.get();
    bool launched = false;
    switch (nt) {
        case 8: launched = launch_split_triangle<8>(sg, boxes, w.slots.get(), bs, P.ndc, p, binom, mp, loc, w.ntiles, s); break;
        case 12: launched = launch_split_triangle<12>(sg, boxes, w.slots.get(), bs, P.ndc, p, binom, mp, loc, w.ntiles, s); break;
        case 16: launched = launch_split_triangle<16>(sg, boxes, w.slots.get(), bs, P.ndc, p, binom, mp, loc, w.ntiles, s); break;
        case 20: launched = launch_split_triangle<20>(sg, boxes, w.slots.get(), bs, P.ndc, p, binom, mp, loc, w.ntiles, s); break;
        case 24: launched = launch_split_triangle<24>(sg, boxes, w.slots.get(), bs, P.ndc, p, binom, mp, loc, w.ntiles, s); break;
        case 28: launched = launch_split_triangle<28>(sg, boxes, w.slots.get(), bs, P.ndc, p, binom, mp, loc, w.ntiles, s); break;
        case 32: launched = launch_split_triangle<32>(sg, boxes, w.slots.get(), bs, P.ndc, p, binom, mp, loc, w.ntiles, s); break;
        default: break;
    }
    if (!launched) return false;
    prof_set_count("m2l_split_nt", (double)nt);
    // 2. the tail on the tensor cores, level by level, added to the locals
    M2LCache *cache = P.m2l_cache;
    const bool deferred = cache && cache->deferred;
    DevBuf<int> err_own;
    if (!deferred) {
        err_own.alloc(1, s);
        FMM_CUDA(cudaMemsetAsync(err_own.get(), 0, sizeof(int), s));
    }
    int *errp = deferred ? cache->err : err_own.get();
    const size_t stride = (size_t)W * P.ndc;
    long long maxbox = 0;
    for (int l = 2; l <= L; l++) maxbox = std::max<long long>(maxbox, T.lend[l] - T.lstart[l]);
    DevBuf<float> arow((size_t)maxbox * P.ndc * 2 * KP, s);
    for (int l = 2; l <= L; l++) {
        const int g0 = 4 * (l - 2);
        if (g0 + 4 > hp->spl.nseg || hp->spl.tile_base[g0 + 4] == hp->spl.tile_base[g0]) continue;
        const int lo = T.lstart[l], nb = T.lend[l] - lo;
        slot_gemm_rows((long long)nb * P.ndc, P.ndc, W, KP, mp + (size_t)lo * stride, arow.get(), s);
        SlotGemmLevel g;
        g.level = l;
        g.lstart = lo;
        g.nd = P.ndc;
        g.W = W;
        g.KP = KP;
        g.arow = arow.get();
        g.bimg = bimg;
        g.out = loc + (size_t)lo * stride;
        g.oscale = 1.0;
        g.group = 27;
        if (!slot_gemm_tc_level(g, hp->spl, errp, s))
            throw FmmError(4, "split-precision M2L: unsupported tensor-core level shape");
    }
    if (!deferred && read_scalar(errp, s) != 0)
        throw FmmError(4, "tensor-core M2L: a wait for an MMA or operand barrier timed out");
    return true;
}

namespace {
struct SlotHold {
    M2LWork w;
    DevBuf<int2> dxy;
};
}  // namespace

bool plan_slots(const Tree &T, int spgh, int tpgh, int tile, cudaStream_t s, SlotPlan &sp) {
    sp = SlotPlan();
    if (T.nlevels < 2) return true;
    CauchyProblem P;
    P.sset.pgh = spgh;
    P.tset.pgh = tpgh;
    auto h = std::make_shared<SlotHold>();
    if (!m2l_work(T, P, tile, s, h->w)) return false;
    const M2LWork &w = h->w;
    sp.nseg = w.nseg;
    sp.ntarg = w.ntarg;
    sp.ntiles = w.ntiles;
    if (w.ntiles == 0) return true;
    const int n = w.nseg;
    sp.tile_base.assign(w.hseg.begin(), w.hseg.begin() + n + 1);
    sp.start.assign(w.hseg.begin() + n + 1, w.hseg.begin() + 2 * n + 1);
    sp.count.assign(w.hseg.begin() + 2 * n + 1, w.hseg.begin() + 3 * n + 1);
    const SlotTables st = make_slot_tables();
    std::vector<int2> d(4 * kSlots);
    for (int c = 0; c < 4; c++)
        for (int k = 0; k < kSlots; k++) d[c * kSlots + k] = make_int2(st.dx[c][k], st.dy[c][k]);
    h->dxy.alloc(d.size(), s);
    FMM_CUDA(cudaMemcpyAsync(h->dxy.get(), d.data(), d.size() * sizeof(int2),
                             cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaStreamSynchronize(s));  // (d is a pageable host vector)
    sp.boxes = (const int *)w.vals.get();
    sp.slots = w.slots.get();
    sp.dxy = h->dxy.get();
    sp.hold = h;
    return true;
}

namespace {
std::atomic<int> g_m2l_form[128];
}

// Form of the mixed-mode M2L for order p: FMM2D_B200_M2L ("simt", "tile"),
// else the setting for the order (fmm2d_b200_set_m2l_form, the autotuner),
// else windows on the tensor cores for the dense levels with slot tables
// for the rest.
int m2l_form(int p) {
    const char *mode = getenv("FMM2D_B200_M2L");
    if (mode && !strcmp(mode, "simt")) return kM2LSimt;
    if (mode && !strcmp(mode, "tile")) return kM2LTile;
    return (p >= 0 && p < 128) ? g_m2l_form[p].load() : kM2LWindow;
}

void set_m2l_form(int p, int form) {
    if (p >= 0 && p < 128) g_m2l_form[p].store(form);
}

bool m2l_fp32(const Tree &T, const CauchyProblem &P, const double2 *mp, double2 *loc,
              cudaStream_t s, float2 *mp32_out) {
    const int L = T.nlevels, p = P.p;
    if (L < 2 || p + 1 > 20) return false;
    const int form = m2l_form(p);
    const bool simt = form == kM2LSimt;
    const bool tile_only = form == kM2LTile;
    const int CH = P.ndc >= 2 ? 2 : 1;
    // FP32 copy of the multipoles of levels >= 2
    const int lo = T.lstart[2];
    const size_t stride = (size_t)(p + 1) * P.ndc;
    const size_t nv = (size_t)(T.nboxes - lo) * stride;
    DevBuf<float2> mp32_own;
    if (!mp32_out) mp32_own.alloc((size_t)T.nboxes * stride, s);
    float2 *mp32p = mp32_out ? mp32_out : mp32_own.get();
    {
        const double2 *src = mp + (size_t)lo * stride;
        float2 *dst = mp32p + (size_t)lo * stride;
        for_each((int64_t)nv, s, [=] __device__(int64_t i) {
            dst[i] = make_float2((float)src[i].x, (float)src[i].y);
        });
    }
    // the bounded waits' error flag: read at the end, or by the caller in
    // the deferred mode
    M2LCache *cache = P.m2l_cache;
    const bool deferred = cache && cache->deferred;
    DevBuf<int> err_own;
    if (!deferred) err_own.alloc(1, s);
    int *errp = deferred ? cache->err : err_own.get();
    FMM_CUDA(cudaMemsetAsync(errp, 0, sizeof(int), s));
    const uint64_t done =
        (simt || tile_only) ? 0 : m2l_window_fp32(T, P, mp32p, loc, errp, s);
    const int wtile = simt ? kFp32Tile : kTcRows / CH;
    bool ok = false;
    const auto wp = m2l_cached<M2LWork>(cache, m2l_key(3, wtile, done), ok,
                                        [&](M2LWork &x) { return m2l_work(T, P, wtile, s, x, done); });
    if (!ok) return false;
    const M2LWork &w = *wp;
    if (w.ntiles > 0 && simt) {
        if (p + 1 <= 12)
            launch_fp32<12>(w, T, P, fp32_tables(p, 12, s), mp32p, loc, s);
        else
            launch_fp32<20>(w, T, P, fp32_tables(p, 20, s), mp32p, loc, s);
    } else if (w.ntiles > 0) {
        // tensor cores: K = N = 2 HALF with HALF = 12 (p < 12) or 20
        const int HALF = p + 1 <= 12 ? 12 : 20;
        const int KP = 2 * HALF;
        const float2 *tab0 = nullptr;
        const float *tab = tc_tables(p, KP, s, &tab0);
        const size_t smem = (size_t)(2 * kTcRows * KP + 2 * KP * KP) * sizeof(float);
        auto launch = [&](auto kern, const M2LWork &ww, int c0) {
            raise_smem_limit(kern, (int)smem);
            const int blocks = std::max(1, std::min(ww.ntiles, kNumSM * 4));
            kern<<<blocks, kTcRows, smem, s>>>(ww.seg(), (const int *)ww.vals.get(), ww.slots.get(),
                                               T.d_boxsize.get(), P.ndc, c0, p, tab, tab0,
                                               mp32p, loc, ww.ntiles, errp);
            FMM_CHECK_LAUNCH();
        };
        int c0 = 0;
        if (CH == 2) {
            for (; P.ndc - c0 >= 2; c0 += 2) {
                if (HALF == 12) launch(m2l_tc_kernel<2, 12>, w, c0);
                else launch(m2l_tc_kernel<2, 20>, w, c0);
            }
        }
        if (c0 < P.ndc) {
            // remaining single channels, one channel per row
            std::shared_ptr<M2LWork> w1;
            const M2LWork *pw = &w;
            if (CH != 1) {
                bool ok1 = false;
                w1 = m2l_cached<M2LWork>(cache, m2l_key(4, kTcRows, done), ok1, [&](M2LWork &x) {
                    return m2l_work(T, P, kTcRows, s, x, done);
                });
                if (!ok1) return false;
                pw = w1.get();
            }
            for (; c0 < P.ndc; c0++) {
                if (HALF == 12) launch(m2l_tc_kernel<1, 12>, *pw, c0);
                else launch(m2l_tc_kernel<1, 20>, *pw, c0);
            }
        }
    }
    if (!deferred && read_scalar(errp, s) != 0)
        throw FmmError(4, "tensor-core M2L: a wait for an MMA or operand barrier timed out");
    // A TF32 x 3 product is accurate to about 2^-22, four times an FP32
    // product.  Measured on 10^5 uniform charges at eps 1e-6 (order 18),
    // the gradient at the sources then has a relative error of 1.6e-6 with
    // the tensor-core forms against 2.0e-7 with the FP32 CUDA-core form.
    // From order kM2LExactFrom on, the leading kM2LExactRows local
    // coefficients -- L_0 .. L_3, which carry most of the gradient at a
    // leaf's points -- are therefore recomputed in FP32 on the CUDA cores:
    // on the window levels from the windows (m2l_window.cu), on the other
    // levels here with the slot tables.
    if (!simt && m2l_exact_rows(p)) {
        bool okr = false;
        const auto wr = m2l_cached<M2LWork>(cache, m2l_key(5, kFp32Tile, done), okr,
                                            [&](M2LWork &x) {
                                                return m2l_work(T, P, kFp32Tile, s, x, done);
                                            });
        if (!okr) return false;
        if (wr->ntiles > 0) {
            const bool hess = std::max(P.sset.n > 0 ? P.sset.pgh : 0, P.tset.n > 0 ? P.tset.pgh : 0) >= 3;
            if (hess)
                launch_fp32<20, kM2LExactRowsHess>(*wr, T, P, fp32_tables(p, 20, s), mp32p, loc, s);
            else
                launch_fp32<20, kM2LExactRows>(*wr, T, P, fp32_tables(p, 20, s), mp32p, loc, s);
        }
    }
    return true;
}

}  // namespace fmm2d
