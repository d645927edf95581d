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

#include <algorithm>
#include <mutex>
#include <stdlib.h>
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

template <int MT, int KS, int CH>
__global__ void __launch_bounds__(128, 4) m2l_dmma_kernel(
    SegTable seg, const int *__restrict__ boxes, const int *__restrict__ slots,
    const double *__restrict__ bs, int ndc, int c0, int p,
    const double *__restrict__ binom, const double2 *__restrict__ mp,
    double2 *__restrict__ loc, int ntiles) {
    // A-operand fragments of B: [mt][ks][lane]
    __shared__ double s_a[MT * KS * 32];
    __shared__ int s_tb[257];
    for (int e = threadIdx.x; e < MT * KS * 32; e += blockDim.x) {
        const int l = e & 31, ks = (e >> 5) % KS, mt = (e >> 5) / KS;
        const int i = mt * 8 + (l >> 2), j = ks * 4 + (l & 3);
        double v = 0.0;
        if (i <= p && j <= p) {
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
                    if (sg_box >= 0 && j <= p)
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
                        const double a = s_a[(mt * KS + ks) * 32 + lane];
                        dmma(tre[mt][0], tre[mt][1], a, bre[ks]);
                        dmma(tim[mt][0], tim[mt][1], a, bim[ks]);
                    }
                }
                double2 wi = w2p;
#pragma unroll
                for (int mt = 0; mt < MT; mt++) {
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

template <int MT, int KS>
void launch_dmma(const SegTable &sg, const int *boxes, const int *slots,
                 const double *bs, int ndc, int p, const double *binom,
                 const double2 *mp, double2 *loc, int ntiles, cudaStream_t s) {
    const int blocks = std::max(1, std::min((ntiles + 3) / 4, kNumSM * 16));
    const char *e = getenv("FMM2D_B200_M2L_CH2");
    const bool ch2 = e && e[0] == '1';
    for (int c0 = 0; c0 < ndc;) {
        if (ch2 && ndc - c0 >= 2 && MT <= 5) {
            m2l_dmma_kernel<MT, KS, 2><<<blocks, 128, 0, s>>>(
                sg, boxes, slots, bs, ndc, c0, p, binom, mp, loc, ntiles);
            c0 += 2;
        } else {
            m2l_dmma_kernel<MT, KS, 1><<<blocks, 128, 0, s>>>(
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
    int nseg = 0, ntarg = 0, ntiles = 0;
    SegTable seg() const {
        const int *h = segd.get();
        return SegTable{h, h + nseg + 1, h + 2 * nseg + 1, h + 3 * nseg + 1, h + 4 * nseg + 1,
                        nseg};
    }
};

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

// Builds the segments (tiles of `tile` boxes) and the slot table; false
// when a list-2 entry falls outside the 27 slots or there are too many
// segments.
bool m2l_work(const Tree &T, const CauchyProblem &P, int tile, cudaStream_t s, M2LWork &w) {
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
        if (np > 0) {
            const int pb = par[b];
            int c = 0;
            for (int j = 0; j < 4; j++)
                if (chi[4 * pb + j] == b) c = j;
            key = (lev[b] - 2) * 4 + c;
        }
        kp[i] = (uint32_t)key;
        vp[i] = (uint32_t)b;
        atomicAdd(&cp[key], 1);
    });
    int bits = 1;
    while ((1 << bits) <= nseg) bits++;
    radix_sort_pairs(kp, vp, w.kt.get(), w.vt.get(), n, bits, s);
    std::vector<int> hc(nseg + 1);
    FMM_CUDA(cudaMemcpyAsync(hc.data(), cp, (nseg + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    FMM_CUDA(cudaStreamSynchronize(s));
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
constexpr int kFp32Tile = 128;

template <int P1, int CH>
__global__ void __launch_bounds__(kFp32Tile) m2l_fp32_kernel(
    SegTable seg, const int *__restrict__ boxes, const int *__restrict__ slots,
    const double *__restrict__ bs, int ndc, int c0, int p, const float2 *__restrict__ Tall,
    const float2 *__restrict__ mp32, double2 *__restrict__ loc, int ntiles) {
    __shared__ float2 sT[P1 * P1];
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
        float2 acc[CH][P1];
        float2 s0[CH];
#pragma unroll
        for (int c = 0; c < CH; c++) {
            s0[c] = make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 0; i < P1; i++) acc[c][i] = make_float2(0.f, 0.f);
        }
        for (int k = 0; k < kSlots; k++) {
            __syncthreads();  // the previous slot's matrix is no longer read
            const float2 *Tk = Tall + ((size_t)cp * kSlots + k) * P1 * P1;
            for (int e = threadIdx.x; e < P1 * P1; e += blockDim.x) sT[e] = Tk[e];
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
                for (int i = 0; i < P1; i++) {
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
            for (int i = 0; i < P1; i++) {
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

template <int P1>
void launch_fp32(const M2LWork &w, const Tree &T, const CauchyProblem &P, const float2 *Tab,
                 const float2 *mp32, double2 *loc, cudaStream_t s) {
    const int blocks = std::max(1, std::min(w.ntiles, kNumSM * 16));
    const SegTable sg = w.seg();
    const int *boxes = (const int *)w.vals.get();
    for (int c0 = 0; c0 < P.ndc;) {
        if (P.ndc - c0 >= 2) {
            m2l_fp32_kernel<P1, 2><<<blocks, kFp32Tile, 0, s>>>(
                sg, boxes, w.slots.get(), T.d_boxsize.get(), P.ndc, c0, P.p, Tab, mp32, loc,
                w.ntiles);
            c0 += 2;
        } else {
            m2l_fp32_kernel<P1, 1><<<blocks, kFp32Tile, 0, s>>>(
                sg, boxes, w.slots.get(), T.d_boxsize.get(), P.ndc, c0, P.p, Tab, mp32, loc,
                w.ntiles);
            c0 += 1;
        }
        FMM_CHECK_LAUNCH();
    }
}

}  // namespace

bool m2l_tensor_fp64(const Tree &T, const CauchyProblem &P, const double2 *mp,
                     double2 *loc, cudaStream_t s) {
    const int L = T.nlevels, p = P.p;
    if (L < 2 || p > 63) return false;
    M2LWork w;
    if (!m2l_work(T, P, 8, s, w)) return false;
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

bool m2l_fp32(const Tree &T, const CauchyProblem &P, const double2 *mp, double2 *loc,
              cudaStream_t s) {
    const int L = T.nlevels, p = P.p;
    if (L < 2 || p + 1 > 20) return false;
    M2LWork w;
    if (!m2l_work(T, P, kFp32Tile, s, w)) return false;
    if (w.ntiles == 0) return true;
    // FP32 copy of the multipoles of levels >= 2
    const int lo = T.lstart[2];
    const size_t stride = (size_t)(p + 1) * P.ndc;
    const size_t nv = (size_t)(T.nboxes - lo) * stride;
    DevBuf<float2> mp32((size_t)T.nboxes * stride, s);
    {
        const double2 *src = mp + (size_t)lo * stride;
        float2 *dst = mp32.get() + (size_t)lo * stride;
        for_each((int64_t)nv, s, [=] __device__(int64_t i) {
            dst[i] = make_float2((float)src[i].x, (float)src[i].y);
        });
    }
    if (p + 1 <= 12)
        launch_fp32<12>(w, T, P, fp32_tables(p, 12, s), mp32.get(), loc, s);
    else
        launch_fp32<20>(w, T, P, fp32_tables(p, 20, s), mp32.get(), loc, s);
    return true;
}

}  // namespace fmm2d
