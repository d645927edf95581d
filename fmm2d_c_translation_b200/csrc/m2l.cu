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

}  // namespace

bool m2l_tensor_fp64(const Tree &T, const CauchyProblem &P, const double2 *mp,
                     double2 *loc, cudaStream_t s) {
    const int L = T.nlevels, p = P.p;
    if (L < 2 || p > 63) return false;
    static std::mutex tables_mu;
    static bool tables_ready[64] = {false};
    int dev = 0;
    FMM_CUDA(cudaGetDevice(&dev));
    std::unique_lock<std::mutex> tables_lock(tables_mu);
    if (!tables_ready[dev]) {
        const SlotTables st = make_slot_tables();
        FMM_CUDA(cudaMemcpyToSymbolAsync(c_slot_dx, st.dx, sizeof(st.dx), 0, cudaMemcpyHostToDevice, s));
        FMM_CUDA(cudaMemcpyToSymbolAsync(c_slot_dy, st.dy, sizeof(st.dy), 0, cudaMemcpyHostToDevice, s));
        FMM_CUDA(cudaMemcpyToSymbolAsync(c_slot_of, st.slot_of, sizeof(st.slot_of), 0, cudaMemcpyHostToDevice, s));
        FMM_CUDA(cudaStreamSynchronize(s));
        tables_ready[dev] = true;
    }
    tables_lock.unlock();
    const int lo = T.lstart[2], n = T.nboxes - lo;
    const int nseg = 4 * (L - 1);
    const int2 *sse = T.srcse.get(), *tse = T.trgse.get();
    const int spgh = P.sset.pgh, tpgh = P.tset.pgh;
    const int *lev = T.level.get(), *par = T.parent.get(), *chi = T.child.get();
    // ---- keys: (level - 2) * 4 + child position, or nseg when not a target
    DevBuf<uint32_t> keys(n, s), vals(n, s), kt(n, s), vt(n, s);
    DevBuf<int> cnt(nseg + 1, s);
    cnt.zero(s);
    uint32_t *kp = keys.get(), *vp = vals.get();
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
    radix_sort_pairs(kp, vp, kt.get(), vt.get(), n, bits, s);
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
        run += (hc[k] + 7) / 8;
        start += hc[k];
    }
    tb[nseg] = run;
    const int ntiles = run, ntarg = start;
    if (ntiles == 0) return true;
    if (nseg + 1 > 257) return false;
    DevBuf<int> segd(h.size(), s);
    FMM_CUDA(cudaMemcpyAsync(segd.get(), h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    // ---- the source box of every (target, slot), from list 2
    DevBuf<int> slots((size_t)ntarg * kSlots, s), err(1, s);
    FMM_CUDA(cudaMemsetAsync(slots.get(), 0xff, (size_t)ntarg * kSlots * sizeof(int), s));
    err.zero(s);
    {
        int *sl = slots.get(), *ep = err.get();
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
    if (read_scalar(err.get(), s) != 0) return false;
    SegTable sg{segd.get(), segd.get() + nseg + 1, segd.get() + 2 * nseg + 1,
                segd.get() + 3 * nseg + 1, segd.get() + 4 * nseg + 1, nseg};
    const int *boxes = (const int *)vp;
    const double *bs = T.d_boxsize.get();
    const double *binom = device_binomials(s);
    const int ks = (p + 1 + 3) / 4;
    const int mt = (p + 1 + 7) / 8;
#define FMM_M2L_CASE(MT_, KS_)                                                   \
    if (mt <= MT_ && ks <= KS_) {                                                \
        launch_dmma<MT_, KS_>(sg, boxes, slots.get(), bs, P.ndc, p, binom, mp,   \
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

}  // namespace fmm2d
