// laplace.cuh -- the Cauchy-kernel FMM passes over a device tree.
//
// Expansions are stored box-major: coefficient k of channel c of box b sits
// at [b * stride + k * ndc + c] (double2), stride = (p + 1) * ndc, the
// reference's mpole(nd, 0:nterms) per box (c_translation/src/laprouts2d.c:31).
#pragma once

#include "common.cuh"
#include "tree.cuh"

#include <stdlib.h>
#include <string.h>

#include <map>
#include <memory>

namespace fmm2d {

// Sorted-order point data and outputs of one evaluation.
struct PointSet {
    const double2 *pos = nullptr;  // (x, y), sorted
    const int2 *se = nullptr;      // per-box [start, end)
    int n = 0;                     // (the sources' n is also the source count)
    int pgh = 0;                   // 0 none, 1 pot, 2 +grad, 3 +hess
    double2 *pot = nullptr, *grad = nullptr, *hess = nullptr;  // [i*ndc + c]
};

// Planning state of the M2L passes that depends on the tree alone (work
// lists of the slot-table kernels, the window runs).  A plan keeps one per
// geometry so that repeated evaluations skip the planning and its host
// synchronisations; with `deferred`, the M2L's bounded-wait error flag is
// left in *err for the caller to read after the evaluation instead of being
// read at the end of the M2L (the form a CUDA graph can hold).
struct M2LCache {
    std::map<uint64_t, std::shared_ptr<void>> items;
    std::map<uint64_t, bool> ok;
    int *err = nullptr;  // device flag of the deferred mode
    bool deferred = false;
};

// The cached object of `key`, or a new one built by build(W &) -> bool
// (kept in the cache when there is one); `ok` receives build's result.
template <class W, class Build>
std::shared_ptr<W> m2l_cached(M2LCache *c, uint64_t key, bool &ok, Build build) {
    if (c) {
        auto it = c->items.find(key);
        if (it != c->items.end()) {
            ok = c->ok[key];
            return std::static_pointer_cast<W>(it->second);
        }
    }
    auto w = std::make_shared<W>();
    ok = build(*w);
    if (c) {
        c->items[key] = w;
        c->ok[key] = ok;
    }
    return w;
}

struct CauchyProblem {
    int ndc = 1;        // Cauchy channels
    int p = 0;          // expansion order (nterms), same on every level
    int ifcharge = 0, ifdipole = 0;
    const double2 *src = nullptr;     // sorted sources
    const double2 *charge = nullptr;  // [i*ndc + c], sorted
    const double2 *dipstr = nullptr;  // [i*ndc + c], sorted
    PointSet sset;                    // sources as targets
    PointSet tset;                    // targets
    double thresh = 0;                // near-field exclusion radius
    int ifnear = 1;
    bool mixed = false;               // FP32 series / pair arithmetic
    bool split = false;               // split-precision M2L (FP64 triangle + TF32 x 3 tail)
    bool real_charge = false;         // complex-Laplace channels (real charges,
                                      // real part of the potential used)
    const int *sleaf = nullptr;       // leaf of every sorted source (set by cauchy_fmm)
    const int *tleaf = nullptr;       // leaf of every sorted target
    const float2 *charge32 = nullptr; // FP32 strengths (mixed near field)
    const float2 *dipstr32 = nullptr;
    const float4 *src_hl = nullptr;   // hi/lo FP32 positions (mixed near field)
    const float4 *trg_hl = nullptr;
    double *timeinfo = nullptr;       // 8 phase times (s), optional
    M2LCache *m2l_cache = nullptr;    // planning kept across evaluations (plans)
    // boxes visited by the Pascal M2M (parents with sources) and L2L (boxes
    // with evaluation points): level l's at ids + lstart[l], cnt[l] of them;
    // by the mixed mode's P2M (leaves with sources) and the P2L (boxes with
    // list-4 entries and evaluation points): ids, *cnt of them (set by
    // cauchy_fmm; the order within a level is arbitrary)
    const int *m2m_ids = nullptr, *m2m_cnt = nullptr;
    const int *l2l_ids = nullptr, *l2l_cnt = nullptr;
    const int *p2m_ids = nullptr, *p2m_cnt = nullptr;
    const int *p2l_ids = nullptr, *p2l_cnt = nullptr;
};

// Runs steps 1-8 of cfmm2dmain (src/laplace/cfmm2d.f:442-1340) on the
// device.  The outputs in sset / tset are overwritten.  In the mixed mode
// the FP32 strengths and hi/lo positions are made here unless the caller
// supplies them (charge32 / dipstr32, src_hl / trg_hl).
// FP32 (x_hi, x_lo, y_hi, y_lo) split of an FP64 position.
__device__ __forceinline__ float4 split_pos(double2 p) {
    const float xh = (float)p.x, yh = (float)p.y;
    return make_float4(xh, (float)(p.x - (double)xh), yh, (float)(p.y - (double)yh));
}
void cauchy_fmm(const Tree &T, const CauchyProblem &P, cudaStream_t s);

// M2L over list 2 on the FP64 tensor cores for all channels and levels
// (m2l.cu); false when the tree does not fit its tiling (the caller then
// uses the per-box kernel).
bool m2l_tensor_fp64(const Tree &T, const CauchyProblem &P, const double2 *mp,
                     double2 *loc, cudaStream_t s);
// Split-precision M2L (m2l.cu): the terms of total order i + j below
// split_triangle_order(p) in FP64 on the DMMA kernel, the rest as TF32 x 3
// slot GEMMs on the tcgen05 tensor cores; false (nothing launched) when
// the order or the tree does not fit.
bool m2l_split_fp64(const Tree &T, const CauchyProblem &P, const double2 *mp, double2 *loc,
                    cudaStream_t s);
int split_triangle_order(int p);

// FP32 M2L of the mixed-precision mode (m2l.cu): one complex matrix per
// (child position, slot) applied to FP32 copies of the multipoles; false
// when the order or the tree does not fit (the caller then uses FP64).
// mp32_out (optional, nboxes * (p + 1) * ndc): receives the FP32 copy of
// the multipoles of levels >= 2 that the M2L reads.
bool m2l_fp32(const Tree &T, const CauchyProblem &P, const double2 *mp, double2 *loc,
              cudaStream_t s, float2 *mp32_out = nullptr);

// Orders from which the tensor-core forms of the mixed M2L recompute the
// leading kM2LExactRows local coefficients in FP32 on the CUDA cores (a
// TF32 x 3 product holds 22 of FP32's 24 bits); FMM2D_B200_M2L_EXACT_ROWS=0
// turns it off.
constexpr int kM2LExactFrom = 17;
constexpr int kM2LExactRows = 4;
// with Hessians requested the rows 0 .. 5: the Hessian at a leaf's points
// takes its leading terms from L_2 .. L_5
constexpr int kM2LExactRowsHess = 6;
inline bool m2l_exact_rows(int p) {
    const char *e = getenv("FMM2D_B200_M2L_EXACT_ROWS");
    return p >= kM2LExactFrom && !(e && !strcmp(e, "0"));
}

// Forms of the mixed-mode M2L, selectable per expansion order.
enum M2LForm { kM2LWindow = 0, kM2LTile = 1, kM2LSimt = 2 };
int m2l_form(int p);
void set_m2l_form(int p, int form);

// M2L of the mixed mode over runs of same-row boxes with shifted tensor-core
// windows (m2l_window.cu), for the target levels whose runs are dense
// enough; returns the set of target levels it evaluated (bit l = level l),
// 0 when it does not apply.  A bounded wait that runs out sets *err.
uint64_t m2l_window_fp32(const Tree &T, const CauchyProblem &P, const float2 *mp32, double2 *loc,
                         int *err, cudaStream_t s);

// Target boxes of levels >= 2 (those with points of an evaluated set)
// grouped into segments by (level, child position) and cut into tiles of
// `tile` boxes, with the source box of each of the 27 list-2 slots of every
// target (m2l.cu).  Within a segment a slot is one translation offset, so a
// tile shares each slot's translation operator.  Segment (l - 2) * 4 + c
// holds the level-l boxes that are child c of their parent.  Source boxes
// without sources are left out of the slots; false when a list-2 entry
// falls outside them.
struct SlotPlan {
    std::shared_ptr<void> hold;  // owns the device arrays below
    const int *boxes = nullptr;  // [ntarg] target boxes, segment after segment
    const int *slots = nullptr;  // [ntarg][27] source box per slot, -1 when none
    const int2 *dxy = nullptr;   // [4][27] slot offset (source - target, box units)
    std::vector<int> tile_base, start, count;  // per segment (host)
    int nseg = 0, ntarg = 0, ntiles = 0;
};
bool plan_slots(const Tree &T, int spgh, int tpgh, int tile, cudaStream_t s, SlotPlan &sp);

// Slot GEMMs of one level on the tensor cores (helm_m2l_tc.cu): for every
// plan row q of the level's four segments (child positions cp) and every
// slot k with a source box sb = slots[q][k],
//     out[boxes[q]] += oscale * Bop[cp][k] A[sb]      (in real form)
// where A[sb] = [Re X_0..W-1 | Im X_0..W-1 | 0] are the source's W complex
// coefficients per channel split into TF32 hi / lo (slot_gemm_rows), and
// Bop[cp][k] the KP x KP real form [[Re B, -Im B], [Im B, Re B]] of the
// slot's complex operator B (entry (n, k) of the hi image at
// slot_bimg_at(n, k, KP), the lo image KP * 16 floats further).  TF32 x 3
// products accumulate in tensor memory one slot at a time, and the slots
// are summed in FP64.
struct SlotGemmLevel {
    int level = 0;                // level of the target boxes (>= 2)
    int lstart = 0;               // box of row 0 of arow and out
    int nd = 1, W = 0, KP = 0;    // channels, coefficients, padded K = N
    const float *arow = nullptr;  // [box - lstart][nd][hi KP | lo KP]
    const float *bimg = nullptr;  // [cp][27][KP / 16][hi KP x 16 | lo KP x 16]
    double2 *out = nullptr;       // [box - lstart][W][nd]
    double oscale = 1.0;
    // slots accumulated in FP32 before each FP64 sum: 1, or 27 for one
    // FP32 accumulation over all slots of a tile
    int group = 1;
};
// K (= N) of W complex coefficients: 2 W rounded up to 16 (at least 32),
// 0 when above the largest supported (96).
int slot_gemm_kp(int W);
// Operand-ready rows of nrow = boxes x nd rows of x ([box][W][nd]).
void slot_gemm_rows(long long nrow, int nd, int W, int KP, const double2 *x, float *arow,
                    cudaStream_t s);
// false (nothing launched) when the level has no tiles or the shape is
// unsupported; *err is set when a bounded wait runs out.
bool slot_gemm_tc_level(const SlotGemmLevel &g, const SlotPlan &spl, int *err, cudaStream_t s);
// Index of Bop entry (output column n, input k) in the hi images of one
// (child position, slot): K chunk k / 16, then the no-swizzle K-major
// layout of the chunk's N x 16 block.
__host__ __device__ inline size_t slot_bimg_at(int n, int k, int KP) {
    const int kc = k >> 4, cc = (k >> 2) & 3, el = k & 3;
    return (size_t)kc * (2 * KP * 16) +
           (size_t)((((cc * (KP / 8) + (n >> 3)) << 5) + ((n & 7) << 2) + el));
}

// Binomial table C(l, m), l, m <= kLdc, built with the reference's Pascal
// recurrence (init_carray, src/common/fmmcommon2d.f).
constexpr int kLdc = 127;
const double *device_binomials(cudaStream_t s);

}  // namespace fmm2d
