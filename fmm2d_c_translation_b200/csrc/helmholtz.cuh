// helmholtz.cuh -- the Helmholtz FMM passes over a device tree.
//
// Expansions follow the reference's scaled Graf form (c_translation/src/
// helmrouts2d.c): a box at level l of order p_l and scale r_l holds
// coefficients n = -p_l..p_l per channel, stored box-major as
// [box][n + p_l][channel] (double2), the reference's mpole(nd, -nterms:nterms).
// Boxes of one level are contiguous, so a box's block is found from a
// per-level offset.
#pragma once

#include <vector>

#include "common.cuh"
#include "tree.cuh"

namespace fmm2d {

// Sorted-order point data and outputs of one Helmholtz evaluation.
// Outputs: pot [k*nd + c], grad [(k*2 + d)*nd + c], hess [(k*3 + d)*nd + c].
struct HPointSet {
    const double2 *pos = nullptr;
    const int2 *se = nullptr;
    int n = 0;
    int pgh = 0;
    double2 *pot = nullptr, *grad = nullptr, *hess = nullptr;
};

struct HelmProblem {
    int nd = 1;
    double2 zk = {0.0, 0.0};
    double eps = 1e-6;
    int ifcharge = 0, ifdipole = 0;
    const double2 *src = nullptr;     // sorted sources
    const double2 *charge = nullptr;  // [k*nd + c]
    const double2 *dipstr = nullptr;  // [k*nd + c]
    const double2 *dipvec = nullptr;  // [k*nd + c] = (v1, v2)
    HPointSet sset, tset;
    int ifnear = 1;
    // M2L of the levels of order <= 23 on the tensor cores in TF32 x 3
    // (helm_m2l_tc.cu); everything else stays FP64
    bool mixed = false;
};

// Runs the steps of hfmm2dmain (c_translation/src/hfmm2d.c:619-1528) on the
// device; the outputs in sset / tset are overwritten.
void helmholtz_fmm(const Tree &T, const HelmProblem &P, cudaStream_t s);

// Direct sums over all sources for every point of `set` (the reference's
// h2d_direct* kernels, c_translation/src/helmkernels2d.c), adding to the
// outputs; pairs with |zk r| below thresh are skipped.
void helmholtz_direct(const HelmProblem &P, int ns, HPointSet set, double thresh,
                      cudaStream_t s);

// One level of the tensor-core M2L of the mixed mode (helm_m2l_tc.cu).
struct HtLevel {
    int level = 0, p = 0, nd = 1, lstart = 0;
    long long nbox = 0;         // boxes of the level
    long long off = 0;          // offset of the level's block in the expansions
    double maxabs = 0.0;        // largest |T(q)| of the level's M2L tables
    const double2 *table = nullptr;  // device: [49][4p + 1] M2L table
    const double *pw = nullptr;      // device: rs^e, e = 0 .. 2p
};
struct SlotPlan;
// Highest expansion order the tensor-core M2L takes.
int helm_m2l_tc_max_order();
// Adds the list-2 interactions of level lv.level to the local expansions
// with the tensor-core M2L; false (nothing launched) when the level does not
// qualify.  spl: slot plan with tiles of 128 / nd target boxes; *err is set
// when a bounded wait of the kernel runs out.
bool helm_m2l_tc_level(const HtLevel &lv, const SlotPlan &spl, const double2 *mp, double2 *loc,
                       int *err, cudaStream_t s);

// High-frequency levels (helm_hf.cu): boxes of more than 16 wavelengths
// (boxlam = |zk| boxsize / 2 pi > 16, the reference's switch) with scale 1,
// where the M2L runs in the diagonal (signature) form.
bool helm_hf_level(double boxlam, double rs);
// The M2L of level l in the diagonal form: d_table is the level's M2L
// table [49][4p + 1] (device), off the level's offset in mp / loc.
void helm_m2l_hf(const Tree &T, int l, int p, int nd, long long off, const double2 *d_table,
                 const double2 *mp, double2 *loc, int sp, int tp, cudaStream_t s);

// Host restatements of the reference's scalar routines.
// h2dterms (c_translation/src/h2dterms.c:19-69): expansion order for a box
// of size bsize; -1 when no order up to 50000 reaches eps.
int helm_nterms(double bsize, double2 zk, double eps);
// h2dall (h2dcommon.c:35-90): hvec[0..n] = H_k(z) rscale^k.
void helm_hvec(int n, double2 z, double rscale, double2 *hvec);
// jbessel2d (cdjseval2d.c:11-160): fjs[0..n] = J_k(z) / rscale^k.
void helm_jvec(int n, double2 z, double rscale, double2 *fjs);

}  // namespace fmm2d
