// engine.cuh -- one FMM evaluation from user arrays to user arrays.
#pragma once

#include "common.cuh"
#include "tree.cuh"

namespace fmm2d {

// kReal: the real-valued Laplace FMM (rfmm2d, src/laplace/rfmm2d.f:27-214):
// real charges, real dipole strengths with dipole vectors, real outputs.
enum Kernel { kLaplace = 0, kCauchy = 1, kHelmholtz = 2, kReal = 3 };
enum Precision { kPrecAuto = 0, kPrecFP64 = 1, kPrecMixed = 2, kPrecSplit = 3 };

// Arguments of the reference's guru drivers (lfmm2d / cfmm2d / hfmm2d and
// their _ndiv forms).  Complex arrays are interleaved (re, im) doubles in
// the reference's column-major layouts.  Pointers may be host memory
// (pageable or pinned) or device memory of the current device; all
// pointers of one call must be of the same kind.
struct FmmCall {
    Kernel kernel = kLaplace;
    int nd = 1;
    double eps = 1e-6;
    double zk[2] = {0, 0};
    int ns = 0;
    const double *sources = nullptr;
    int ifcharge = 0;
    const double *charge = nullptr;
    int ifdipole = 0;
    const double *dipstr = nullptr;
    const double *dipvec = nullptr;  // Laplace / Helmholtz only
    int ifpgh = 0;
    double *pot = nullptr, *grad = nullptr, *hess = nullptr;
    int nt = 0;
    const double *targ = nullptr;
    int ifpghtarg = 0;
    double *pottarg = nullptr, *gradtarg = nullptr, *hesstarg = nullptr;
    int ndiv = -1;       // < 0: from eps (lndiv2d / hndiv2d)
    int idivflag = 0;
    int ifnear = 1;
    double *timeinfo = nullptr;  // 8 entries, optional
    int precision = kPrecAuto;
};

// Geometry of a Laplace / Cauchy evaluation (tree, lists, points in tree
// order); laplace_geometry builds it from the positions of `c` (host or
// device arrays, on_dev saying which), laplace_evaluate runs one evaluation
// over it with the strengths and outputs of `c`.
struct LapGeometry {
    bool lap = true, mixed = false;
    bool split = false;  // split-precision M2L, every other pass FP64
    bool real = false;  // rfmm2d: one real-charge channel per density
    int nd = 1, ndc = 2, ns = 0, nt = 0, p = 0;
    double eps = 0, thresh = 0;
    Tree T;
    DevBuf<double2> src_s, trg_s;
    DevBuf<float4> src_hl, trg_hl;  // mixed mode: FP32 hi/lo positions
};
void laplace_geometry(const FmmCall &c, bool on_dev, cudaStream_t s, LapGeometry &G);
// m2l: planning kept across evaluations (plans), null for a one-shot call;
// sync = false leaves the final stream synchronisation to the caller (the
// form a CUDA graph can capture).
//
// Host-array calls overlap their copies with the compute through `io`:
// strengths_dev says the strength pointers of `c` already hold device
// copies (staged on a copy stream while the tree was built; the caller made
// `s` wait for them), and with a copy stream each output array's
// device-to-host copy runs there as soon as its scatter kernel has
// finished, overlapping the remaining scatters.
struct M2LCache;
struct EvalIO {
    bool strengths_dev = false;
    cudaStream_t copy = nullptr;
};
void laplace_evaluate(const FmmCall &c, const LapGeometry &G, bool on_dev, cudaStream_t s,
                      M2LCache *m2l = nullptr, bool sync = true, const EvalIO &io = EvalIO());

// A batch of independent lfmm2d / cfmm2d problems (nd = 1) with the same
// eps and flags, evaluated as one forest: one launch per level and pass for
// the whole batch.  Arrays per problem, host or device (all of one kind
// per array list); a null charge / dipstr list means no charges / dipoles.
struct BatchCall {
    Kernel kernel = kLaplace;
    double eps = 1e-6;
    int nprob = 0;
    const int *ns = nullptr, *nt = nullptr;
    const double *const *sources = nullptr, *const *targ = nullptr;
    const double *const *charge = nullptr, *const *dipstr = nullptr, *const *dipvec = nullptr;
    int ifpgh = 0, ifpghtarg = 0;
    double *const *pot = nullptr, *const *grad = nullptr, *const *hess = nullptr;
    double *const *pottarg = nullptr, *const *gradtarg = nullptr, *const *hesstarg = nullptr;
    int precision = kPrecAuto;
};
int run_laplace_batch(const BatchCall &b);

// Runs the evaluation on the calling thread's current device; returns the
// reference's ier (0 ok, 4 failure) after recording any error message.
int run_fmm(const FmmCall &c);

// Helmholtz direct sum (h2d_direct*), incrementing the outputs; host or
// device arrays of one kind.  Returns 0 or 4.
int run_helm_direct(int nd, const double *zk, int ns, const double *sources, int ifcharge,
                    const double *charge, int ifdipole, const double *dipstr,
                    const double *dipvec, int nt, const double *targ, int ifpgh, double *pot,
                    double *grad, double *hess, double thresh);

// Expansion order of the Laplace FMM (l2dterms, c_translation/src/l2dterms.c).
int laplace_nterms(double eps);
// Leaf capacity (lndiv2d.f / hndiv2d.c).
int leaf_capacity(double eps, int ns, int nt);

// Leaf capacity of the mixed-precision complex-Laplace mode for order p
// (falls back to `fallback`), and its setter (ndiv <= 0 clears).
int mixed_leaf_capacity(int p, int fallback);
void set_mixed_leaf_capacity(int p, int ndiv);

// Process-wide precision policy (env FMM2D_B200_PRECISION=auto|fp64|mixed,
// or fmm2d_b200_set_precision).
int current_precision();
void set_precision(int p);

}  // namespace fmm2d
