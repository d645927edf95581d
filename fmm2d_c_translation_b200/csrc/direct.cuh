// direct.cuh -- device direct sums (every target against every source).
#pragma once

#include "common.cuh"

namespace fmm2d {

enum { kFormLaplace = 0, kFormCauchy = 1 };

// Device pointers; layouts as the reference's direct kernels with nd
// densities: charge/dipstr [i*nd + j], dipvec [(i*2 + c)*nd + j],
// pot [t*nd + j], Laplace grad [(t*2 + c)*nd + j] / hess [(t*3 + c)*nd + j],
// Cauchy grad / hess [t*nd + j].
struct DirectArgs {
    int form = kFormLaplace;
    int nd = 1;
    int ns = 0;
    const double2 *src = nullptr;
    int ifcharge = 0, ifdipole = 0;
    const double2 *chg = nullptr, *dip = nullptr;
    const double *dv = nullptr;
    int nt = 0;
    const double2 *trg = nullptr;
    int pgh = 1;
    double2 *pot = nullptr, *grad = nullptr, *hess = nullptr;
    double thresh = 0;
    int strict = 0;
};

int direct_outputs(int form, int pgh);
int direct_chunks(int ns, int nt, int nd);
int direct_strict(int form, int ifcharge, int ifdipole, int pgh);
// Throws FmmError(4) when an array that the flags require is NULL: sources,
// targ and pot always; charge when ifcharge; dipstr (and, for the Laplace
// form, dipvec) when ifdipole; grad when ifpgh >= 2; hess when ifpgh == 3.
void check_direct_arrays(int form, const void *sources, int ifcharge,
                         const void *charge, int ifdipole, const void *dipstr,
                         const void *dipvec, const void *targ, int ifpgh,
                         const void *pot, const void *grad, const void *hess);
// Adds the direct sum into a.pot/grad/hess; `part` holds
// nchunk * nd * nt * direct_outputs(form, pgh) double2 of scratch.
void direct_sum(const DirectArgs &a, double2 *part, int nchunk, cudaStream_t s);

}  // namespace fmm2d
