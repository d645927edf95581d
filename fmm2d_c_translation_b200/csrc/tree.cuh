// tree.cuh -- the adaptive, level-restricted quadtree and its interaction
// lists, built on the device.
//
// The box arrays, the box numbering and the point permutations are
// bit-identical to the reference's pts_tree_build / pts_tree_sort /
// computelists (c_translation/src/pts_tree2d.c, tree_routs2d.c) on the same
// inputs.  Ids are 0-based on the device (-1 = none); export_reference_tree
// converts to the reference's 1-based packed `itree` layout.
#pragma once

#include "common.cuh"

namespace fmm2d {

// List capacities of the reference (c_translation/src/tree_routs2d.c:325-345).
constexpr int kMaxList1 = 13;
constexpr int kMaxList2 = 27;
constexpr int kMaxList3 = 20;
constexpr int kMaxList4 = 5;
constexpr int kMaxLevels = 51;  // nlmax of the reference drivers

struct Tree {
    int nlevels = 0;
    int nboxes = 0;
    int cap = 0;
    std::vector<double> boxsize;       // [0..nlevels]
    std::vector<int> lstart, lend;     // box id range [lstart, lend) per level
    DevBuf<double2> centers;
    DevBuf<int> level, parent, nchild, child;  // child: 4 per box
    DevBuf<int> nnbors, nbors;                 // nbors: 9 per box
    // point ranges per box, [start, end) into the sorted order
    DevBuf<int2> srcse, trgse;
    // sorted position -> input index
    DevBuf<int> isrc, itarg;
    // interaction lists
    DevBuf<int> nlist1, list1, nlist2, list2, nlist3, list3, nlist4, list4;
    DevBuf<double> d_boxsize;  // boxsize per level on the device
    int nroots = 1;            // > 1: a forest of independent problems
};

// Builds the tree over ns sources and nt targets (device arrays of (x, y)
// pairs).  idivflag: 0 refine on source count, 1 on target count, 2 on the
// larger.  Follows pts_tree_mem / pts_tree_build / pts_tree_sort.
void build_tree(const double2 *d_src, int ns, const double2 *d_targ, int nt,
                int ndiv, int idivflag, int nlmax, cudaStream_t s, Tree &T);

// A forest of independent trees for a batch of problems: the concatenated
// points of problem k are [soff[k], soff[k+1]) and [toff[k], toff[k+1]),
// already translated so that every problem's bounding square is centred at
// the origin; bs0 is the common root size.  The roots are boxes 0 .. k-1,
// each level holds the boxes of all problems, and no list crosses problems
// (each root is its own only colleague).
void build_forest(const double2 *d_src, const std::vector<int> &soff, const double2 *d_targ,
                  const std::vector<int> &toff, int ndiv, int idivflag, int nlmax, double bs0,
                  cudaStream_t s, Tree &T);

// computelists (c_translation/src/tree_routs2d.c:369-510).
void compute_lists(Tree &T, cudaStream_t s);

// Copies the tree to host arrays in the reference's layout: itree
// (ltree = 17*nboxes + 2*(nlevels+1) entries, 1-based), iptr(8),
// centers(2, nboxes), boxsize(0:nlevels), isrc(ns), isrcse(2, nboxes),
// itarg(nt), itargse(2, nboxes).  Any output pointer may be null.
void export_reference_tree(const Tree &T, int ns, int nt, int *itree,
                           int *iptr, double *centers, double *boxsize,
                           int *isrc, int *isrcse, int *itarg, int *itargse,
                           cudaStream_t s);

}  // namespace fmm2d
