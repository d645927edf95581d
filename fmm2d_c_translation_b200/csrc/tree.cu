// tree.cu -- device construction of the reference's adaptive quadtree.
//
// The reference builds its tree serially (c_translation/src/pts_tree2d.c,
// tree_routs2d.c).  Every step it takes is either "for each box of one
// level, decide something from data of coarser levels" or "append the
// children of the flagged boxes of a range, in box order".  The first maps
// to one kernel per level; the second to a prefix sum over the flags (the
// same role cumsum plays in tree_refine_boxes) followed by one kernel that
// writes the children at their scanned positions.  With the same FP64
// operations in the same order (box centers by repeated center +/- bs/2,
// child choice by `p - c < 0`, the 1.05-scaled distance tests), the box
// numbering, centers and point permutation come out identical.
#include "sort.cuh"
#include "tree.cuh"

#include <algorithm>
#include <cstring>

namespace fmm2d {
namespace {

// Child j (0-based) of a box: the reference numbers children 1..4 as
// (-x,-y), (+x,-y), (-x,+y), (+x,+y) (tree_routs2d.c:77-86).
__device__ __forceinline__ double2 child_center(double2 c, double bs, int j) {
    const double hx = ((j & 1) ? bs : -bs) * 0.5;
    const double hy = ((j & 2) ? bs : -bs) * 0.5;
    return make_double2(__dadd_rn(c.x, hx), __dadd_rn(c.y, hy));
}

// Which child of a box with center c holds point p (pts_tree2d.c:697-748):
// first split on y, then on x, comparing `p - c < 0`.
__device__ __forceinline__ int child_digit(double2 p, double2 c) {
    const int right = (__dsub_rn(p.x, c.x) < 0.0) ? 0 : 1;
    const int upper = (__dsub_rn(p.y, c.y) < 0.0) ? 0 : 2;
    return right + upper;
}

__device__ __forceinline__ bool within(double2 a, double2 b, double d) {
    return fabs(__dsub_rn(a.x, b.x)) <= d && fabs(__dsub_rn(a.y, b.y)) <= d;
}

// Path keys.  The box that holds a point at level m is fixed by the child
// digits (0..3, the reference's child number minus 1) the point takes at
// levels 1..m, each decided by `p - c < 0` against the FP64 center of its
// box one level up.  A center depends only on the path (repeated
// c +/- bs/2), so the digits of every level can be computed for every point
// up front, without the tree.  Word w of a key holds the digits of levels
// 16w+1 .. 16w+16, two bits each, the coarsest level in the top bits;
// sorting by the words, first word most significant, orders the points by
// path, which is the order of the reference's nested stable partitions.
constexpr int kKeyWords = 4;  // up to 64 levels (nlmax of the reference is 51)

struct KeyView {
    const uint32_t *w[kKeyWords];  // sorted key words, one array per word
};

__device__ __forceinline__ int key_digit(const KeyView &kv, int64_t k, int m) {
    const int w = (m - 1) >> 4, sh = 2 * (15 - ((m - 1) & 15));
    return (int)((kv.w[w][k] >> sh) & 3u);
}

// Common leading digits (levels) of the sorted keys at positions a and b.
__device__ __forceinline__ int key_lcp(const KeyView &kv, int nw, int64_t a, int64_t b) {
    for (int w = 0; w < nw; w++) {
        const uint32_t x = kv.w[w][a] ^ kv.w[w][b];
        if (x) return 16 * w + (__clz(x) >> 1);
    }
    return 16 * nw;
}

// Number of boxes of every level 1..ds that hold more than ndiv of the
// n key-sorted points: a box of level l is a run of equal l-digit prefixes,
// and the run starting at k (a start when the prefix differs from k-1's,
// i.e. l > lcp(k-1, k)) holds more than ndiv points when the point ndiv
// further on still shares the prefix (l <= lcp(k, k + ndiv)).  Each point
// adds one to the levels in (lcp(k-1, k), lcp(k, k + ndiv)].
__global__ void __launch_bounds__(256) refine_count_kernel(KeyView kv, int64_t n, int ndiv,
                                                           int ds, int nw,
                                                           unsigned long long *__restrict__ cnt) {
    __shared__ unsigned int sc[65];
    for (int l = threadIdx.x; l <= 64; l += blockDim.x) sc[l] = 0;
    __syncthreads();
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        if (k + ndiv >= n) continue;
        const int a = k == 0 ? 0 : key_lcp(kv, nw, k - 1, k);
        const int b = min(key_lcp(kv, nw, k, k + ndiv), ds);
        for (int l = a + 1; l <= b; l++) atomicAdd(&sc[l], 1u);
    }
    __syncthreads();
    for (int l = threadIdx.x; l <= 64; l += blockDim.x)
        if (sc[l]) atomicAdd(&cnt[l], (unsigned long long)sc[l]);
}

// Path keys of n points: nw words per point, word-major (word w of point i
// at words[w * n + i]); digits of levels beyond `ds` are 0.  bsl[m] is the
// box size of level m, obtained by repeated halving as the reference does.
__global__ void __launch_bounds__(256) path_key_kernel(
    const double2 *__restrict__ pts, int n, double2 c0, const double *__restrict__ bsl,
    int ds, int nw, uint32_t *__restrict__ words) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double2 p = pts[i];
        double2 c = c0;
        for (int w = 0; w < nw; w++) {
            uint32_t key = 0;
#pragma unroll 4
            for (int t = 0; t < 16; t++) {
                const int m = 16 * w + t + 1;
                int d = 0;
                if (m <= ds) {
                    d = child_digit(p, c);
                    c = child_center(c, bsl[m], d);
                }
                key = (key << 2) | (uint32_t)d;
            }
            words[(size_t)w * n + i] = key;
        }
    }
}

// Input order inside every leaf of at most kLeafSort points: one warp per
// leaf sorts the leaf's input indices with a bitonic network, over the
// lanes' registers for up to 32 points, in shared memory for more.
constexpr int kLeafSort = 256;

__global__ void __launch_bounds__(256) leaf_order_kernel(
    int nb, const int *__restrict__ nch, const int2 *__restrict__ rng,
    const uint32_t *__restrict__ idx, int *__restrict__ perm) {
    __shared__ uint32_t sh_all[8][kLeafSort];
    const int lane = threadIdx.x & 31;
    uint32_t *sh = sh_all[threadIdx.x >> 5];
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); b < nb; b += warps) {
        if (nch[b] != 0) continue;
        const int2 r = rng[b];
        const int cnt = r.y - r.x;
        if (cnt <= 0) continue;
        if (cnt <= 32) {
            uint32_t v = lane < cnt ? idx[r.x + lane] : 0xffffffffu;
            if (cnt > 1) {
#pragma unroll
                for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
                    for (int j = k >> 1; j > 0; j >>= 1) {
                        const uint32_t o = __shfl_xor_sync(0xffffffffu, v, j);
                        const bool up = (lane & k) == 0, low = (lane & j) == 0;
                        v = (low == up) ? min(v, o) : max(v, o);
                    }
            }
            if (lane < cnt) perm[r.x + lane] = (int)v;
            continue;
        }
        // 33 .. kLeafSort points (the caller guarantees the bound)
        int n2 = 64;
        while (n2 < cnt) n2 <<= 1;
        for (int i = lane; i < n2; i += 32) sh[i] = i < cnt ? idx[r.x + i] : 0xffffffffu;
        __syncwarp();
        for (int k = 2; k <= n2; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < n2; i += 32) {
                    const int ij = i ^ j;
                    if (ij > i) {
                        const uint32_t a = sh[i], c = sh[ij];
                        const bool up = (i & k) == 0;
                        if ((a > c) == up) {
                            sh[i] = c;
                            sh[ij] = a;
                        }
                    }
                }
                __syncwarp();
            }
        for (int i = lane; i < cnt; i += 32) perm[r.x + i] = (int)sh[i];
        __syncwarp();
    }
}

struct Builder {
    Tree &T;
    cudaStream_t s;
    DevBuf<int> iflag;
    DevBuf<int> cnt_s, cnt_t;  // point counts per box (levelwise build only)
    // key build: every box's [start, end) range in the key-sorted sources
    // and targets, and the sorted key words
    bool ranges = false;
    DevBuf<int2> rs, rt;
    KeyView kvs{}, kvt{};

    Builder(Tree &t, cudaStream_t st) : T(t), s(st) {}

    // Grow every per-box array to hold at least `need` boxes.
    void ensure(int need) {
        if (need <= T.cap) return;
        int nc = std::max(need, T.cap + T.cap / 2 + 64);
        size_t keep = (size_t)T.nboxes;
        T.centers.grow(nc, keep, s);
        T.level.grow(nc, keep, s);
        T.parent.grow(nc, keep, s);
        T.nchild.grow(nc, keep, s);
        T.child.grow((size_t)4 * nc, 4 * keep, s);
        T.nnbors.grow(nc, keep, s);
        T.nbors.grow((size_t)9 * nc, 9 * keep, s);
        iflag.grow(nc, keep, s);
        if (cnt_s.size()) cnt_s.grow(nc, keep, s);
        if (cnt_t.size()) cnt_t.grow(nc, keep, s);
        if (ranges) {
            rs.grow(nc, keep, s);
            rt.grow(nc, keep, s);
        }
        T.cap = nc;
    }

    // Point ranges of the boxes [nb0, nb1), all just created as children (4
    // per parent, in child order): within the parent's range the key-sorted
    // points are ordered by their digit at the children's level, so child j
    // starts at the first point whose digit is >= j (binary search).
    void set_child_ranges(int nb0, int nb1) {
        if (!ranges || nb1 <= nb0) return;
        const int *par = T.parent.get(), *lev = T.level.get();
        int2 *rs0 = rs.get(), *rt0 = rt.get();
        const KeyView ks0 = kvs, kt0 = kvt;
        const int64_t nn = nb1 - nb0;
        // both point sets in one launch: items [0, nn) sources, [nn, 2 nn) targets
        {
            for_each(2 * nn, s, [=] __device__(int64_t ii) {
                const bool tset = ii >= nn;
                const int64_t i = tset ? ii - nn : ii;
                int2 *r = tset ? rt0 : rs0;
                const KeyView kv = tset ? kt0 : ks0;
                const int kb = nb0 + (int)i, j = (int)(i & 3);
                const int m = lev[kb];
                const int2 pr = r[par[kb]];
                auto first_ge = [&](int dj) {
                    int lo = pr.x, hi = pr.y;
                    while (lo < hi) {
                        const int mid = lo + ((hi - lo) >> 1);
                        if (key_digit(kv, mid, m) < dj)
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    return lo;
                };
                const int a = (j == 0 || pr.x == pr.y) ? pr.x : first_ge(j);
                const int b = (j == 3 || pr.x == pr.y) ? pr.y : first_ge(j + 1);
                r[kb] = make_int2(a, b);
            });
        }
    }

    // Appends 4 children to every box b in [lo, hi) with sel(b) true, in box
    // order.  Returns the number of refined boxes.  Mirrors
    // tree_refine_boxes and, with set_flags, tree_refine_boxes_flag, whose
    // children get flag 3 under a flag-1 parent and 0 otherwise.  `sel` is
    // evaluated before any array grows.
    // known >= 0: the caller knows the number of refined boxes (no host
    // synchronisation); the device's own count goes to *check, and no child
    // is written beyond the capacity in case the two differ.
    template <class Sel>
    int refine_range(int lo, int hi, int newlevel, double bs, Sel sel,
                     bool set_flags, int known = -1, int *check = nullptr) {
        const int n = hi - lo;
        if (n <= 0) return 0;
        DevBuf<int> f(n, s), off(n, s), tot(1, s);
        int *fp = f.get();
        for_each(n, s, [=] __device__(int64_t i) { fp[i] = sel(lo + (int)i) ? 1 : 0; });
        exclusive_scan_i32(fp, off.get(), n, check ? check : tot.get(), s);
        const int nref = known >= 0 ? known : read_scalar(tot.get(), s);
        if (nref == 0) return 0;
        ensure(T.nboxes + 4 * nref);
        const int cap = T.cap;
        if (known >= 0) {
            // a known count that was too large must leave no box unset: the
            // ones no parent fills hang under the root (the check at the end
            // of the build then rebuilds the tree)
            const int nb0k = T.nboxes;
            int *lev = T.level.get(), *par = T.parent.get(), *nch = T.nchild.get(),
                *chi = T.child.get();
            double2 *cenk = T.centers.get();
            for_each(4 * (int64_t)nref, s, [=] __device__(int64_t i) {
                const int kb = nb0k + (int)i;
                cenk[kb] = cenk[0];
                par[kb] = 0;
                lev[kb] = newlevel;
                nch[kb] = 0;
                for (int l = 0; l < 4; l++) chi[4 * kb + l] = -1;
            });
        }
        const int nb0 = T.nboxes;
        double2 *cen = T.centers.get();
        int *lev = T.level.get(), *par = T.parent.get(), *nch = T.nchild.get();
        int *chi = T.child.get(), *flg = iflag.get();
        int *cs = cnt_s.get(), *ct = cnt_t.get();
        const int *op = off.get();
        for_each(n, s, [=] __device__(int64_t i) {
            if (!fp[i]) return;
            const int b = lo + (int)i;
            const int base = nb0 + 4 * op[i];
            if (base + 4 > cap) return;  // (a known count that was wrong: caught by *check)
            const double2 c = cen[b];
            const int cf = (set_flags && flg[b] == 1) ? 3 : 0;
            nch[b] = 4;
            for (int j = 0; j < 4; j++) {
                const int kb = base + j;
                cen[kb] = child_center(c, bs, j);
                par[kb] = b;
                nch[kb] = 0;
                lev[kb] = newlevel;
                for (int l = 0; l < 4; l++) chi[4 * kb + l] = -1;
                chi[4 * b + j] = kb;
                if (set_flags) flg[kb] = cf;
                if (cs) cs[kb] = 0;
                if (ct) ct[kb] = 0;
            }
        });
        T.nboxes += 4 * nref;
        set_child_ranges(nb0, T.nboxes);
        return nref;
    }

    // Splits the selected boxes among the items [0, n1 + n2) -- item i is
    // box lo + i for i < n1, else tlo + (i - n1) -- given their selection
    // flags fp, its exclusive scan op and the number selected, nref (exact:
    // counted from the same flags).  Four children per selected box are
    // appended in item order, which is the order of the reference's
    // per-level calls (a level range before its tail).  A child's level and
    // size follow from its parent's level (d_bsl: box size per level), so
    // the items may span several levels in box order.  Children get flag 3
    // under a flag-1 parent and 0 otherwise (tree_refine_boxes_flag); with
    // set_flags false the flags are left alone (tree_refine_boxes).
    void split_items(int lo, int n1, int tlo, int n2, const int *fp, const int *op, int nref,
                     const double *d_bsl, bool set_flags = true) {
        if (nref <= 0) return;
        ensure(T.nboxes + 4 * nref);
        const int nb0 = T.nboxes, cap = T.cap;
        double2 *cen = T.centers.get();
        int *lev = T.level.get(), *par = T.parent.get(), *nch = T.nchild.get();
        int *chi = T.child.get(), *flg = iflag.get();
        int *cs = cnt_s.get(), *ct = cnt_t.get();
        for_each((int64_t)n1 + n2, s, [=] __device__(int64_t i) {
            if (!fp[i]) return;
            const int b = i < n1 ? lo + (int)i : tlo + (int)(i - n1);
            const int base = nb0 + 4 * op[i];
            if (base + 4 > cap) return;
            const double2 c = cen[b];
            const int nl = lev[b] + 1;
            const double bs = d_bsl[nl];
            const int cf = set_flags && flg[b] == 1 ? 3 : 0;
            nch[b] = 4;
            for (int j = 0; j < 4; j++) {
                const int kb = base + j;
                cen[kb] = child_center(c, bs, j);
                par[kb] = b;
                nch[kb] = 0;
                lev[kb] = nl;
                for (int l = 0; l < 4; l++) chi[4 * kb + l] = -1;
                chi[4 * b + j] = kb;
                if (set_flags) flg[kb] = cf;
                if (cs) cs[kb] = 0;
                if (ct) ct[kb] = 0;
            }
        });
        T.nboxes += 4 * nref;
        set_child_ranges(nb0, T.nboxes);
    }

    std::vector<double> host_dist(int kind) const {
        // 1.05-scaled distance thresholds per level, evaluated exactly as the
        // reference writes them.
        std::vector<double> d(T.nlevels + 2, 0.0);
        const std::vector<double> &bs = T.boxsize;
        for (int l = 0; l <= T.nlevels; l++) {
            switch (kind) {
                case 0: d[l] = 1.05 * bs[l]; break;  // colleagues
                case 1:  // flag pass (pts_tree2d.c:800)
                    if (l >= 2) d[l] = 1.05 * (bs[l - 1] + bs[l - 2]) / 2.0;
                    break;
                case 2:  // flag+ pass (pts_tree2d.c:829)
                    if (l >= 1) d[l] = 1.05 * (bs[l] + bs[l - 1]) / 2.0;
                    break;
                case 3:  // updateflags / list 1 (tree_routs2d.c:215, 466)
                    if (l + 1 <= T.nlevels)
                        d[l] = 1.05 * (bs[l] + bs[l + 1]) / 2.0;
                    else
                        d[l] = 1.05 * (bs[l] + bs[l] / 2) / 2.0;
                    break;
            }
        }
        return d;
    }

    // computecoll (tree_routs2d.c:140-195) for levels [l0, l1].
    void computecoll(int l0, int l1) {
        int *nnb = T.nnbors.get(), *nb = T.nbors.get();
        const int *par = T.parent.get(), *chi = T.child.get();
        const double2 *cen = T.centers.get();
        if (l0 == 0) {
            // roots (one per problem of a forest): their own only colleague
            for_each(T.lend[0] - T.lstart[0], s, [=] __device__(int64_t i) {
                const int b = (int)i;
                nnb[b] = 1;
                nb[9 * b] = b;
                for (int k = 1; k < 9; k++) nb[9 * b + k] = -1;
            });
            l0 = 1;
        }
        for (int l = l0; l <= l1; l++) {
            const int lo = T.lstart[l], n = T.lend[l] - T.lstart[l];
            const double d = 1.05 * T.boxsize[l];
            for_each(n, s, [=] __device__(int64_t i) {
                const int b = lo + (int)i;
                const int dad = par[b];
                const double2 cb = cen[b];
                int cnt = 0;
                for (int k = 0; k < nnb[dad]; k++) {
                    const int jb = nb[9 * dad + k];
                    for (int j = 0; j < 4; j++) {
                        const int kb = chi[4 * jb + j];
                        if (kb >= 0 && within(cen[kb], cb, d) && cnt < 9)
                            nb[9 * b + cnt++] = kb;
                    }
                }
                nnb[b] = cnt;
                for (int k = cnt; k < 9; k++) nb[9 * b + k] = -1;
            });
        }
    }

    // pts_tree_reorg (pts_tree2d.c:966-1085): on every level >= 2 the boxes
    // of the level range come first, then the appended ("tail") boxes of
    // that level, each group in its current order.
    void reorg(const std::vector<int> &tstart, const std::vector<int> &tend) {
        const int L = T.nlevels;
        const int nb = T.nboxes;
        std::vector<int> h(4 * (L + 1), 0);  // lstart, lend, tstart, nstart
        int cur = T.lstart[std::min(2, L)];
        std::vector<int> nstart(L + 1), nend(L + 1);
        for (int l = 0; l <= L; l++) {
            if (l < 2) {
                nstart[l] = T.lstart[l];
                nend[l] = T.lend[l];
                continue;
            }
            nstart[l] = cur;
            cur += (T.lend[l] - T.lstart[l]) + (tend[l] - tstart[l]);
            nend[l] = cur;
        }
        for (int l = 0; l <= L; l++) {
            h[4 * l + 0] = T.lstart[l];
            h[4 * l + 1] = T.lend[l];
            h[4 * l + 2] = tstart[l];
            h[4 * l + 3] = nstart[l];
        }
        DevBuf<int> lv(h.size(), s);
        FMM_CUDA(cudaMemcpyAsync(lv.get(), h.data(), h.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
        DevBuf<int> map(nb, s);
        int *mp = map.get();
        const int *lvp = lv.get(), *levp = T.level.get();
        for_each(nb, s, [=] __device__(int64_t i) {
            const int b = (int)i, l = levp[b];
            int m;
            if (l < 2) {
                m = b;
            } else {
                const int ls = lvp[4 * l], le = lvp[4 * l + 1];
                const int ts = lvp[4 * l + 2], ns0 = lvp[4 * l + 3];
                m = (b >= ls && b < le) ? ns0 + (b - ls) : ns0 + (le - ls) + (b - ts);
            }
            mp[b] = m;
        });
        DevBuf<double2> cen2(T.cap, s);
        DevBuf<int> lev2(T.cap, s), par2(T.cap, s), nch2(T.cap, s),
            chi2((size_t)4 * T.cap, s), flg2(T.cap, s);
        DevBuf<int2> rs2, rt2;
        if (ranges) {
            rs2.alloc(T.cap, s);
            rt2.alloc(T.cap, s);
        }
        const double2 *cen = T.centers.get();
        const int *par = T.parent.get(), *nch = T.nchild.get(),
                  *chi = T.child.get(), *flg = iflag.get();
        const int2 *ra = rs.get(), *rb = rt.get();
        double2 *c2 = cen2.get();
        int *l2 = lev2.get(), *p2 = par2.get(), *n2 = nch2.get(),
            *h2 = chi2.get(), *f2 = flg2.get();
        int2 *ra2 = rs2.get(), *rb2 = rt2.get();
        for_each(nb, s, [=] __device__(int64_t i) {
            const int b = (int)i, m = mp[b];
            if (ra2) {
                ra2[m] = ra[b];
                rb2[m] = rb[b];
            }
            c2[m] = cen[b];
            l2[m] = levp[b];
            n2[m] = nch[b];
            f2[m] = flg[b];
            p2[m] = par[b] < 0 ? -1 : mp[par[b]];
            for (int j = 0; j < 4; j++) {
                const int c = chi[4 * b + j];
                h2[4 * m + j] = c < 0 ? -1 : mp[c];
            }
        });
        T.centers = std::move(cen2);
        T.level = std::move(lev2);
        T.parent = std::move(par2);
        T.nchild = std::move(nch2);
        T.child = std::move(chi2);
        iflag = std::move(flg2);
        if (ranges) {
            rs = std::move(rs2);
            rt = std::move(rt2);
        }
        for (int l = 2; l <= L; l++) {
            T.lstart[l] = nstart[l];
            T.lend[l] = nend[l];
        }
    }

    // Number of boxes whose flag lies in [f0, f1].
    int count_flags(int f0, int f1) {
        DevBuf<int> c(1, s);
        c.zero(s);
        int *cp = c.get();
        const int *fl = iflag.get();
        for_each(T.nboxes, s, [=] __device__(int64_t i) {
            const int f = fl[i];
            const bool hit = f >= f0 && f <= f1;
            const unsigned m = __ballot_sync(__activemask(), hit);
            if (hit && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(cp, __popc(m));
        });
        return read_scalar(cp, s);
    }

    // pts_tree_fix_lr (pts_tree2d.c:767-964).
    void fix_lr() {
        const int L = T.nlevels;
        int *flg = iflag.get();
        const int *nch = T.nchild.get(), *par = T.parent.get(),
                  *lev = T.level.get();
        const double2 *cen = T.centers.get();
        iflag.zero(s);
        const std::vector<double> d1 = host_dist(1), d2 = host_dist(2),
                                  d3 = host_dist(3);
        DevBuf<double> dd1(L + 2, s);
        FMM_CUDA(cudaMemcpyAsync(dd1.get(), d1.data(), d1.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
        const double *dp1 = dd1.get();
        {
            // flag: leaves among the granddad's colleagues that touch the dad.
            const int *nnb = T.nnbors.get(), *nb = T.nbors.get();
            const int lo = T.lstart[2], n = T.lend[L] - T.lstart[2];
            for_each(n, s, [=] __device__(int64_t i) {
                const int b = lo + (int)i;
                const int idad = par[b], igd = par[idad];
                const double dist = dp1[lev[b]];
                const double2 cd = cen[idad];
                for (int k = 0; k < nnb[igd]; k++) {
                    const int jb = nb[9 * igd + k];
                    if (nch[jb] == 0 && flg[jb] == 0 && within(cen[jb], cd, dist))
                        flg[jb] = 1;
                }
            });
        }
        for (int l = L; l >= 1; l--) {
            // flag+: leaves among the dad's colleagues that touch a flagged box.
            const int *nnb = T.nnbors.get(), *nb = T.nbors.get();
            const int lo = T.lstart[l], n = T.lend[l] - T.lstart[l];
            const double dist = d2[l];
            for_each(n, s, [=] __device__(int64_t i) {
                const int b = lo + (int)i;
                const int f = flg[b];
                if (f != 1 && f != 2) return;
                const int dad = par[b];
                const double2 cb = cen[b];
                for (int k = 0; k < nnb[dad]; k++) {
                    const int jb = nb[9 * dad + k];
                    if (nch[jb] == 0 && flg[jb] == 0 && within(cen[jb], cb, dist))
                        flg[jb] = 2;
                }
            });
        }
        // Nothing flagged: the tree is level-restricted already, and every
        // remaining step (subdivision, reorganisation, colleagues, the
        // flag++ pass) would leave it as it is.
        if (count_flags(1, 2) == 0) return;
        // Subdivide flag and flag+ boxes of the original levels 1 .. L-2.
        // Their flags are final and the children of every level are
        // appended after those of the coarser levels, so all levels split
        // in one pass over the boxes in box order; the per-level counts (one
        // synchronisation) give each level's range of new boxes.
        std::vector<int> ts(L + 1, 0), te(L + 1, 0);
        std::vector<int> nsplit(L + 1, 0);
        DevBuf<double> d_bsl(T.boxsize.size(), s);
        FMM_CUDA(cudaMemcpyAsync(d_bsl.get(), T.boxsize.data(), T.boxsize.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
        if (L >= 3) {
            const int lo = T.lstart[1], n = T.lend[L - 2] - lo;
            DevBuf<int> cnt(L + 1, s), f(std::max(n, 1), s), off(std::max(n, 1), s);
            cnt.zero(s);
            int *cp = cnt.get(), *fp = f.get();
            const int *fl = iflag.get();
            for_each(n, s, [=] __device__(int64_t i) {
                const int b = lo + (int)i;
                const bool hit = fl[b] > 0;
                fp[i] = hit ? 1 : 0;
                const int key = hit ? lev[b] : -1;
                const unsigned am = __activemask();
                const unsigned peers = __match_any_sync(am, key);
                if (key >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1)
                    atomicAdd(&cp[key], __popc(peers));
            });
            exclusive_scan_i32(fp, off.get(), n, nullptr, s);
            read_small(nsplit.data(), cp, (L + 1) * sizeof(int), s);
            int nb = T.nboxes, nref = 0;
            for (int l = 1; l <= L - 2; l++) {
                ts[l + 1] = nb;
                nb += 4 * nsplit[l];
                te[l + 1] = nb;
                nref += nsplit[l];
            }
            split_items(lo, n, 0, 0, fp, off.get(), nref, d_bsl.get());
        }
        reorg(ts, te);
        computecoll(0, L);
        {
            int *fl = iflag.get();
            for_each(T.nboxes, s, [=] __device__(int64_t i) {
                if (fl[i] != 3) fl[i] = 0;
            });
        }
        // no flag++ box: no further subdivision
        if (count_flags(3, 3) == 0) return;
        std::fill(ts.begin(), ts.end(), 0);
        std::fill(te.begin(), te.end(), 0);
        for (int l = 2; l <= L - 2; l++) {
            // updateflags (tree_routs2d.c:197-252) on the level range and on
            // this level's tail: a flag++ box is subdivided only when a child
            // of one of its colleagues has children and touches it.
            const int *nnb = T.nnbors.get(), *nb = T.nbors.get(),
                      *chi = T.child.get(), *nchp = T.nchild.get();
            const double2 *cp = T.centers.get();
            int *fl = iflag.get();
            const double dist = d3[l];
            const int lo = T.lstart[l], n1 = T.lend[l] - T.lstart[l];
            const int tlo = ts[l], n2 = te[l] - ts[l];
            ts[l + 1] = T.nboxes;
            // the selection (final flag > 0) of the level and its tail, in
            // item order, scanned for the children's places; the count is
            // the one synchronisation of the level
            DevBuf<int> f(std::max(n1 + n2, 1), s), off(std::max(n1 + n2, 1), s), tot(1, s);
            int *fp = f.get();
            for_each(n1 + n2, s, [=] __device__(int64_t i) {
                const int b = i < n1 ? lo + (int)i : tlo + (int)(i - n1);
                if (fl[b] != 3) {
                    fp[i] = fl[b] > 0 ? 1 : 0;
                    return;
                }
                int f = 0;
                const double2 cb = cp[b];
                for (int k = 0; k < nnb[b] && !f; k++) {
                    const int jb = nb[9 * b + k];
                    for (int j = 0; j < 4; j++) {
                        const int kb = chi[4 * jb + j];
                        if (kb >= 0 && nchp[kb] > 0 && within(cp[kb], cb, dist)) {
                            f = 1;
                            break;
                        }
                    }
                }
                fl[b] = f;
                fp[i] = f;
            });
            int nref = 0;
            if (n1 + n2 > 0) {
                exclusive_scan_i32(fp, off.get(), n1 + n2, tot.get(), s);
                read_small(&nref, tot.get(), sizeof(int), s);
            }
            split_items(lo, n1, tlo, n2, fp, off.get(), nref, d_bsl.get());
            te[l + 1] = T.nboxes;
            // colleagues of the new boxes from their dad's (current) list
            const int nlo = ts[l + 1], nn = te[l + 1] - ts[l + 1];
            if (nn > 0) {
                int *nnbw = T.nnbors.get(), *nbw = T.nbors.get();
                const int *parp = T.parent.get(), *chip = T.child.get();
                const double2 *cq = T.centers.get();
                const double dcol = 1.05 * T.boxsize[l + 1];
                for_each(nn, s, [=] __device__(int64_t i) {
                    const int b = nlo + (int)i;
                    const int dad = parp[b];
                    const double2 cb = cq[b];
                    int cnt = 0;
                    for (int k = 0; k < nnbw[dad]; k++) {
                        const int jb = nbw[9 * dad + k];
                        for (int j = 0; j < 4; j++) {
                            const int kb = chip[4 * jb + j];
                            if (kb >= 0 && within(cq[kb], cb, dcol) && cnt < 9)
                                nbw[9 * b + cnt++] = kb;
                        }
                    }
                    nnbw[b] = cnt;
                    for (int k = cnt; k < 9; k++) nbw[9 * b + k] = -1;
                });
            }
        }
        reorg(ts, te);
        computecoll(0, L);
    }

    // pts_tree_sort (pts_tree2d.c:1087-1119): the permutation and the
    // per-box point ranges for one point set.
    void sort_points(const double2 *d_pts, int n, DevBuf<int2> &se,
                     DevBuf<int> &perm) {
        const int nb = T.nboxes, L = T.nlevels;
        se.alloc(nb, s);
        perm.alloc(std::max(n, 1), s);
        DevBuf<int> cnt(nb, s), start(nb, s);
        cnt.zero(s);
        DevBuf<uint32_t> keys(std::max(n, 1), s), vals(std::max(n, 1), s);
        int *cp = cnt.get();
        const int *nch = T.nchild.get(), *chi = T.child.get();
        const double2 *cen = T.centers.get();
        uint32_t *kp = keys.get(), *vp = vals.get();
        // leaf of every point, found by descending from the root
        for_each(n, s, [=] __device__(int64_t i) {
            const double2 p = d_pts[i];
            int b = 0;
            while (nch[b] > 0) b = chi[4 * b + child_digit(p, cen[b])];
            kp[i] = (uint32_t)b;
            atomicAdd(&cp[b], 1);
        });
        // subtree counts, deepest level first
        for (int l = L; l >= 0; l--) {
            const int lo = T.lstart[l], m = T.lend[l] - T.lstart[l];
            for_each(m, s, [=] __device__(int64_t i) {
                const int b = lo + (int)i;
                if (nch[b] > 0) {
                    int t = 0;
                    for (int j = 0; j < 4; j++) t += cp[chi[4 * b + j]];
                    cp[b] = t;
                }
            });
        }
        // depth-first starts, root first
        int *sp = start.get();
        FMM_CUDA(cudaMemsetAsync(sp, 0, sizeof(int), s));
        for (int l = 0; l < L; l++) {
            const int lo = T.lstart[l], m = T.lend[l] - T.lstart[l];
            for_each(m, s, [=] __device__(int64_t i) {
                const int b = lo + (int)i;
                if (nch[b] > 0) {
                    int st = sp[b];
                    for (int j = 0; j < 4; j++) {
                        const int c = chi[4 * b + j];
                        sp[c] = st;
                        st += cp[c];
                    }
                }
            });
        }
        int2 *sep = se.get();
        for_each(nb, s, [=] __device__(int64_t i) {
            sep[i] = make_int2(sp[i], sp[i] + cp[i]);
        });
        if (n == 0) return;
        // stable sort of (leaf start, input index)
        for_each(n, s, [=] __device__(int64_t i) {
            kp[i] = (uint32_t)sp[kp[i]];
            vp[i] = (uint32_t)i;
        });
        int bits = 1;
        while ((1LL << bits) < (long long)n) bits++;
        DevBuf<uint32_t> kt(n, s), vt(n, s);
        radix_sort_pairs(kp, vp, kt.get(), vt.get(), n, bits, s);
        FMM_CUDA(cudaMemcpyAsync(perm.get(), vp, (size_t)n * sizeof(int),
                                 cudaMemcpyDeviceToDevice, s));
    }

    // Key build: the per-box ranges become srcse / itargse as they are (the
    // leaves hold the same points, in the same order of leaves, as the
    // reference's sorted arrays); inside every leaf the points go back to
    // input order.  `idx` maps key-sorted positions to input indices.
    // prob (forests): the problem, i.e. the root, of every input point.
    void finish_points(const uint32_t *idx, const KeyView &kv, int n, const DevBuf<int2> &R,
                       DevBuf<int2> &se, DevBuf<int> &perm, const uint32_t *prob = nullptr) {
        const int nb = T.nboxes;
        se.alloc(nb, s);
        FMM_CUDA(cudaMemcpyAsync(se.get(), R.get(), (size_t)nb * sizeof(int2),
                                 cudaMemcpyDeviceToDevice, s));
        perm.alloc(std::max(n, 1), s);
        if (n == 0) return;
        const int *nch = T.nchild.get(), *chi = T.child.get();
        const int2 *rp = R.get();
        DevBuf<int> big(1, s);
        big.zero(s);
        int *bp = big.get();
        for_each(nb, s, [=] __device__(int64_t i) {
            const int2 r = rp[i];
            if (nch[i] == 0 && r.y - r.x > kLeafSort) atomicExch(bp, 1);
        });
        if (read_scalar(bp, s) == 0) {
            const int blocks = std::max(1, std::min((nb + 7) / 8, kNumSM * 16));
            leaf_order_kernel<<<blocks, 256, 0, s>>>(nb, nch, rp, idx, perm.get());
            FMM_CHECK_LAUNCH();
            return;
        }
        // some leaf holds more than kLeafSort points: stable sort of the
        // input order by the start of each point's leaf
        DevBuf<uint32_t> keys(n, s), vals(n, s), kt(n, s), vt(n, s);
        uint32_t *kp = keys.get(), *vp = vals.get();
        for_each(n, s, [=] __device__(int64_t k) {
            int b = prob ? (int)prob[idx[k]] : 0, m = 0;
            while (nch[b] > 0) {
                m++;
                b = chi[4 * b + key_digit(kv, k, m)];
            }
            kp[idx[k]] = (uint32_t)rp[b].x;
            vp[k] = (uint32_t)k;
        });
        int bits = 1;
        while ((1LL << bits) < (long long)n) bits++;
        radix_sort_pairs(kp, vp, kt.get(), vt.get(), n, bits, s);
        FMM_CUDA(cudaMemcpyAsync(perm.get(), vp, (size_t)n * sizeof(int),
                                 cudaMemcpyDeviceToDevice, s));
    }
};

// Key-sorted order of one point set: the input index of every sorted
// position and the sorted key words.
struct KeyedPoints {
    DevBuf<uint32_t> idx;
    std::vector<DevBuf<uint32_t>> words;
    KeyView view() const {
        KeyView v{};
        for (size_t w = 0; w < words.size() && w < (size_t)kKeyWords; w++) v.w[w] = words[w].get();
        return v;
    }
};

// Computes the path keys of levels 1..ds and sorts the points by them
// (stable, so equal keys keep input order).
// prob (optional): the problem of every input point of a forest, pbits its
// bit count; the points are then sorted by (problem, path).
void key_sort(const double2 *pts, int n, double2 c0, const double *d_bsl, int ds,
              KeyedPoints &kp, cudaStream_t s, const uint32_t *prob = nullptr, int pbits = 0) {
    const int nw = (ds + 15) / 16;
    kp.words.clear();
    kp.words.resize(nw);
    if (n <= 0) return;
    DevBuf<uint32_t> raw((size_t)nw * n, s);
    {
        const int blocks = (int)std::min<int64_t>(((int64_t)n + 255) / 256, kNumSM * 8);
        path_key_kernel<<<blocks, 256, 0, s>>>(pts, n, c0, d_bsl, ds, nw, raw.get());
        FMM_CHECK_LAUNCH();
    }
    kp.idx.alloc(n, s);
    uint32_t *ip = kp.idx.get();
    for_each(n, s, [=] __device__(int64_t i) { ip[i] = (uint32_t)i; });
    DevBuf<uint32_t> key(n, s), kt(n, s), vt(n, s);
    uint32_t *kp0 = key.get();
    const uint32_t *rw = raw.get();
    // least significant word first; only the bits of levels <= ds
    for (int w = nw - 1; w >= 0; w--) {
        const uint32_t *src = rw + (size_t)w * n;
        if (w == nw - 1)
            FMM_CUDA(cudaMemcpyAsync(kp0, src, (size_t)n * sizeof(uint32_t),
                                     cudaMemcpyDeviceToDevice, s));
        else
            for_each(n, s, [=] __device__(int64_t k) { kp0[k] = src[ip[k]]; });
        const int used = 2 * std::min(16, ds - 16 * w);
        const int lo = (32 - used) & ~7;
        radix_sort_pairs(kp0, ip, kt.get(), vt.get(), n, 32, s, lo);
    }
    if (prob && pbits > 0) {
        for_each(n, s, [=] __device__(int64_t k) { kp0[k] = prob[ip[k]]; });
        radix_sort_pairs(kp0, ip, kt.get(), vt.get(), n, pbits, s);
    }
    for (int w = 0; w < nw; w++) {
        kp.words[w].alloc(n, s);
        uint32_t *o = kp.words[w].get();
        if (w == 0 && !(prob && pbits > 0)) {
            FMM_CUDA(cudaMemcpyAsync(o, kp0, (size_t)n * sizeof(uint32_t),
                                     cudaMemcpyDeviceToDevice, s));
        } else {
            const uint32_t *src = rw + (size_t)w * n;
            for_each(n, s, [=] __device__(int64_t k) { o[k] = src[ip[k]]; });
        }
    }
}

// Bounding box of sources and targets (pts_tree2d.c:493-513): exact min/max.
__global__ void bbox_kernel(const double2 *__restrict__ a, int na,
                            const double2 *__restrict__ b, int nb,
                            double *__restrict__ out /* 4 per block */) {
    double xmn = INFINITY, xmx = -INFINITY, ymn = INFINITY, ymx = -INFINITY;
    const int64_t n = (int64_t)na + nb;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 p = i < na ? a[i] : b[i - na];
        xmn = fmin(xmn, p.x);
        xmx = fmax(xmx, p.x);
        ymn = fmin(ymn, p.y);
        ymx = fmax(ymx, p.y);
    }
    for (int o = 16; o > 0; o >>= 1) {
        xmn = fmin(xmn, __shfl_xor_sync(0xffffffffu, xmn, o));
        xmx = fmax(xmx, __shfl_xor_sync(0xffffffffu, xmx, o));
        ymn = fmin(ymn, __shfl_xor_sync(0xffffffffu, ymn, o));
        ymx = fmax(ymx, __shfl_xor_sync(0xffffffffu, ymx, o));
    }
    __shared__ double sh[4][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh[0][w] = xmn;
        sh[1][w] = xmx;
        sh[2][w] = ymn;
        sh[3][w] = ymx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
            xmn = fmin(xmn, sh[0][k]);
            xmx = fmax(xmx, sh[1][k]);
            ymn = fmin(ymn, sh[2][k]);
            ymx = fmax(ymx, sh[3][k]);
        }
        out[4 * blockIdx.x + 0] = xmn;
        out[4 * blockIdx.x + 1] = xmx;
        out[4 * blockIdx.x + 2] = ymn;
        out[4 * blockIdx.x + 3] = ymx;
    }
}

// Moves every point of a refined box of the current level into its child
// and counts the points per child.  The counts are aggregated before they
// reach global memory: in a shared-memory histogram when the new level has
// at most kHistChildren boxes (the shallow levels, where every point would
// otherwise hit the same few counters), by warp-level grouping otherwise.
constexpr int kHistChildren = 8192;

template <bool HIST>
__global__ void __launch_bounds__(256) assign_children_kernel(
    int n, const double2 *__restrict__ pts, int *__restrict__ pbox, int lo,
    int hi, const int *__restrict__ flag, const double2 *__restrict__ cen,
    const int *__restrict__ chi, int clo, int nchildren, int *__restrict__ cnt) {
    extern __shared__ int hist[];
    if (HIST) {
        for (int k = threadIdx.x; k < nchildren; k += blockDim.x) hist[k] = 0;
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n;
         base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        int key = -1;
        if (i < n) {
            const int b = pbox[i];
            if (b >= lo && b < hi && flag[b - lo]) {
                key = chi[4 * b + child_digit(pts[i], cen[b])];
                pbox[i] = key;
            }
        }
        if (HIST) {
            if (key >= 0) atomicAdd(&hist[key - clo], 1);
        } else {
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            if (key >= 0 && lane == __ffs(peers) - 1) atomicAdd(&cnt[key], __popc(peers));
        }
    }
    if (HIST) {
        __syncthreads();
        for (int k = threadIdx.x; k < nchildren; k += blockDim.x)
            if (hist[k]) atomicAdd(&cnt[clo + k], hist[k]);
    }
}

}  // namespace

namespace {

// The reference's level-by-level construction (pts_tree2d.c:541-611): every
// level moves each point of a refined box into its child.  Kept beside the
// key build (FMM2D_B200_TREE=levelwise) as an independent construction of
// the same tree.
void build_levelwise(const double2 *d_src, int ns, const double2 *d_targ, int nt, int ndiv,
                     int idivflag, int nlmax, double2 c0, cudaStream_t s, Tree &T) {
    Builder B(T, s);
    B.cnt_s.alloc(1, s);
    B.cnt_t.alloc(1, s);
    B.ensure(1024);
    T.nboxes = 1;
    T.lstart.push_back(0);
    T.lend.push_back(1);
    {
        double2 *cen = T.centers.get();
        int *lev = T.level.get(), *par = T.parent.get(), *nch = T.nchild.get(),
            *chi = T.child.get(), *cs = B.cnt_s.get(), *ct = B.cnt_t.get();
        const double cx = c0.x, cy = c0.y;
        for_each(1, s, [=] __device__(int64_t) {
            cen[0] = make_double2(cx, cy);
            lev[0] = 0;
            par[0] = -1;
            nch[0] = 0;
            for (int j = 0; j < 4; j++) chi[j] = -1;
            cs[0] = ns;
            ct[0] = nt;
        });
    }
    // ---- initial levelwise refinement (pts_tree2d.c:541-611) ----
    DevBuf<int> pbs(std::max(ns, 1), s), pbt(std::max(nt, 1), s);
    pbs.zero(s);
    pbt.zero(s);
    int ilev = 0;
    for (ilev = 0; ilev <= nlmax - 1; ilev++) {
        const int lo = T.lstart[ilev], hi = T.lend[ilev];
        const int *cs = B.cnt_s.get(), *ct = B.cnt_t.get();
        const int dflag = idivflag, nd = ndiv;
        auto sel = [=] __device__(int b) {
            const int nss = cs[b], ntt = ct[b];
            const int nn = dflag == 0 ? nss : (dflag == 1 ? ntt : (nss > ntt ? nss : ntt));
            return nn > nd;
        };
        T.boxsize.push_back(T.boxsize[ilev] / 2);
        const int nb0 = T.nboxes;
        // refine flags are re-derived from the counts inside refine_range;
        // keep them for the point pass below.
        DevBuf<int> f(hi - lo, s);
        int *fp = f.get();
        for_each(hi - lo, s, [=] __device__(int64_t i) { fp[i] = sel(lo + (int)i) ? 1 : 0; });
        const int nref = B.refine_range(
            lo, hi, ilev + 1, T.boxsize[ilev + 1],
            [=] __device__(int b) { return fp[b - lo] != 0; }, false);
        if (nref == 0) {
            T.boxsize.pop_back();
            break;
        }
        T.lstart.push_back(nb0);
        T.lend.push_back(T.nboxes);
        const double2 *cen = T.centers.get();
        const int *chi = T.child.get();
        const int nch = T.nboxes - nb0;
        for (int set = 0; set < 2; set++) {
            const int n = set == 0 ? ns : nt;
            if (n <= 0) continue;
            const double2 *pts = set == 0 ? d_src : d_targ;
            int *pb = set == 0 ? pbs.get() : pbt.get();
            int *cnt = set == 0 ? B.cnt_s.get() : B.cnt_t.get();
            const int blocks = (int)std::min<int64_t>(((int64_t)n + 255) / 256, kNumSM * 4);
            if (nch <= kHistChildren)
                assign_children_kernel<true><<<blocks, 256, nch * sizeof(int), s>>>(
                    n, pts, pb, lo, hi, fp, cen, chi, nb0, nch, cnt);
            else
                assign_children_kernel<false><<<blocks, 256, 0, s>>>(
                    n, pts, pb, lo, hi, fp, cen, chi, nb0, nch, cnt);
            FMM_CHECK_LAUNCH();
        }
    }
    T.nlevels = ilev;
    prof_mark("tree_refine", s);
    pbs.release();
    pbt.release();
    B.cnt_s.release();
    B.cnt_t.release();
    // ---- colleagues and level restriction ----
    B.computecoll(0, T.nlevels);
    if (T.nlevels >= 2) B.fix_lr();
    prof_mark("tree_fixlr", s);
    // ---- point permutations ----
    B.sort_points(d_src, ns, T.srcse, T.isrc);
    B.sort_points(d_targ, nt, T.trgse, T.itarg);
    prof_mark("tree_sort", s);
}

// Key build: sort the points once by their path keys of levels 1..ds, then
// refine level by level with every box's point count read off its range in
// the sorted order (three binary searches per refined box instead of a pass
// over all points).  Returns false when the tree needs digits of levels
// beyond ds; the caller then retries with more.
// Forest (F non-null): F->nroots roots share the root square; root r holds
// the points [soff[r], soff[r+1]) and [toff[r], toff[r+1]) of the
// concatenated arrays, whose problem ids (sprob, tprob) order the sort.
struct ForestRoots {
    int nroots = 1;
    const int *d_soff = nullptr, *d_toff = nullptr;
    const uint32_t *sprob = nullptr, *tprob = nullptr;
    int pbits = 0;
};

// Refinement without a host synchronisation per level: for one tree split
// on the source counts (idivflag 0) the number of boxes refined on every
// level follows from the sorted keys alone (refine_count_kernel), so the
// levels are built with known counts, each level's own device count is
// checked against them at the end, and a mismatch rebuilds the tree the
// synchronous way.  FMM2D_B200_TREE_SYNC=1 always takes the synchronous way.
bool presized_refinement(const ForestRoots *F, int idivflag) {
    const char *e = getenv("FMM2D_B200_TREE_SYNC");
    return !F && idivflag == 0 && !(e && !strcmp(e, "1"));
}

bool build_by_keys(const double2 *d_src, int ns, const double2 *d_targ, int nt, int ndiv,
                   int idivflag, int nlmax, double2 c0, int ds, cudaStream_t s, Tree &T,
                   const ForestRoots *F = nullptr, bool sync_levels = false) {
    const double bs0 = T.boxsize[0];
    T = Tree();
    T.boxsize.push_back(bs0);
    Builder B(T, s);
    B.ranges = true;
    std::vector<double> bsl(ds + 1);
    bsl[0] = bs0;
    for (int l = 1; l <= ds; l++) bsl[l] = bsl[l - 1] / 2;
    DevBuf<double> d_bsl(ds + 1, s);
    FMM_CUDA(cudaMemcpyAsync(d_bsl.get(), bsl.data(), bsl.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s));
    KeyedPoints ks, kt;
    const int nroots = F ? F->nroots : 1;
    // presized form: the targets are sorted once the source keys have shown
    // that ds digits suffice (a deeper tree retries with more digits)
    const bool known = !sync_levels && presized_refinement(F, idivflag);
    auto sort_targets = [&]() {
        key_sort(d_targ, nt, c0, d_bsl.get(), ds, kt, s, F ? F->tprob : nullptr, F ? F->pbits : 0);
        B.kvt = kt.view();
    };
    key_sort(d_src, ns, c0, d_bsl.get(), ds, ks, s, F ? F->sprob : nullptr, F ? F->pbits : 0);
    B.kvs = ks.view();
    if (!known) sort_targets();
    B.ensure(std::max(1024, 4 * nroots));
    T.nboxes = nroots;
    T.lstart.push_back(0);
    T.lend.push_back(nroots);
    {
        double2 *cen = T.centers.get();
        int *lev = T.level.get(), *par = T.parent.get(), *nch = T.nchild.get(),
            *chi = T.child.get();
        int2 *r0 = B.rs.get(), *r1 = B.rt.get();
        const int *so = F ? F->d_soff : nullptr, *to = F ? F->d_toff : nullptr;
        for_each(nroots, s, [=] __device__(int64_t i) {
            const int b = (int)i;
            cen[b] = c0;
            lev[b] = 0;
            par[b] = -1;
            nch[b] = 0;
            for (int j = 0; j < 4; j++) chi[4 * b + j] = -1;
            r0[b] = so ? make_int2(so[b], so[b + 1]) : make_int2(0, ns);
            r1[b] = to ? make_int2(to[b], to[b + 1]) : make_int2(0, nt);
        });
    }
    // known refinement counts per level (presized form): level 0 from the
    // source count, levels 1..ds from the keys, one synchronisation
    std::vector<unsigned long long> kc(65, 0);
    DevBuf<int> chk(known ? nlmax + 1 : 0, s);
    if (known) {
        kc[0] = ns > ndiv ? 1 : 0;
        if (ns > 0 && ds >= 1) {
            DevBuf<unsigned long long> dc(65, s);
            dc.zero(s);
            const int nw = (ds + 15) / 16;
            const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)ns + 255) / 256, kNumSM * 8));
            refine_count_kernel<<<blocks, 256, 0, s>>>(B.kvs, ns, ndiv, ds, nw, dc.get());
            FMM_CHECK_LAUNCH();
            read_small(kc.data() + 1, dc.get() + 1, 64 * sizeof(unsigned long long), s);
        }
        // a box of the deepest digit level still to be split: more digits
        if (ds < 64 && ds <= nlmax - 1 && kc[ds] > 0) return false;
        sort_targets();
        long long tot = nroots;
        for (int l = 0; l < std::min(ds, nlmax); l++) {
            if (kc[l] == 0) break;
            tot += 4 * (long long)kc[l];
        }
        if (tot > (long long)INT32_MAX / 20) throw FmmError(4, "tree too large");
        B.ensure((int)tot);
        chk.zero(s);
    }
    DevBuf<int> nflag(1, s);
    int ilev = 0;
    for (ilev = 0; ilev <= nlmax - 1; ilev++) {
        const int lo = T.lstart[ilev], hi = T.lend[ilev];
        const int2 *ra = B.rs.get(), *rb = B.rt.get();
        const int dflag = idivflag, nd = ndiv;
        const bool last = ilev + 1 > ds;
        if (known && last) break;  // (no box of level ds is split: checked above)
        DevBuf<int> f(hi - lo, s);
        int *fp = f.get();
        if (known) {
            // the capacity holds every level's known count; the new boxes
            // are set to defaults in the selection's own launch, so a known
            // count above the device's leaves no box unset (the ones no
            // parent fills hang under the root, and the count check after
            // the last level rebuilds the tree)
            const int nref = (int)kc[ilev], n = hi - lo;
            if (nref == 0) break;
            T.boxsize.push_back(T.boxsize[ilev] / 2);
            const int nb0 = T.nboxes;
            const int nset = std::max(n, 4 * nref);
            DevBuf<int> off(n, s);
            double2 *cen = T.centers.get();
            int *lev = T.level.get(), *par = T.parent.get(), *nch = T.nchild.get(),
                *chi = T.child.get();
            const int newlevel = ilev + 1;
            for_each(nset, s, [=] __device__(int64_t i) {
                if (i < n) {
                    const int b = lo + (int)i;
                    const int nss = ra[b].y - ra[b].x, ntt = rb[b].y - rb[b].x;
                    const int nn = dflag == 0 ? nss : (dflag == 1 ? ntt : (nss > ntt ? nss : ntt));
                    fp[i] = nn > nd ? 1 : 0;
                }
                if (i < 4 * (int64_t)nref) {
                    const int kb = nb0 + (int)i;
                    cen[kb] = cen[0];
                    par[kb] = 0;
                    lev[kb] = newlevel;
                    nch[kb] = 0;
                    for (int l = 0; l < 4; l++) chi[4 * kb + l] = -1;
                }
            });
            exclusive_scan_i32(fp, off.get(), n, chk.get() + ilev, s);
            B.split_items(lo, n, 0, 0, fp, off.get(), nref, d_bsl.get(), false);
            T.lstart.push_back(nb0);
            T.lend.push_back(T.nboxes);
            continue;
        }
        int *nf = nflag.get();
        if (last) nflag.zero(s);
        for_each(hi - lo, s, [=] __device__(int64_t i) {
            const int b = lo + (int)i;
            const int nss = ra[b].y - ra[b].x, ntt = rb[b].y - rb[b].x;
            const int nn = dflag == 0 ? nss : (dflag == 1 ? ntt : (nss > ntt ? nss : ntt));
            fp[i] = nn > nd ? 1 : 0;
            if (last && nn > nd) atomicAdd(nf, 1);
        });
        if (last) {
            if (read_scalar(nf, s) > 0) return false;
            break;
        }
        T.boxsize.push_back(T.boxsize[ilev] / 2);
        const int nb0 = T.nboxes;
        if (known && kc[ilev] == 0) {
            T.boxsize.pop_back();
            break;
        }
        const int nref = B.refine_range(
            lo, hi, ilev + 1, T.boxsize[ilev + 1],
            [=] __device__(int b) { return fp[b - lo] != 0; }, false,
            known ? (int)kc[ilev] : -1, known ? chk.get() + ilev : nullptr);
        if (nref == 0) {
            T.boxsize.pop_back();
            break;
        }
        T.lstart.push_back(nb0);
        T.lend.push_back(T.nboxes);
    }
    T.nlevels = ilev;
    if (known && ilev > 0) {
        // every level's own count must equal the one the keys gave
        std::vector<int> h(ilev);
        read_small(h.data(), chk.get(), ilev * sizeof(int), s);
        for (int l = 0; l < ilev; l++)
            if ((unsigned long long)h[l] != kc[l]) {
                T.boxsize.resize(1);
                return build_by_keys(d_src, ns, d_targ, nt, ndiv, idivflag, nlmax, c0, ds, s, T, F,
                                     true);
            }
    }
    prof_mark("tree_refine", s);
    B.computecoll(0, T.nlevels);
    if (T.nlevels >= 2) B.fix_lr();
    prof_mark("tree_fixlr", s);
    B.finish_points(ks.idx.get(), B.kvs, ns, B.rs, T.srcse, T.isrc, F ? F->sprob : nullptr);
    B.finish_points(kt.idx.get(), B.kvt, nt, B.rt, T.trgse, T.itarg, F ? F->tprob : nullptr);
    prof_mark("tree_sort", s);
    return true;
}

}  // namespace

void build_tree(const double2 *d_src, int ns, const double2 *d_targ, int nt,
                int ndiv, int idivflag, int nlmax, cudaStream_t s, Tree &T) {
    T = Tree();
    // ---- root: bounding square of sources and targets ----
    const int nblk = 2 * kNumSM;
    prof_mark("tree_start", s);
    DevBuf<double> part(4 * nblk, s);
    bbox_kernel<<<nblk, 256, 0, s>>>(d_src, ns, d_targ, nt, part.get());
    FMM_CHECK_LAUNCH();
    std::vector<double> hp(4 * nblk);
    read_small(hp.data(), part.get(), hp.size() * sizeof(double), s);
    double xmin = hp[0], xmax = hp[1], ymin = hp[2], ymax = hp[3];
    for (int k = 1; k < nblk; k++) {
        xmin = std::min(xmin, hp[4 * k]);
        xmax = std::max(xmax, hp[4 * k + 1]);
        ymin = std::min(ymin, hp[4 * k + 2]);
        ymax = std::max(ymax, hp[4 * k + 3]);
    }
    double bs0 = xmax - xmin;
    const double sizey = ymax - ymin;
    if (sizey > bs0) bs0 = sizey;
    T.boxsize.push_back(bs0);
    const double2 c0 = make_double2((xmin + xmax) / 2, (ymin + ymax) / 2);
    const char *mode = getenv("FMM2D_B200_TREE");
    if (mode && !strcmp(mode, "levelwise")) {
        build_levelwise(d_src, ns, d_targ, nt, ndiv, idivflag, nlmax, c0, s, T);
    } else {
        // first guess of the depth: a uniform distribution's, plus one level
        const int64_t nref = idivflag == 0 ? ns : (idivflag == 1 ? nt : std::max(ns, nt));
        int ds = 2;
        for (int64_t q = std::max<int64_t>(ndiv, 1); q < nref && ds < nlmax; q *= 4) ds++;
        ds = std::min(ds, nlmax);
        while (!build_by_keys(d_src, ns, d_targ, nt, ndiv, idivflag, nlmax, c0, ds, s, T))
            ds = std::min(nlmax, ds + 8);
    }
    T.d_boxsize.alloc(T.nlevels + 2, s);
    std::vector<double> bsx(T.boxsize);
    bsx.push_back(T.boxsize.back() / 2);
    FMM_CUDA(cudaMemcpyAsync(T.d_boxsize.get(), bsx.data(),
                             bsx.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaStreamSynchronize(s));
}

void build_forest(const double2 *d_src, const std::vector<int> &soff, const double2 *d_targ,
                  const std::vector<int> &toff, int ndiv, int idivflag, int nlmax, double bs0,
                  cudaStream_t s, Tree &T) {
    T = Tree();
    const int nprob = (int)soff.size() - 1;
    const int ns = soff.back(), nt = toff.back();
    T.boxsize.push_back(bs0);
    DevBuf<int> dso(nprob + 1, s), dto(nprob + 1, s);
    FMM_CUDA(cudaMemcpyAsync(dso.get(), soff.data(), (nprob + 1) * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaMemcpyAsync(dto.get(), toff.data(), (nprob + 1) * sizeof(int),
                             cudaMemcpyHostToDevice, s));
    // problem of every point (binary search in the offsets)
    DevBuf<uint32_t> sp(std::max(ns, 1), s), tp(std::max(nt, 1), s);
    auto prob_of = [&](int n, const int *off, uint32_t *out) {
        for_each(n, s, [=] __device__(int64_t i) {
            int lo = 0, hi = nprob;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (off[mid] <= i) lo = mid; else hi = mid;
            }
            out[i] = (uint32_t)lo;
        });
    };
    prob_of(ns, dso.get(), sp.get());
    prob_of(nt, dto.get(), tp.get());
    ForestRoots F;
    F.nroots = nprob;
    F.d_soff = dso.get();
    F.d_toff = dto.get();
    F.sprob = sp.get();
    F.tprob = tp.get();
    F.pbits = 1;
    while ((1 << F.pbits) < nprob) F.pbits++;
    int64_t nref = 0;
    for (int k = 0; k < nprob; k++) {
        const int64_t a = soff[k + 1] - soff[k], b = toff[k + 1] - toff[k];
        nref = std::max<int64_t>(nref, idivflag == 0 ? a : (idivflag == 1 ? b : std::max(a, b)));
    }
    int ds = 2;
    for (int64_t q = std::max<int64_t>(ndiv, 1); q < nref && ds < nlmax; q *= 4) ds++;
    ds = std::min(ds, nlmax);
    const double2 c0 = make_double2(0.0, 0.0);
    while (!build_by_keys(d_src, ns, d_targ, nt, ndiv, idivflag, nlmax, c0, ds, s, T, &F)) {
        T.boxsize.assign(1, bs0);
        ds = std::min(nlmax, ds + 8);
    }
    T.nroots = nprob;
    T.d_boxsize.alloc(T.nlevels + 2, s);
    std::vector<double> bsx(T.boxsize);
    bsx.push_back(T.boxsize.back() / 2);
    FMM_CUDA(cudaMemcpyAsync(T.d_boxsize.get(), bsx.data(), bsx.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s));
    FMM_CUDA(cudaStreamSynchronize(s));
}

void compute_lists(Tree &T, cudaStream_t s) {
    const int nb = T.nboxes;
    T.nlist1.alloc(nb, s);
    T.list1.alloc((size_t)kMaxList1 * nb, s);
    T.nlist2.alloc(nb, s);
    T.list2.alloc((size_t)kMaxList2 * nb, s);
    T.nlist3.alloc(nb, s);
    T.list3.alloc((size_t)kMaxList3 * nb, s);
    T.nlist4.alloc(nb, s);
    T.list4.alloc((size_t)kMaxList4 * nb, s);
    const int L = T.nlevels;
    std::vector<double> dcol(L + 2, 0.0), dl1(L + 2, 0.0);
    for (int l = 0; l <= L; l++) {
        dcol[l] = 1.05 * T.boxsize[l];
        const double bsn = l + 1 <= L ? T.boxsize[l + 1] : T.boxsize[l] / 2;
        dl1[l] = 1.05 * (T.boxsize[l] + bsn) / 2.0;
    }
    DevBuf<double> dd(2 * (L + 2), s);
    std::vector<double> hd(dcol);
    hd.insert(hd.end(), dl1.begin(), dl1.end());
    FMM_CUDA(cudaMemcpyAsync(dd.get(), hd.data(), hd.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s));
    DevBuf<int> err(1, s);
    err.zero(s);
    const double *dc = dd.get(), *d1 = dd.get() + (L + 2);
    const int *lev = T.level.get(), *par = T.parent.get(),
              *nch = T.nchild.get(), *chi = T.child.get(),
              *nnb = T.nnbors.get(), *nbr = T.nbors.get();
    const double2 *cen = T.centers.get();
    int *n1 = T.nlist1.get(), *l1 = T.list1.get(), *n2 = T.nlist2.get(),
        *l2 = T.list2.get(), *n3 = T.nlist3.get(), *l3 = T.list3.get(),
        *n4 = T.nlist4.get(), *l4 = T.list4.get(), *ep = err.get();
    for_each(nb, s, [=] __device__(int64_t i) {
        const int b = (int)i;
        const int l = lev[b];
        int c1 = 0, c2 = 0, c3 = 0, c4 = 0;
        if (l == 0) {
            if (nch[b] == 0) l1[kMaxList1 * b + c1++] = b;
            n1[b] = c1;
            n2[b] = 0;
            n3[b] = 0;
            n4[b] = 0;
            return;
        }
        const double2 cb = cen[b];
        const int dad = par[b];
        // list 2: children of the dad's colleagues that are not adjacent
        const double d = dc[l];
        for (int k = 0; k < nnb[dad]; k++) {
            const int jb = nbr[9 * dad + k];
            for (int j = 0; j < nch[jb]; j++) {
                const int kb = chi[4 * jb + j];
                const double2 ck = cen[kb];
                if (fabs(__dsub_rn(ck.x, cb.x)) >= d || fabs(__dsub_rn(ck.y, cb.y)) >= d) {
                    if (c2 < kMaxList2) l2[kMaxList2 * b + c2] = kb;
                    c2++;
                }
            }
        }
        // entries the reference appends while processing the coarser level:
        // leaves among the dad's colleagues go to list 1 when they touch this
        // box, else to list 4 (tree_routs2d.c:463-501), in box order.
        if (l >= 2) {
            int a1[9], a4[9], m1 = 0, m4 = 0;
            const double dd2 = d1[l - 1];
            for (int k = 0; k < nnb[dad]; k++) {
                const int ib = nbr[9 * dad + k];
                if (nch[ib] != 0) continue;
                const double2 ci = cen[ib];
                const double xd = fabs(__dsub_rn(cb.x, ci.x)), yd = fabs(__dsub_rn(cb.y, ci.y));
                if (xd < dd2 && yd < dd2)
                    a1[m1++] = ib;
                else
                    a4[m4++] = ib;
            }
            for (int x = 1; x < m1; x++)
                for (int y = x; y > 0 && a1[y - 1] > a1[y]; y--) {
                    int t = a1[y]; a1[y] = a1[y - 1]; a1[y - 1] = t;
                }
            for (int x = 1; x < m4; x++)
                for (int y = x; y > 0 && a4[y - 1] > a4[y]; y--) {
                    int t = a4[y]; a4[y] = a4[y - 1]; a4[y - 1] = t;
                }
            for (int x = 0; x < m1; x++) {
                if (c1 < kMaxList1) l1[kMaxList1 * b + c1] = a1[x];
                c1++;
            }
            for (int x = 0; x < m4; x++) {
                if (c4 < kMaxList4) l4[kMaxList4 * b + c4] = a4[x];
                c4++;
            }
        }
        // lists 1 and 3 of a leaf
        if (nch[b] == 0) {
            const double dd3 = d1[l];
            for (int k = 0; k < nnb[b]; k++) {
                const int jb = nbr[9 * b + k];
                if (nch[jb] == 0) {
                    if (c1 < kMaxList1) l1[kMaxList1 * b + c1] = jb;
                    c1++;
                } else {
                    for (int j = 0; j < nch[jb]; j++) {
                        const int kb = chi[4 * jb + j];
                        const double2 ck = cen[kb];
                        const double xd = fabs(__dsub_rn(ck.x, cb.x)), yd = fabs(__dsub_rn(ck.y, cb.y));
                        if (xd < dd3 && yd < dd3) {
                            if (c1 < kMaxList1) l1[kMaxList1 * b + c1] = kb;
                            c1++;
                        } else {
                            if (c3 < kMaxList3) l3[kMaxList3 * b + c3] = kb;
                            c3++;
                        }
                    }
                }
            }
        }
        if (c1 > kMaxList1 || c2 > kMaxList2 || c3 > kMaxList3 || c4 > kMaxList4)
            atomicExch(ep, 1);
        n1[b] = c1 < kMaxList1 ? c1 : kMaxList1;
        n2[b] = c2 < kMaxList2 ? c2 : kMaxList2;
        n3[b] = c3 < kMaxList3 ? c3 : kMaxList3;
        n4[b] = c4 < kMaxList4 ? c4 : kMaxList4;
    });
    if (read_scalar(err.get(), s) != 0)
        throw FmmError(4, "interaction list exceeds the reference's capacity");
}

void export_reference_tree(const Tree &T, int ns, int nt, int *itree,
                           int *iptr, double *centers, double *boxsize,
                           int *isrc, int *isrcse, int *itarg, int *itargse,
                           cudaStream_t s) {
    const int nb = T.nboxes, L = T.nlevels;
    auto d2h = [&](void *dst, const void *src, size_t bytes) {
        if (bytes) FMM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    };
    std::vector<int> lev(nb), par(nb), nch(nb), chi(4 * (size_t)nb), nnb(nb),
        nbr(9 * (size_t)nb);
    std::vector<int2> sse(nb), tse(nb);
    std::vector<int> ps(std::max(ns, 0)), pt(std::max(nt, 0));
    std::vector<double2> cen(nb);
    d2h(lev.data(), T.level.get(), nb * sizeof(int));
    d2h(par.data(), T.parent.get(), nb * sizeof(int));
    d2h(nch.data(), T.nchild.get(), nb * sizeof(int));
    d2h(chi.data(), T.child.get(), 4 * (size_t)nb * sizeof(int));
    d2h(nnb.data(), T.nnbors.get(), nb * sizeof(int));
    d2h(nbr.data(), T.nbors.get(), 9 * (size_t)nb * sizeof(int));
    d2h(sse.data(), T.srcse.get(), nb * sizeof(int2));
    d2h(tse.data(), T.trgse.get(), nb * sizeof(int2));
    d2h(cen.data(), T.centers.get(), nb * sizeof(double2));
    if (ns > 0) d2h(ps.data(), T.isrc.get(), ns * sizeof(int));
    if (nt > 0) d2h(pt.data(), T.itarg.get(), nt * sizeof(int));
    FMM_CUDA(cudaStreamSynchronize(s));
    int ip[8];
    ip[0] = 1;
    ip[1] = 2 * (L + 1) + 1;
    ip[2] = ip[1] + nb;
    ip[3] = ip[2] + nb;
    ip[4] = ip[3] + nb;
    ip[5] = ip[4] + 4 * nb;
    ip[6] = ip[5] + nb;
    ip[7] = ip[6] + 9 * nb;
    if (iptr)
        for (int k = 0; k < 8; k++) iptr[k] = ip[k];
    if (itree) {
        for (int l = 0; l <= L; l++) {
            itree[2 * l] = T.lstart[l] + 1;
            itree[2 * l + 1] = T.lend[l];
        }
        auto one = [](int v) { return v < 0 ? -1 : v + 1; };
        for (int b = 0; b < nb; b++) {
            itree[ip[1] - 1 + b] = lev[b];
            itree[ip[2] - 1 + b] = one(par[b]);
            itree[ip[3] - 1 + b] = nch[b];
            for (int j = 0; j < 4; j++) itree[ip[4] - 1 + 4 * b + j] = one(chi[4 * b + j]);
            itree[ip[5] - 1 + b] = nnb[b];
            for (int j = 0; j < 9; j++) itree[ip[6] - 1 + 9 * b + j] = one(nbr[9 * b + j]);
        }
    }
    if (centers)
        for (int b = 0; b < nb; b++) {
            centers[2 * b] = cen[b].x;
            centers[2 * b + 1] = cen[b].y;
        }
    if (boxsize)
        for (int l = 0; l <= L; l++) boxsize[l] = T.boxsize[l];
    if (isrc)
        for (int i = 0; i < ns; i++) isrc[i] = ps[i] + 1;
    if (itarg)
        for (int i = 0; i < nt; i++) itarg[i] = pt[i] + 1;
    if (isrcse)
        for (int b = 0; b < nb; b++) {
            isrcse[2 * b] = sse[b].x + 1;
            isrcse[2 * b + 1] = sse[b].y;
        }
    if (itargse)
        for (int b = 0; b < nb; b++) {
            itargse[2 * b] = tse[b].x + 1;
            itargse[2 * b + 1] = tse[b].y;
        }
}

}  // namespace fmm2d
