// autotune.cu -- in-library autotuner of the mixed-precision Laplace path.
//
// For one expansion order (from eps) it times full evaluations of a
// workload of the caller's shape over a grid of leaf capacities and M2L
// forms and keeps the fastest pair in the per-order tables that later
// mixed-mode calls read (mixed_leaf_capacity, m2l_form).  The timed call is
// the library's own C-ABI path with device arrays (tree, lists, all passes,
// outputs in input order), so the choice accounts for every phase the
// leaf capacity moves: a larger leaf shifts work from M2L, P2M/L2P and the
// tree to the near field.
#include "engine.cuh"
#include "laplace.cuh"
#include "runtime.cuh"

#include <chrono>
#include <vector>

namespace fmm2d {
namespace {

__device__ __forceinline__ double unit_hash(uint64_t x) {
    // splitmix64 finaliser -> [0, 1)
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    x ^= x >> 31;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

// Seeded uniform points in [0, 1]^2 and strengths in [-1, 1] + i [-1, 1].
void fill_uniform(double *a, int64_t n, uint64_t seed, double lo, double hi, cudaStream_t s) {
    for_each(n, s, [=] __device__(int64_t i) {
        a[i] = lo + (hi - lo) * unit_hash(seed * 0x100000001b3ull + (uint64_t)i);
    });
}

double time_call(const FmmCall &c, int reps) {
    double best = 1e300;
    for (int r = 0; r < reps; r++) {
        const auto t0 = std::chrono::steady_clock::now();
        const int ier = run_fmm(c);
        const auto t1 = std::chrono::steady_clock::now();
        if (ier != 0) return -1.0;
        best = std::min(best, std::chrono::duration<double, std::milli>(t1 - t0).count());
    }
    return best;
}

}  // namespace

int autotune_mixed(int kernel, double eps, int ns, const double *sources, int nt,
                   const double *targ, int ifcharge, int ifdipole, int ifpgh, int ifpghtarg,
                   int *best_ndiv, int *best_form, double *best_ms) {
    return guarded([&] {
        if (ns < 1 || nt < 0 || (!ifcharge && !ifdipole) || (kernel != kLaplace && kernel != kCauchy))
            throw FmmError(4, "autotune: invalid workload");
        const int p = laplace_nterms(eps);
        CallCtx ctx;
        cudaStream_t s = ctx.stream();
        const bool lap = kernel == kLaplace;
        // inputs: the caller's points (host or device) or seeded uniform ones
        DevBuf<double> src(2 * (size_t)ns, s), trg(2 * (size_t)std::max(nt, 1), s);
        auto put = [&](DevBuf<double> &d, const double *h, int64_t n, uint64_t seed) {
            if (h)
                FMM_CUDA(cudaMemcpyAsync(d.get(), h, n * sizeof(double), cudaMemcpyDefault, s));
            else
                fill_uniform(d.get(), n, seed, 0.0, 1.0, s);
        };
        put(src, sources, 2 * (int64_t)ns, 11);
        if (nt > 0) put(trg, targ, 2 * (int64_t)nt, 12);
        DevBuf<double> chg(2 * (size_t)ns, s), dip(2 * (size_t)ns, s), dv(2 * (size_t)ns, s);
        fill_uniform(chg.get(), 2 * (int64_t)ns, 13, -1.0, 1.0, s);
        fill_uniform(dip.get(), 2 * (int64_t)ns, 14, -1.0, 1.0, s);
        fill_uniform(dv.get(), 2 * (int64_t)ns, 15, -1.0, 1.0, s);
        const int gc = lap ? 2 : 1, hc = lap ? 3 : 1;
        auto outn = [&](int n, int pgh) {
            return (size_t)2 * n * (pgh >= 1) + (size_t)2 * gc * n * (pgh >= 2) +
                   (size_t)2 * hc * n * (pgh >= 3);
        };
        DevBuf<double> out(std::max<size_t>(outn(ns, ifpgh) + outn(nt, ifpghtarg), 1), s);
        FMM_CUDA(cudaStreamSynchronize(s));
        FmmCall c;
        c.kernel = (Kernel)kernel;
        c.nd = 1;
        c.eps = eps;
        c.ns = ns;
        c.sources = src.get();
        c.ifcharge = ifcharge;
        c.charge = ifcharge ? chg.get() : nullptr;
        c.ifdipole = ifdipole;
        c.dipstr = ifdipole ? dip.get() : nullptr;
        c.dipvec = (ifdipole && lap) ? dv.get() : nullptr;
        c.ifpgh = ifpgh;
        double *o = out.get();
        c.pot = ifpgh >= 1 ? o : nullptr;
        c.grad = ifpgh >= 2 ? o + 2 * (size_t)ns : nullptr;
        c.hess = ifpgh >= 3 ? o + 2 * (size_t)ns * (1 + gc) : nullptr;
        o += outn(ns, ifpgh);
        c.nt = nt;
        c.targ = nt > 0 ? trg.get() : nullptr;
        c.ifpghtarg = nt > 0 ? ifpghtarg : 0;
        c.pottarg = ifpghtarg >= 1 ? o : nullptr;
        c.gradtarg = ifpghtarg >= 2 ? o + 2 * (size_t)nt : nullptr;
        c.hesstarg = ifpghtarg >= 3 ? o + 2 * (size_t)nt * (1 + gc) : nullptr;
        c.precision = kPrecMixed;
        // the grid: the mixed mode's M2L forms exist for orders below 20
        const int ndivs[] = {12, 16, 20, 24, 32, 40, 48, 64};
        std::vector<int> forms = {kM2LWindow};
        if (p + 1 <= 20) {
            forms.push_back(kM2LTile);
            forms.push_back(kM2LSimt);
        }
        const int old_ndiv = mixed_leaf_capacity(p, -1);
        const int old_form = m2l_form(p);
        double best = 1e300;
        int bn = -1, bf = kM2LWindow;
        try {
            for (int f : forms)
                for (int nd : ndivs) {
                    set_mixed_leaf_capacity(p, nd);
                    set_m2l_form(p, f);
                    if (time_call(c, 1) < 0) continue;  // warm-up (pool, tables)
                    const double ms = time_call(c, 2);
                    if (ms >= 0 && ms < best) {
                        best = ms;
                        bn = nd;
                        bf = f;
                    }
                }
        } catch (...) {
            set_mixed_leaf_capacity(p, old_ndiv > 0 ? old_ndiv : 0);
            set_m2l_form(p, old_form);
            throw;
        }
        if (bn < 0) {
            set_mixed_leaf_capacity(p, old_ndiv > 0 ? old_ndiv : 0);
            set_m2l_form(p, old_form);
            throw FmmError(4, "autotune: no candidate evaluated");
        }
        set_mixed_leaf_capacity(p, bn);
        set_m2l_form(p, bf);
        if (best_ndiv) *best_ndiv = bn;
        if (best_form) *best_form = bf;
        if (best_ms) *best_ms = best;
    });
}

}  // namespace fmm2d

FMM_EXPORT int fmm2d_b200_autotune(int kernel, double eps, int ns, const double *sources, int nt,
                                   const double *targ, int ifcharge, int ifdipole, int ifpgh,
                                   int ifpghtarg, int *best_ndiv, int *best_form,
                                   double *best_ms) {
    return fmm2d::autotune_mixed(kernel, eps, ns, sources, nt, targ, ifcharge, ifdipole, ifpgh,
                                 ifpghtarg, best_ndiv, best_form, best_ms);
}

FMM_EXPORT int fmm2d_b200_set_m2l_form(int nterms, int form) {
    if (nterms < 0 || nterms >= 128 || form < 0 || form > 2) return 4;
    fmm2d::set_m2l_form(nterms, form);
    return 0;
}

FMM_EXPORT int fmm2d_b200_m2l_form(int nterms) { return fmm2d::m2l_form(nterms); }
