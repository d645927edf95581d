// engine.cu -- the driver layer of one evaluation (the reference's
// lfmm2d / cfmm2d / hfmm2d drivers, src/laplace/lfmm2d.f:29-225,
// c_translation/src/cfmm2d.c:1053-1401 and hfmm2d.c:1529-1907): inputs to
// the device, tree and lists, gather into tree order (with the
// complex-Laplace two-channel split), the FMM passes, scatter back to input
// order (with the channel recombination), outputs to the caller.
#include "engine.cuh"
#include "helmholtz.cuh"
#include "laplace.cuh"
#include "runtime.cuh"
#include "tree.cuh"

#include <atomic>
#include <memory>
#include <mutex>
#include <cmath>
#include <stdlib.h>
#include <string.h>

namespace fmm2d {

namespace {

std::atomic<int> g_precision{-1};

bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Inputs of one call on the device: either the caller's own device arrays
// or copies of its host arrays.
template <class T>
struct InBuf {
    DevBuf<T> own;
    const T *ptr = nullptr;
    void set(const void *user, size_t n, bool on_dev, cudaStream_t s) {
        if (!user || n == 0) {
            ptr = nullptr;
            return;
        }
        if (on_dev) {
            ptr = static_cast<const T *>(user);
            return;
        }
        own.alloc(n, s);
        FMM_CUDA(cudaMemcpyAsync(own.get(), user, n * sizeof(T),
                                 cudaMemcpyHostToDevice, s));
        ptr = own.get();
    }
};

// Outputs in the caller's layout on the device (T = double2 for complex
// outputs, double for the real-valued Laplace FMM).
template <class T = double2>
struct OutBufT {
    DevBuf<T> own;
    T *ptr = nullptr;
    void *user = nullptr;
    size_t n = 0;
    bool on_dev = false;
    void set(void *u, size_t count, bool dev, cudaStream_t s) {
        user = u;
        n = count;
        on_dev = dev;
        if (!u || !count) {
            ptr = nullptr;
            return;
        }
        if (dev) {
            ptr = static_cast<T *>(u);
        } else {
            own.alloc(count, s);
            ptr = own.get();
        }
    }
    void flush(cudaStream_t s) {
        if (ptr && !on_dev)
            FMM_CUDA(cudaMemcpyAsync(user, ptr, n * sizeof(T),
                                     cudaMemcpyDeviceToHost, s));
    }
};
using OutBuf = OutBufT<double2>;

}  // namespace

int current_precision() {
    int p = g_precision.load();
    if (p < 0) {
        const char *e = getenv("FMM2D_B200_PRECISION");
        p = kPrecAuto;
        if (e && !strcmp(e, "fp64")) p = kPrecFP64;
        if (e && !strcmp(e, "mixed")) p = kPrecMixed;
        if (e && !strcmp(e, "split")) p = kPrecSplit;
        g_precision.store(p);
    }
    return p;
}

void set_precision(int p) { g_precision.store(p); }

// c_translation/src/l2dterms.c:26-67: the first j >= 2 with
// |(sqrt(2)/2)^j / 1.5^(j+1)| < eps (j <= 100), else 1.
int laplace_nterms(double eps) {
    const double z2 = std::sqrt(2.0) / 2.0;
    for (int j = 2; j <= 100; j++) {
        const double t = std::pow(z2, (double)j) * (1.0 / std::pow(1.5, (double)(j + 1)));
        if (t < eps) return j;
    }
    return 1;
}

// src/laplace/lndiv2d.f:1-39 (identical table in hndiv2d.c:15-48).
int leaf_capacity(double eps, int ns, int nt) {
    if (eps >= 0.5e0) return 3;
    if (eps >= 0.5e-1) return 5;
    if (eps >= 0.5e-2) return 8;
    if (eps >= 0.5e-3) return 10;
    if (eps >= 0.5e-6) return 15;
    if (eps >= 0.5e-9) return 20;
    if (eps >= 0.5e-12) return 25;
    if (eps >= 0.5e-15) return 45;
    return ns + nt;
}

// Leaf capacity of the mixed-precision complex-Laplace evaluation.  That
// mode is held to eps against the direct sum, not to the reference's tree,
// so its leaf capacity is chosen for speed: FMM2D_B200_MIXED_NDIV, else the
// value set for the order (fmm2d_b200_set_leaf_capacity), else the default
// measured on a B200 (10^7 + 10^7 uniform points, eps 1e-6, windowed
// tensor-core M2L: 24 points per leaf 26.6 ms, 16 27.1 ms, 64 28.1 ms, 32
// and 40 slower still, their leaves straddling two levels): 24 for orders
// >= 14, 40 below.
namespace {
std::mutex g_ndiv_mu;
int g_mixed_ndiv[128] = {0};
bool g_mixed_default_off = false;
}  // namespace

int mixed_leaf_capacity(int p, int fallback) {
    const char *e = getenv("FMM2D_B200_MIXED_NDIV");
    if (e && atoi(e) > 0) return atoi(e);
    std::lock_guard<std::mutex> g(g_ndiv_mu);
    if (p >= 0 && p < 128 && g_mixed_ndiv[p] > 0) return g_mixed_ndiv[p];
    if (g_mixed_default_off) return fallback;
    return p >= 14 ? 24 : 40;
}

void set_mixed_leaf_capacity(int p, int ndiv) {
    std::lock_guard<std::mutex> g(g_ndiv_mu);
    if (p >= 0 && p < 128) g_mixed_ndiv[p] = ndiv > 0 ? ndiv : 0;
    // ndiv < 0 for every order: back to the reference's rule
    if (ndiv < 0) g_mixed_default_off = true;
    if (ndiv > 0) g_mixed_default_off = false;
}

// Geometry of a Laplace / Cauchy evaluation: the tree, its lists and the
// points in tree order.  It depends on the points, eps and the precision
// only, so a plan keeps it on the device for many evaluations.
void laplace_geometry(const FmmCall &c, bool on_dev, cudaStream_t s, LapGeometry &G) {
    // (the real-valued form takes the complex-Laplace paths with one
    // real-charge channel per density)
    const bool lap = c.kernel == kLaplace || c.kernel == kReal;
    G.lap = lap;
    G.real = c.kernel == kReal;
    G.nd = c.nd;
    G.ndc = c.kernel == kLaplace ? 2 * c.nd : c.nd;
    G.ns = c.ns;
    G.nt = c.nt;
    G.eps = c.eps;
    G.p = laplace_nterms(c.eps);
    // mixed precision for eps >= 1e-6 unless all-FP64 is requested
    const int prec = c.precision;
    G.mixed = prec == kPrecMixed || (prec == kPrecAuto && c.eps >= 0.5e-6);
    G.split = !G.mixed && prec == kPrecSplit;
    InBuf<double2> src_in, trg_in;
    src_in.set(c.sources, c.ns, on_dev, s);
    trg_in.set(c.nt > 0 ? c.targ : nullptr, c.nt, on_dev, s);
    prof_mark("h2d", s);
    int ndiv = c.ndiv >= 0 ? c.ndiv : leaf_capacity(c.eps, c.ns, c.nt);
    // (complex-Laplace only: the Cauchy potential's far field takes the
    // complex q log z, whose branch terms depend on the tree, so the Cauchy
    // form keeps the reference's tree to reproduce the reference's values)
    if (c.ndiv < 0 && G.mixed && lap) ndiv = mixed_leaf_capacity(G.p, ndiv);
    const int idivflag = c.ndiv >= 0 ? c.idivflag : 0;
    build_tree(src_in.ptr, c.ns, trg_in.ptr, c.nt, ndiv, idivflag, kMaxLevels, s, G.T);
    compute_lists(G.T, s);
    prof_mark("lists", s);
    const Tree &T = G.T;
    G.src_s.alloc(c.ns, s);
    G.trg_s.alloc(std::max(c.nt, 1), s);
    if (G.mixed) {
        G.src_hl.alloc(c.ns, s);
        G.trg_hl.alloc(std::max(c.nt, 1), s);
    }
    // points in tree order (and their hi/lo FP32 split for the mixed near
    // field)
    auto gather = [&](int n, const int *perm, const double2 *in, double2 *o, float4 *hl) {
        for_each(n, s, [=] __device__(int64_t k) {
            const double2 v = in[perm[k]];
            o[k] = v;
            if (hl) hl[k] = split_pos(v);
        });
    };
    gather(c.ns, T.isrc.get(), src_in.ptr, G.src_s.get(), G.src_hl.get());
    if (c.nt > 0) gather(c.nt, T.itarg.get(), trg_in.ptr, G.trg_s.get(), G.trg_hl.get());
    // thresh = boxsize(0) * 2^-51 (c_translation/src/cfmm2d.c:994)
    G.thresh = T.boxsize[0] * std::ldexp(1.0, -51);
    // (the caller's host copies are released on this stream)
}

// One evaluation over a geometry: strengths into tree order, the FMM
// passes, outputs back to input order in the caller's layout.  Only the
// strength and output pointers and the flags of `c` are read.
void laplace_evaluate(const FmmCall &c, const LapGeometry &G, bool on_dev, cudaStream_t s,
                      M2LCache *m2l, bool sync, const EvalIO &io) {
    const bool lap = G.lap, real = G.real;
    const int nd = G.nd, ndc = G.ndc, ns = G.ns, nt = G.nt;
    const Tree &T = G.T;
    // strengths: complex (interleaved doubles) or, for rfmm2d, real
    InBuf<double> chg_in, dip_in;
    InBuf<double> dv_in;
    const size_t sw = real ? 1 : 2;
    const bool in_dev = on_dev || io.strengths_dev;
    if (c.ifcharge) chg_in.set(c.charge, sw * nd * ns, in_dev, s);
    if (c.ifdipole) {
        dip_in.set(c.dipstr, sw * nd * ns, in_dev, s);
        if (lap) dv_in.set(c.dipvec, (size_t)2 * nd * ns, in_dev, s);
    }
    // ---- strengths into tree order (and their FP32 copies for the mixed
    // near field) ----
    DevBuf<double2> chg_s, dip_s;
    DevBuf<float2> chg32, dip32;
    const bool mixed = G.mixed;
    {
        const int *perm = T.isrc.get();
        auto put = [=] __device__(double2 *o, float2 *o32, size_t a, double2 v) {
            if (o) o[a] = v;
            if (o32) o32[a] = make_float2((float)v.x, (float)v.y);
        };
        // one pass over the points for charges and dipoles together; the
        // mixed mode's passes read only the FP32 copies while the P2M and
        // P2L run their warp-per-box forms (order <= 39), so the FP64
        // copies are not made there
        const bool ifc = c.ifcharge, ifd = c.ifdipole;
        const bool keep64 = !mixed || G.p + 1 > 40;
        if (ifc) {
            if (keep64) chg_s.alloc((size_t)ns * ndc, s);
            if (mixed) chg32.alloc((size_t)ns * ndc, s);
        }
        if (ifd) {
            if (keep64) dip_s.alloc((size_t)ns * ndc, s);
            if (mixed) dip32.alloc((size_t)ns * ndc, s);
        }
        const double2 *q = reinterpret_cast<const double2 *>(chg_in.ptr),
                      *d = reinterpret_cast<const double2 *>(dip_in.ptr);
        const double *qr = chg_in.ptr, *dr = dip_in.ptr;
        const double *dv = dv_in.ptr;
        double2 *qo = chg_s.get(), *dout = dip_s.get();
        float2 *q32 = chg32.get(), *d32 = dip32.get();
        for_each(ns, s, [=] __device__(int64_t k) {
            const int i = perm[k];
            for (int j = 0; j < nd; j++) {
                if (real) {
                    // charge1 = charge, dipstr1 = dipstr * (-(v1 + i v2))
                    // (rfmm2d.f:133-149)
                    if (ifc) put(qo, q32, (size_t)k * ndc + j, make_double2(qr[(size_t)i * nd + j], 0.0));
                    if (ifd) {
                        const double dd = dr[(size_t)i * nd + j];
                        const double v1 = dv[((size_t)i * 2 + 0) * nd + j];
                        const double v2 = dv[((size_t)i * 2 + 1) * nd + j];
                        put(dout, d32, (size_t)k * ndc + j, make_double2(-dd * v1, -dd * v2));
                    }
                    continue;
                }
                if (ifc) {
                    const double2 v = q[(size_t)i * nd + j];
                    if (lap) {
                        // charge1(1:2, j, i) = (Re q, Im q)  (lfmm2d.f:141-147)
                        put(qo, q32, (size_t)k * ndc + 2 * j, make_double2(v.x, 0.0));
                        put(qo, q32, (size_t)k * ndc + 2 * j + 1, make_double2(v.y, 0.0));
                    } else {
                        put(qo, q32, (size_t)k * ndc + j, v);
                    }
                }
                if (ifd) {
                    const double2 v = d[(size_t)i * nd + j];
                    if (lap) {
                        // dipstr1 = (Re d, Im d) * (-(v1 + i v2))  (lfmm2d.f:149-157)
                        const double v1 = dv[((size_t)i * 2 + 0) * nd + j];
                        const double v2 = dv[((size_t)i * 2 + 1) * nd + j];
                        put(dout, d32, (size_t)k * ndc + 2 * j, make_double2(-v.x * v1, -v.x * v2));
                        put(dout, d32, (size_t)k * ndc + 2 * j + 1,
                            make_double2(-v.y * v1, -v.y * v2));
                    } else {
                        put(dout, d32, (size_t)k * ndc + j, v);
                    }
                }
            }
        });
    }
    prof_mark("gather", s);
    chg_in.own.release();
    dip_in.own.release();
    dv_in.own.release();
    // ---- outputs in tree order ----
    const int spgh = c.ifpgh, tpgh = nt > 0 ? c.ifpghtarg : 0;
    DevBuf<double2> spot, sgrad, shess, tpot, tgrad, thess;
    // (the far-field pass is the first writer of every output)
    auto mk = [&](DevBuf<double2> &b, int n, bool need) {
        if (need && n > 0) b.alloc((size_t)n * ndc, s);
    };
    mk(spot, ns, spgh >= 1);
    mk(sgrad, ns, spgh >= 2);
    mk(shess, ns, spgh >= 3);
    mk(tpot, nt, tpgh >= 1);
    mk(tgrad, nt, tpgh >= 2);
    mk(thess, nt, tpgh >= 3);
    CauchyProblem P;
    P.ndc = ndc;
    P.p = G.p;
    P.ifcharge = c.ifcharge;
    P.ifdipole = c.ifdipole;
    P.src = G.src_s.get();
    P.charge = chg_s.get();
    P.dipstr = dip_s.get();
    P.sset.pos = G.src_s.get();
    P.sset.se = T.srcse.get();
    P.sset.n = ns;
    P.sset.pgh = spgh;
    P.sset.pot = spot.get();
    P.sset.grad = sgrad.get();
    P.sset.hess = shess.get();
    P.tset.pos = G.trg_s.get();
    P.tset.se = T.trgse.get();
    P.tset.n = nt;
    P.tset.pgh = tpgh;
    P.tset.pot = tpot.get();
    P.tset.grad = tgrad.get();
    P.tset.hess = thess.get();
    P.thresh = G.thresh;
    P.ifnear = c.ifnear;
    P.mixed = G.mixed;
    P.split = G.split;
    P.real_charge = lap;
    P.m2l_cache = m2l;
    if (mixed) {
        P.charge32 = chg32.get();
        P.dipstr32 = dip32.get();
        P.src_hl = G.src_hl.get();
        P.trg_hl = G.trg_hl.get();
    }
    // ---- back to input order, in the caller's layout ----
    // (with a copy stream, each output's device-to-host copy starts once its
    // scatter is done; the staging buffers live until the copies are)
    std::vector<std::unique_ptr<OutBufT<double2>>> keep2;
    std::vector<std::unique_ptr<OutBufT<double>>> keep1;
    std::vector<cudaEvent_t> evs;
    const bool overlap = io.copy && !on_dev;
    // (declared after the buffers, so it runs first: on any exit, copies
    // still in flight finish before the buffers are freed)
    struct CopyGuard {
        cudaStream_t c;
        std::vector<cudaEvent_t> &e;
        ~CopyGuard() {
            if (c) cudaStreamSynchronize(c);
            for (cudaEvent_t x : e) cudaEventDestroy(x);
        }
    } copy_guard{overlap ? io.copy : nullptr, evs};
    auto flush = [&](auto &ob) {
        if (!ob.ptr || on_dev) return;
        if (!overlap) {
            ob.flush(s);
            return;
        }
        cudaEvent_t e;
        FMM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        evs.push_back(e);
        FMM_CUDA(cudaEventRecord(e, s));
        FMM_CUDA(cudaStreamWaitEvent(io.copy, e, 0));
        ob.flush(io.copy);
    };
    auto unsort = [&](int n, const int *perm, int pgh, const DevBuf<double2> &po,
                      const DevBuf<double2> &gr, const DevBuf<double2> &he,
                      double *upot, double *ugrad, double *uhess) {
        if (pgh <= 0 || n <= 0) return;
        const int gcomp = lap ? 2 : 1, hcomp = lap ? 3 : 1;
        // Walked in input order through the inverse permutation: each point
        // reads its outputs in tree order (whole 32-byte sectors) and the
        // writes in the caller's layout are coalesced, instead of writing
        // half sectors at random (measured on a B200: the scatters of
        // 10^7 + 10^7 points with pot and grad took 1.13 ms against 1.55).
        DevBuf<int> invb(n, s);
        int *inv = invb.get();
        for_each(n, s, [=] __device__(int64_t k) { inv[perm[k]] = (int)k; });
        if (real) {
            // rfmm2d.f:159-214: pot = Re pot1, grad = (Re g1, -Im g1),
            // hess = (Re h1, -Im h1, -Re h1), all real
            keep1.emplace_back(new OutBufT<double>());
            keep1.emplace_back(new OutBufT<double>());
            keep1.emplace_back(new OutBufT<double>());
            OutBufT<double> &op = *keep1[keep1.size() - 3], &og = *keep1[keep1.size() - 2],
                            &oh = *keep1.back();
            op.set(upot, (size_t)nd * n, on_dev, s);
            if (pgh >= 2) og.set(ugrad, (size_t)nd * 2 * n, on_dev, s);
            if (pgh >= 3) oh.set(uhess, (size_t)nd * 3 * n, on_dev, s);
            const double2 *P0 = po.get(), *G0 = gr.get(), *H0 = he.get();
            double *up = op.ptr, *ug = og.ptr, *uh = oh.ptr;
            for_each(n, s, [=] __device__(int64_t i) {
                const int k = inv[i];
                for (int j = 0; j < nd; j++) {
                    const size_t a = (size_t)k * ndc + j;
                    up[(size_t)i * nd + j] = P0[a].x;
                    if (pgh >= 2) {
                        ug[((size_t)i * 2 + 0) * nd + j] = G0[a].x;
                        ug[((size_t)i * 2 + 1) * nd + j] = -G0[a].y;
                    }
                    if (pgh >= 3) {
                        uh[((size_t)i * 3 + 0) * nd + j] = H0[a].x;
                        uh[((size_t)i * 3 + 1) * nd + j] = -H0[a].y;
                        uh[((size_t)i * 3 + 2) * nd + j] = -H0[a].x;
                    }
                }
            });
            flush(op);
            flush(og);
            flush(oh);
            return;
        }
        keep2.emplace_back(new OutBuf());
        keep2.emplace_back(new OutBuf());
        keep2.emplace_back(new OutBuf());
        OutBuf &op = *keep2[keep2.size() - 3], &og = *keep2[keep2.size() - 2], &oh = *keep2.back();
        op.set(upot, (size_t)nd * n, on_dev, s);
        if (pgh >= 2) og.set(ugrad, (size_t)nd * gcomp * n, on_dev, s);
        if (pgh >= 3) oh.set(uhess, (size_t)nd * hcomp * n, on_dev, s);
        const double2 *P0 = po.get(), *G0 = gr.get(), *H0 = he.get();
        double2 *up = op.ptr, *ug = og.ptr, *uh = oh.ptr;
        for_each(n, s, [=] __device__(int64_t i) {
            const int k = inv[i];
            for (int j = 0; j < nd; j++) {
                if (lap) {
                    // lfmm2d.f:168-225: pot = Re pot1(1) + i Re pot1(2),
                    // grad(1) = Re g1 + i Re g2, grad(2) = -Im g1 - i Im g2,
                    // hess likewise with hess(3) = -hess(1).
                    const size_t a = (size_t)k * ndc + 2 * j;
                    const double2 p1 = P0[a], p2 = P0[a + 1];
                    up[(size_t)i * nd + j] = make_double2(p1.x, p2.x);
                    if (pgh >= 2) {
                        const double2 g1 = G0[a], g2 = G0[a + 1];
                        ug[((size_t)i * 2 + 0) * nd + j] = make_double2(g1.x, g2.x);
                        ug[((size_t)i * 2 + 1) * nd + j] = make_double2(-g1.y, -g2.y);
                    }
                    if (pgh >= 3) {
                        const double2 h1 = H0[a], h2 = H0[a + 1];
                        uh[((size_t)i * 3 + 0) * nd + j] = make_double2(h1.x, h2.x);
                        uh[((size_t)i * 3 + 1) * nd + j] = make_double2(-h1.y, -h2.y);
                        uh[((size_t)i * 3 + 2) * nd + j] = make_double2(-h1.x, -h2.x);
                    }
                } else {
                    const size_t a = (size_t)k * ndc + j, o = (size_t)i * nd + j;
                    up[o] = P0[a];
                    if (pgh >= 2) ug[o] = G0[a];
                    if (pgh >= 3) uh[o] = H0[a];
                }
            }
        });
        flush(op);
        flush(og);
        flush(oh);
    };
    cauchy_fmm(T, P, s);
    unsort(nt, T.itarg.get(), tpgh, tpot, tgrad, thess, c.pottarg, c.gradtarg, c.hesstarg);
    unsort(ns, T.isrc.get(), spgh, spot, sgrad, shess, c.pot, c.grad, c.hess);
    if (overlap) {
        // the call ends (and the staging buffers are freed on s) after the copies
        cudaEvent_t e;
        FMM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        evs.push_back(e);
        FMM_CUDA(cudaEventRecord(e, io.copy));
        FMM_CUDA(cudaStreamWaitEvent(s, e, 0));
    }
    // (the outputs, copied to host arrays where the caller's are, are
    // complete when the call returns)
    if (sync) FMM_CUDA(cudaStreamSynchronize(s));
    prof_mark("scatter_d2h", s);
}

namespace {

void run_laplace_family(const FmmCall &c, CallCtx &ctx) {
    cudaStream_t s = ctx.stream();
    const bool on_dev = is_device_ptr(c.sources);
    prof_begin(s, c.timeinfo != nullptr);
    if (on_dev) {
        LapGeometry G;
        laplace_geometry(c, on_dev, s, G);
        laplace_evaluate(c, G, on_dev, s);
    } else {
        // Host arrays: the positions go to the device first, at the link's
        // full rate; the strengths follow on the copy stream while the tree
        // is built on s; the targets' outputs come back on the copy stream
        // while the sources' are computed, then the sources'.
        cudaStream_t cs = ctx.copy_stream();
        const size_t sw = c.kernel == kReal ? 1 : 2;
        const size_t nsd = (size_t)c.nd * c.ns;
        DevBuf<double2> dsrc(c.ns, s), dtrg(c.nt > 0 ? c.nt : 0, s);
        FMM_CUDA(cudaMemcpyAsync(dsrc.get(), c.sources, (size_t)c.ns * sizeof(double2),
                                 cudaMemcpyHostToDevice, s));
        if (c.nt > 0 && c.targ)
            FMM_CUDA(cudaMemcpyAsync(dtrg.get(), c.targ, (size_t)c.nt * sizeof(double2),
                                     cudaMemcpyHostToDevice, s));
        DevBuf<double> dq, dd, dv;
        if (c.ifcharge) dq.alloc(sw * nsd, s);
        if (c.ifdipole) {
            dd.alloc(sw * nsd, s);
            if (c.kernel != kCauchy) dv.alloc(2 * nsd, s);
        }
        cudaEvent_t e0, e1;
        FMM_CUDA(cudaEventCreateWithFlags(&e0, cudaEventDisableTiming));
        FMM_CUDA(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
        // (declared after the buffers, so it runs first: on any exit the
        // copies finish before the buffers are freed)
        struct EvGuard {
            cudaEvent_t a, b;
            cudaStream_t cs;
            ~EvGuard() {
                cudaStreamSynchronize(cs);
                cudaEventDestroy(a);
                cudaEventDestroy(b);
            }
        } guard{e0, e1, cs};
        // (after the positions' copies and the allocations, which are ordered on s)
        FMM_CUDA(cudaEventRecord(e0, s));
        FMM_CUDA(cudaStreamWaitEvent(cs, e0, 0));
        auto up = [&](DevBuf<double> &b, const double *h, size_t n) {
            if (b.get() && h)
                FMM_CUDA(cudaMemcpyAsync(b.get(), h, n * sizeof(double), cudaMemcpyHostToDevice, cs));
        };
        up(dq, c.charge, sw * nsd);
        up(dd, c.dipstr, sw * nsd);
        up(dv, c.dipvec, 2 * nsd);
        FMM_CUDA(cudaEventRecord(e1, cs));
        LapGeometry G;
        FmmCall cg = c;
        cg.sources = reinterpret_cast<const double *>(dsrc.get());
        cg.targ = c.nt > 0 ? reinterpret_cast<const double *>(dtrg.get()) : nullptr;
        laplace_geometry(cg, true, s, G);
        dsrc.release();
        dtrg.release();
        FMM_CUDA(cudaStreamWaitEvent(s, e1, 0));
        FmmCall c2 = c;
        c2.charge = c.ifcharge ? dq.get() : nullptr;
        c2.dipstr = c.ifdipole ? dd.get() : nullptr;
        c2.dipvec = (c.ifdipole && c.kernel != kCauchy) ? dv.get() : nullptr;
        EvalIO io;
        io.strengths_dev = true;
        io.copy = cs;
        laplace_evaluate(c2, G, false, s, nullptr, true, io);
    }
    prof_end(s);
    if (c.timeinfo) prof_timeinfo(c.timeinfo);
}


// Gathers the Helmholtz inputs into tree order: charges and dipole
// strengths (nd, ns) complex, dipole vectors (nd, 2, ns) as (v1, v2) pairs.
struct HelmInputs {
    DevBuf<double2> src, trg, chg, dip, dv;
};

void gather_helm(const FmmCall &c, const Tree &T, const double2 *src, const double2 *trg,
                 const double2 *q, const double2 *d, const double *dv, HelmInputs &o,
                 cudaStream_t s) {
    const int nd = c.nd, ns = c.ns, nt = c.nt;
    o.src.alloc(ns, s);
    o.trg.alloc(std::max(nt, 1), s);
    const int *perm = T.isrc.get();
    {
        double2 *so = o.src.get();
        for_each(ns, s, [=] __device__(int64_t k) { so[k] = src[perm[k]]; });
    }
    if (nt > 0) {
        const int *pt = T.itarg.get();
        double2 *to = o.trg.get();
        for_each(nt, s, [=] __device__(int64_t k) { to[k] = trg[pt[k]]; });
    }
    if (c.ifcharge) {
        o.chg.alloc((size_t)ns * nd, s);
        double2 *qo = o.chg.get();
        for_each((int64_t)ns * nd, s, [=] __device__(int64_t t) {
            const int64_t k = t / nd, j = t % nd;
            qo[t] = q[(int64_t)perm[k] * nd + j];
        });
    }
    if (c.ifdipole) {
        o.dip.alloc((size_t)ns * nd, s);
        o.dv.alloc((size_t)ns * nd, s);
        double2 *dout = o.dip.get(), *vout = o.dv.get();
        for_each((int64_t)ns * nd, s, [=] __device__(int64_t t) {
            const int64_t k = t / nd, j = t % nd, i = perm[k];
            dout[t] = d[i * nd + j];
            vout[t] = make_double2(dv[(i * 2 + 0) * nd + j], dv[(i * 2 + 1) * nd + j]);
        });
    }
}

void run_helmholtz(const FmmCall &c, CallCtx &ctx) {
    cudaStream_t s = ctx.stream();
    const int nd = c.nd, ns = c.ns, nt = c.nt;
    if (c.zk[0] == 0.0 && c.zk[1] == 0.0) throw FmmError(4, "zk must be nonzero");
    const bool on_dev = is_device_ptr(c.sources);
    prof_begin(s, c.timeinfo != nullptr);
    InBuf<double2> src_in, trg_in, chg_in, dip_in;
    InBuf<double> dv_in;
    src_in.set(c.sources, ns, on_dev, s);
    trg_in.set(nt > 0 ? c.targ : nullptr, nt, on_dev, s);
    // Host arrays: the strengths go to the device on the copy stream while
    // the tree is built on s, and the outputs come back on it array by array.
    cudaStream_t cs = on_dev ? nullptr : ctx.copy_stream();
    std::vector<cudaEvent_t> evs;
    auto event_on = [&](cudaStream_t st) {
        cudaEvent_t e;
        FMM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        evs.push_back(e);
        FMM_CUDA(cudaEventRecord(e, st));
        return e;
    };
    if (on_dev) {
        if (c.ifcharge) chg_in.set(c.charge, (size_t)nd * ns, true, s);
        if (c.ifdipole) {
            dip_in.set(c.dipstr, (size_t)nd * ns, true, s);
            dv_in.set(c.dipvec, (size_t)2 * nd * ns, true, s);
        }
    } else {
        if (c.ifcharge) chg_in.own.alloc((size_t)nd * ns, s);
        if (c.ifdipole) {
            dip_in.own.alloc((size_t)nd * ns, s);
            dv_in.own.alloc((size_t)2 * nd * ns, s);
        }
        FMM_CUDA(cudaStreamWaitEvent(cs, event_on(s), 0));  // the allocations are ordered on s
        auto up = [&](auto &b, const double *h, size_t bytes) {
            if (!b.own.get() || !h) return;
            FMM_CUDA(cudaMemcpyAsync(b.own.get(), h, bytes, cudaMemcpyHostToDevice, cs));
            b.ptr = b.own.get();
        };
        up(chg_in, c.charge, (size_t)nd * ns * sizeof(double2));
        up(dip_in, c.dipstr, (size_t)nd * ns * sizeof(double2));
        up(dv_in, c.dipvec, (size_t)2 * nd * ns * sizeof(double));
    }
    const cudaEvent_t strengths_in = on_dev ? nullptr : event_on(cs);
    std::vector<std::unique_ptr<OutBuf>> keep;  // output staging, alive until the copies end
    // (declared after every buffer that a copy uses, so that on any exit the
    // copies still in flight finish before those buffers are freed)
    struct CopyGuard {
        cudaStream_t c;
        std::vector<cudaEvent_t> &e;
        ~CopyGuard() {
            if (c) cudaStreamSynchronize(c);
            for (cudaEvent_t x : e) cudaEventDestroy(x);
        }
    } copy_guard{cs, evs};
    prof_mark("h2d", s);
    // hndiv2d (c_translation/src/hndiv2d.c) has the lndiv2d table
    const int ndiv = c.ndiv >= 0 ? c.ndiv : leaf_capacity(c.eps, ns, nt);
    const int idivflag = c.ndiv >= 0 ? c.idivflag : 0;
    Tree T;
    build_tree(src_in.ptr, ns, trg_in.ptr, nt, ndiv, idivflag, kMaxLevels, s, T);
    compute_lists(T, s);
    prof_mark("lists", s);
    HelmInputs in;
    if (strengths_in) FMM_CUDA(cudaStreamWaitEvent(s, strengths_in, 0));
    gather_helm(c, T, src_in.ptr, trg_in.ptr, chg_in.ptr, dip_in.ptr, dv_in.ptr, in, s);
    prof_mark("gather", s);
    src_in.own.release();
    chg_in.own.release();
    dip_in.own.release();
    dv_in.own.release();
    const int spgh = c.ifpgh, tpgh = nt > 0 ? c.ifpghtarg : 0;
    DevBuf<double2> spot, sgrad, shess, tpot, tgrad, thess;
    auto mk = [&](DevBuf<double2> &b, int n, int comps, bool need) {
        if (need && n > 0) b.alloc((size_t)n * nd * comps, s);
    };
    mk(spot, ns, 1, spgh >= 1);
    mk(sgrad, ns, 2, spgh >= 2);
    mk(shess, ns, 3, spgh >= 3);
    mk(tpot, nt, 1, tpgh >= 1);
    mk(tgrad, nt, 2, tpgh >= 2);
    mk(thess, nt, 3, tpgh >= 3);
    HelmProblem P;
    P.nd = nd;
    P.zk = make_double2(c.zk[0], c.zk[1]);
    P.eps = c.eps;
    P.ifcharge = c.ifcharge;
    P.ifdipole = c.ifdipole;
    P.src = in.src.get();
    P.charge = in.chg.get();
    P.dipstr = in.dip.get();
    P.dipvec = in.dv.get();
    P.sset = HPointSet{in.src.get(), T.srcse.get(), ns, spgh, spot.get(), sgrad.get(), shess.get()};
    P.tset = HPointSet{in.trg.get(), T.trgse.get(), nt, tpgh, tpot.get(), tgrad.get(), thess.get()};
    P.ifnear = c.ifnear;
    P.mixed = c.precision == kPrecMixed || (c.precision == kPrecAuto && c.eps >= 0.5e-6);
    helmholtz_fmm(T, P, s);
    // back to input order: per point, nd * comps consecutive values
    auto unsort = [&](int n, const int *perm, int pgh, const DevBuf<double2> &po,
                      const DevBuf<double2> &gr, const DevBuf<double2> &he, double *upot,
                      double *ugrad, double *uhess) {
        if (pgh <= 0 || n <= 0) return;
        auto one = [&](const DevBuf<double2> &b, double *user, int comps) {
            keep.emplace_back(new OutBuf());
            OutBuf &ob = *keep.back();
            ob.set(user, (size_t)n * nd * comps, on_dev, s);
            const int w = nd * comps;
            const double2 *src = b.get();
            double2 *dst = ob.ptr;
            for_each((int64_t)n * w, s, [=] __device__(int64_t t) {
                const int64_t k = t / w, j = t % w;
                dst[(int64_t)perm[k] * w + j] = src[t];
            });
            if (cs) {
                FMM_CUDA(cudaStreamWaitEvent(cs, event_on(s), 0));
                ob.flush(cs);
            }
        };
        one(po, upot, 1);
        if (pgh >= 2) one(gr, ugrad, 2);
        if (pgh >= 3) one(he, uhess, 3);
    };
    unsort(ns, T.isrc.get(), spgh, spot, sgrad, shess, c.pot, c.grad, c.hess);
    unsort(nt, T.itarg.get(), tpgh, tpot, tgrad, thess, c.pottarg, c.gradtarg, c.hesstarg);
    if (cs) FMM_CUDA(cudaStreamWaitEvent(s, event_on(cs), 0));
    FMM_CUDA(cudaStreamSynchronize(s));
    prof_mark("scatter_d2h", s);
    prof_end(s);
    if (c.timeinfo) prof_timeinfo(c.timeinfo);
}

}  // namespace

// Helmholtz direct sum over all sources at nt targets (h2d_direct*,
// c_translation/src/helmkernels2d.c); increments pot(nd,nt), grad(nd,2,nt),
// hess(nd,3,nt).  Host or device arrays.
int run_helm_direct(int nd, const double *zk, int ns, const double *sources, int ifcharge,
                    const double *charge, int ifdipole, const double *dipstr,
                    const double *dipvec, int nt, const double *targ, int ifpgh, double *pot,
                    double *grad, double *hess, double thresh) {
    return guarded([&] {
        if (nd < 1 || ns < 0 || nt < 0 || ifpgh < 1 || ifpgh > 3 || (!ifcharge && !ifdipole))
            throw FmmError(4, "invalid direct-sum arguments");
        if (nt == 0 || ns == 0) return;
        CallCtx ctx;
        cudaStream_t s = ctx.stream();
        const bool od = is_device_ptr(sources);
        InBuf<double2> S, Tg, Q, D;
        InBuf<double> V;
        S.set(sources, ns, od, s);
        Tg.set(targ, nt, od, s);
        if (ifcharge) Q.set(charge, (size_t)nd * ns, od, s);
        DevBuf<double2> dv;
        if (ifdipole) {
            D.set(dipstr, (size_t)nd * ns, od, s);
            V.set(dipvec, (size_t)2 * nd * ns, od, s);
            dv.alloc((size_t)nd * ns, s);
            const double *vp = V.ptr;
            double2 *vo = dv.get();
            const int ndd = nd;
            for_each((int64_t)ns * nd, s, [=] __device__(int64_t t) {
                const int64_t k = t / ndd, j = t % ndd;
                vo[t] = make_double2(vp[(k * 2 + 0) * ndd + j], vp[(k * 2 + 1) * ndd + j]);
            });
        }
        // outputs are incremented: bring the caller's values in
        OutBuf Po, G, H;
        Po.set(pot, (size_t)nd * nt, od, s);
        if (ifpgh >= 2) G.set(grad, (size_t)nd * 2 * nt, od, s);
        if (ifpgh >= 3) H.set(hess, (size_t)nd * 3 * nt, od, s);
        auto load = [&](OutBuf &b, const double *u, size_t n) {
            if (b.ptr && !od)
                FMM_CUDA(cudaMemcpyAsync(b.ptr, u, n * sizeof(double2), cudaMemcpyHostToDevice, s));
        };
        load(Po, pot, (size_t)nd * nt);
        if (ifpgh >= 2) load(G, grad, (size_t)nd * 2 * nt);
        if (ifpgh >= 3) load(H, hess, (size_t)nd * 3 * nt);
        HelmProblem P;
        P.nd = nd;
        P.zk = make_double2(zk[0], zk[1]);
        P.ifcharge = ifcharge;
        P.ifdipole = ifdipole;
        P.src = S.ptr;
        P.charge = Q.ptr;
        P.dipstr = D.ptr;
        P.dipvec = dv.get();
        HPointSet X{Tg.ptr, nullptr, nt, ifpgh, Po.ptr, G.ptr, H.ptr};
        helmholtz_direct(P, ns, X, thresh, s);
        Po.flush(s);
        G.flush(s);
        H.flush(s);
        FMM_CUDA(cudaStreamSynchronize(s));
    });
}


namespace {

// Bounding box of each problem's sources and targets: one block per
// problem, exact min / max (as the single-problem bounding box).
__global__ void __launch_bounds__(256) seg_bbox_kernel(const double2 *__restrict__ src,
                                                       const int *__restrict__ so,
                                                       const double2 *__restrict__ trg,
                                                       const int *__restrict__ to,
                                                       double *__restrict__ out) {
    const int k = blockIdx.x;
    double xmn = INFINITY, xmx = -INFINITY, ymn = INFINITY, ymx = -INFINITY;
    for (int set = 0; set < 2; set++) {
        const double2 *p = set ? trg : src;
        const int a = set ? to[k] : so[k], b = set ? to[k + 1] : so[k + 1];
        for (int i = a + threadIdx.x; i < b; i += blockDim.x) {
            const double2 v = p[i];
            xmn = fmin(xmn, v.x);
            xmx = fmax(xmx, v.x);
            ymn = fmin(ymn, v.y);
            ymx = fmax(ymx, v.y);
        }
    }
    __shared__ double sh[4][256];
    sh[0][threadIdx.x] = xmn;
    sh[1][threadIdx.x] = xmx;
    sh[2][threadIdx.x] = ymn;
    sh[3][threadIdx.x] = ymx;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            sh[0][threadIdx.x] = fmin(sh[0][threadIdx.x], sh[0][threadIdx.x + h]);
            sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + h]);
            sh[2][threadIdx.x] = fmin(sh[2][threadIdx.x], sh[2][threadIdx.x + h]);
            sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 4) out[4 * k + threadIdx.x] = sh[threadIdx.x][0];
}

// p -= center of its problem, one block per problem.
__global__ void __launch_bounds__(256) seg_shift_kernel(double2 *__restrict__ p,
                                                        const int *__restrict__ off,
                                                        const double2 *__restrict__ cen) {
    const int k = blockIdx.x;
    const double2 c = cen[k];
    for (int i = off[k] + threadIdx.x; i < off[k + 1]; i += blockDim.x) {
        const double2 v = p[i];
        p[i] = make_double2(v.x - c.x, v.y - c.y);
    }
}

}  // namespace

int run_laplace_batch(const BatchCall &b) {
    return guarded([&] {
        const int np = b.nprob;
        if (np < 1) throw FmmError(4, "batch: no problems");
        if (b.kernel != kLaplace && b.kernel != kCauchy)
            throw FmmError(4, "batch: kernel must be 0 (lfmm2d) or 1 (cfmm2d)");
        const bool ifc = b.charge != nullptr, ifd = b.dipstr != nullptr;
        const bool lap = b.kernel == kLaplace;
        if (!ifc && !ifd) throw FmmError(4, "batch: no charges and no dipoles");
        if (ifd && lap && !b.dipvec) throw FmmError(4, "batch: dipole vectors missing");
        std::vector<int> so(np + 1, 0), to(np + 1, 0);
        for (int k = 0; k < np; k++) {
            const int nk = b.ns[k], mk = b.nt ? b.nt[k] : 0;
            if (nk < 1 || mk < 0) throw FmmError(4, "batch: ns must be >= 1 and nt >= 0");
            if ((int64_t)so[k] + nk > INT32_MAX || (int64_t)to[k] + mk > INT32_MAX)
                throw FmmError(4, "batch: more than 2^31 points in all");
            so[k + 1] = so[k] + nk;
            to[k + 1] = to[k] + mk;
        }
        const int NS = so[np], NT = to[np];
        CallCtx ctx;
        cudaStream_t s = ctx.stream();
        prof_begin(s);
        // ---- concatenated inputs ----
        DevBuf<double2> src(NS, s), trg(std::max(NT, 1), s);
        DevBuf<double2> chg(ifc ? NS : 0, s), dip(ifd ? NS : 0, s);
        DevBuf<double> dv((ifd && lap) ? 2 * (size_t)NS : 0, s);
        auto in = [&](void *dst, const double *user, size_t bytes) {
            if (bytes) FMM_CUDA(cudaMemcpyAsync(dst, user, bytes, cudaMemcpyDefault, s));
        };
        for (int k = 0; k < np; k++) {
            const size_t nk = b.ns[k], mk = to[k + 1] - to[k];
            in(src.get() + so[k], b.sources[k], nk * sizeof(double2));
            if (mk) in(trg.get() + to[k], b.targ[k], mk * sizeof(double2));
            if (ifc) in(chg.get() + so[k], b.charge[k], nk * sizeof(double2));
            if (ifd) in(dip.get() + so[k], b.dipstr[k], nk * sizeof(double2));
            if (ifd && lap) in(dv.get() + 2 * (size_t)so[k], b.dipvec[k], 2 * nk * sizeof(double));
        }
        prof_mark("h2d", s);
        // ---- every problem centred at the origin, one common root size ----
        DevBuf<int> dso(np + 1, s), dto(np + 1, s);
        FMM_CUDA(cudaMemcpyAsync(dso.get(), so.data(), (np + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
        FMM_CUDA(cudaMemcpyAsync(dto.get(), to.data(), (np + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
        DevBuf<double> bb(4 * (size_t)np, s);
        seg_bbox_kernel<<<np, 256, 0, s>>>(src.get(), dso.get(), trg.get(), dto.get(), bb.get());
        FMM_CHECK_LAUNCH();
        std::vector<double> hb(4 * (size_t)np);
        FMM_CUDA(cudaMemcpyAsync(hb.data(), bb.get(), hb.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        FMM_CUDA(cudaStreamSynchronize(s));
        std::vector<double2> cen(np);
        double R = 0.0;
        for (int k = 0; k < np; k++) {
            const double *q = &hb[4 * (size_t)k];
            cen[k] = make_double2((q[0] + q[1]) / 2, (q[2] + q[3]) / 2);
            R = std::max(R, std::max(q[1] - q[0], q[3] - q[2]));
        }
        if (!(R > 0.0)) R = 1.0;  // every problem a single point
        DevBuf<double2> dcen(np, s);
        FMM_CUDA(cudaMemcpyAsync(dcen.get(), cen.data(), np * sizeof(double2), cudaMemcpyHostToDevice, s));
        seg_shift_kernel<<<np, 256, 0, s>>>(src.get(), dso.get(), dcen.get());
        FMM_CHECK_LAUNCH();
        if (NT > 0) {
            seg_shift_kernel<<<np, 256, 0, s>>>(trg.get(), dto.get(), dcen.get());
            FMM_CHECK_LAUNCH();
        }
        // ---- the forest and the geometry ----
        LapGeometry G;
        G.lap = lap;
        G.nd = 1;
        G.ndc = lap ? 2 : 1;
        G.ns = NS;
        G.nt = NT;
        G.eps = b.eps;
        G.p = laplace_nterms(b.eps);
        G.mixed = b.precision == kPrecMixed || (b.precision == kPrecAuto && b.eps >= 0.5e-6);
        G.split = !G.mixed && b.precision == kPrecSplit;
        int ndiv = leaf_capacity(b.eps, NS, NT);
        if (G.mixed && lap) ndiv = mixed_leaf_capacity(G.p, ndiv);
        build_forest(src.get(), so, NT > 0 ? trg.get() : nullptr, to, ndiv, 0, kMaxLevels, R, s, G.T);
        compute_lists(G.T, s);
        prof_mark("lists", s);
        G.src_s.alloc(NS, s);
        G.trg_s.alloc(std::max(NT, 1), s);
        if (G.mixed) {
            G.src_hl.alloc(NS, s);
            G.trg_hl.alloc(std::max(NT, 1), s);
        }
        auto gather = [&](int n, const int *perm, const double2 *inp, double2 *o, float4 *hl) {
            for_each(n, s, [=] __device__(int64_t k) {
                const double2 v = inp[perm[k]];
                o[k] = v;
                if (hl) hl[k] = split_pos(v);
            });
        };
        gather(NS, G.T.isrc.get(), src.get(), G.src_s.get(), G.src_hl.get());
        if (NT > 0) gather(NT, G.T.itarg.get(), trg.get(), G.trg_s.get(), G.trg_hl.get());
        G.thresh = R * std::ldexp(1.0, -51);
        // ---- one evaluation of the whole forest into concatenated outputs ----
        const size_t gc = lap ? 2 : 1, hc = lap ? 3 : 1;
        const int sp = b.ifpgh, tp = NT > 0 ? b.ifpghtarg : 0;
        DevBuf<double2> opot(sp >= 1 ? NS : 0, s), ograd(sp >= 2 ? gc * NS : 0, s),
            ohess(sp >= 3 ? hc * NS : 0, s), tpot(tp >= 1 ? NT : 0, s),
            tgrad(tp >= 2 ? gc * NT : 0, s), thess(tp >= 3 ? hc * NT : 0, s);
        FmmCall c;
        c.kernel = b.kernel;
        c.nd = 1;
        c.eps = b.eps;
        c.ns = NS;
        c.nt = NT;
        c.ifcharge = ifc;
        c.ifdipole = ifd;
        c.charge = reinterpret_cast<const double *>(chg.get());
        c.dipstr = reinterpret_cast<const double *>(dip.get());
        c.dipvec = dv.get();
        c.ifpgh = sp;
        c.ifpghtarg = tp;
        c.pot = reinterpret_cast<double *>(opot.get());
        c.grad = reinterpret_cast<double *>(ograd.get());
        c.hess = reinterpret_cast<double *>(ohess.get());
        c.pottarg = reinterpret_cast<double *>(tpot.get());
        c.gradtarg = reinterpret_cast<double *>(tgrad.get());
        c.hesstarg = reinterpret_cast<double *>(thess.get());
        laplace_evaluate(c, G, true, s);
        // ---- back to each problem's arrays ----
        auto outk = [&](double *user, const DevBuf<double2> &d, size_t comps, size_t off, size_t n) {
            if (user && n)
                FMM_CUDA(cudaMemcpyAsync(user, d.get() + comps * off, comps * n * sizeof(double2),
                                         cudaMemcpyDefault, s));
        };
        for (int k = 0; k < np; k++) {
            const size_t nk = b.ns[k], mk = to[k + 1] - to[k];
            if (sp >= 1) outk(b.pot[k], opot, 1, so[k], nk);
            if (sp >= 2) outk(b.grad[k], ograd, gc, so[k], nk);
            if (sp >= 3) outk(b.hess[k], ohess, hc, so[k], nk);
            if (tp >= 1) outk(b.pottarg[k], tpot, 1, to[k], mk);
            if (tp >= 2) outk(b.gradtarg[k], tgrad, gc, to[k], mk);
            if (tp >= 3) outk(b.hesstarg[k], thess, hc, to[k], mk);
        }
        FMM_CUDA(cudaStreamSynchronize(s));
        prof_mark("scatter_d2h", s);
        prof_end(s);
    });
}

int run_fmm(const FmmCall &c) {
    return guarded([&] {
        if (c.ns < 1) throw FmmError(4, "ns must be at least 1");
        if (c.nt < 0) throw FmmError(4, "nt must be non-negative");
        if (c.nd < 1) throw FmmError(4, "nd must be at least 1");
        if (!c.ifcharge && !c.ifdipole)
            throw FmmError(4, "at least one of ifcharge / ifdipole must be 1");
        CallCtx ctx;
        switch (c.kernel) {
            case kLaplace:
            case kCauchy:
            case kReal:
                run_laplace_family(c, ctx);
                break;
            case kHelmholtz:
                run_helmholtz(c, ctx);
                break;
            default:
                throw FmmError(4, "unknown kernel");
        }
    });
}

}  // namespace fmm2d
