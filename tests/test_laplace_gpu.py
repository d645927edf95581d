"""GPU Laplace (lfmm2d_*) and Cauchy (cfmm2d_*) evaluations against the
reference's own C translation on the same inputs, through the C ABI.

In all-FP64 mode the GPU runs the reference's algorithm on the
bit-identical tree with the same expansion order, so the two differ only
by floating-point rounding: relative l2 difference <= 1e-11 per output.
"""
import ctypes

import numpy as np
import pytest

import pointsets as ps
import refimpl
import wrappers as W

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-11


@pytest.fixture(scope="module")
def glib():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    L.fmm2d_b200_set_precision(1)
    yield L
    L.fmm2d_b200_set_precision(0)


def inputs(ns, nt, seed, dist="uniform"):
    rng = np.random.default_rng(seed)
    if dist == "uniform":
        src, trg = ps.uniform(ns, seed), ps.uniform(nt, seed + 1)
    elif dist == "blobs":
        src, trg = ps.blobs(ns, seed), ps.blobs(nt, seed + 1)
    else:
        src = ps.starfish(ns, seed)[0]
        trg = ps.near_curve_targets(nt, seed + 1)
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    th = rng.uniform(0, 2 * np.pi, ns)
    v = np.stack([np.cos(th), np.sin(th)])
    return src, trg, q, d, v


def compare(glib, family, variant, eps, src, trg, q, d, v, tol):
    got, ierg = W.call(glib, family, variant, eps, src, q, d, v, trg)
    want, ierr = W.call(refimpl.ref(), family, variant, eps, src, q, d, v, trg)
    assert ierg == 0 and ierr == 0
    assert set(got) == set(want)
    for k in want:
        e = W.rel_err(got[k], want[k])
        assert e <= tol, f"{family}fmm2d_{variant} {k}: rel err {e:.3e}"


@pytest.mark.parametrize("variant", W.VARIANTS)
@pytest.mark.parametrize("family", ["l", "c"])
def test_wrappers_small(glib, family, variant):
    src, trg, q, d, v = inputs(200, 100, 11)
    compare(glib, family, variant, 1e-6, src, trg, q, d, v, TOL_FP64)


@pytest.mark.parametrize("eps", [1e-3, 1e-6, 1e-9, 1e-12])
@pytest.mark.parametrize("dist", ["uniform", "blobs", "starfish"])
def test_lfmm_st_cd_h_sizes(glib, eps, dist):
    src, trg, q, d, v = inputs(20000, 8000, 21, dist)
    compare(glib, "l", "st_cd_h", eps, src, trg, q, d, v, TOL_FP64)


@pytest.mark.parametrize("variant", ["st_cd_h", "s_c_g", "t_d_p"])
def test_cfmm_medium(glib, variant):
    src, trg, q, d, v = inputs(30000, 12000, 31, "blobs")
    compare(glib, "c", variant, 1e-9, src, trg, q, d, v, TOL_FP64)


def test_guru_nd2(glib):
    """lfmm2d_ with nd = 2 densities through the guru driver."""
    ns, nt, nd = 3000, 1000, 2
    rng = np.random.default_rng(5)
    src, trg = ps.uniform(ns, 5), ps.uniform(nt, 6)
    q = np.asfortranarray(rng.standard_normal((nd, ns)) + 1j * rng.standard_normal((nd, ns)))
    d = np.asfortranarray(rng.standard_normal((nd, ns)) + 1j * rng.standard_normal((nd, ns)))
    v = np.asfortranarray(rng.standard_normal((nd, 2, ns)))
    res = []
    for L in (glib, refimpl.ref()):
        pot = np.zeros((nd, ns), np.complex128, order="F")
        grad = np.zeros((nd, 2, ns), np.complex128, order="F")
        hess = np.zeros((nd, 3, ns), np.complex128, order="F")
        pt = np.zeros((nd, nt), np.complex128, order="F")
        gt = np.zeros((nd, 2, nt), np.complex128, order="F")
        ht = np.zeros((nd, 3, nt), np.complex128, order="F")
        ier = ctypes.c_int(-1)
        I = lambda x: ctypes.byref(ctypes.c_int(x))
        L.lfmm2d_(I(nd), ctypes.byref(ctypes.c_double(1e-9)), I(ns), W._p(src),
                  I(1), W._p(q), I(1), W._p(d), W._p(v), I(0), I(3),
                  W._p(pot), W._p(grad), W._p(hess), I(nt), W._p(trg), I(3),
                  W._p(pt), W._p(gt), W._p(ht), ctypes.byref(ier))
        assert ier.value == 0
        res.append((pot, grad, hess, pt, gt, ht))
    for a, b in zip(*res):
        assert W.rel_err(a, b) <= TOL_FP64


def test_against_direct_sum(glib):
    """Accuracy of the GPU FMM against the FP64 direct-sum oracle."""
    ns = 20000
    src, trg, q, d, v = inputs(ns, 1, 41, "blobs")
    for eps in (1e-3, 1e-6, 1e-9, 1e-12):
        got, ier = W.call(glib, "l", "s_cd_g", eps, src, q, d, v)
        assert ier == 0
        m = 300
        pot = np.zeros(m, np.complex128)
        grad = np.zeros((m, 2), np.complex128)
        s = np.ascontiguousarray(src.T)
        refimpl.orc().oracle_l2d_direct(
            ns, W._p(s), 1, W._p(q), 1, W._p(d), W._p(np.ascontiguousarray(v.T)),
            0, m, W._p(s), 2, W._p(pot), W._p(grad), None, 1e-300)
        assert W.rel_err(got["pot"][:m], pot) < 10 * eps
        assert W.rel_err(got["grad"][:m], grad) < 100 * eps


@pytest.mark.parametrize("p2p", ["flat", "group"])
@pytest.mark.parametrize("far", ["leaf", "point"])
@pytest.mark.parametrize("variant", ["st_cd_h", "st_c_g", "t_d_p"])
def test_pass_forms_agree(glib, monkeypatch, p2p, far, variant):
    """Every form of the evaluation passes (near field with flattened or
    grouped lanes; far field per leaf or per point) gives the reference's
    values, on a tree with list-3 and list-4 boxes."""
    monkeypatch.setenv("FMM2D_B200_P2P", p2p)
    monkeypatch.setenv("FMM2D_B200_FAR", far)
    src, trg, q, d, v = inputs(20000, 8000, 51, "starfish")
    compare(glib, "l", variant, 1e-9, src, trg, q, d, v, TOL_FP64)
