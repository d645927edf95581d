"""Mixed-precision mode (FP32 series and pair arithmetic, FP64 geometry and
output accumulation): for eps >= 1e-6 every result stays within the
requested eps of the FP64 direct sum and of the reference FMM at the same
eps (relative l2 over sampled points)."""
import numpy as np
import pytest

import pointsets as ps
import refimpl
import wrappers as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mlib():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    L.fmm2d_b200_set_precision(2)
    yield L
    L.fmm2d_b200_set_precision(0)


def inputs(ns, nt, seed, dist):
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


def direct(src, q, d, v, pts, m, pgh):
    ns = src.shape[1]
    pot = np.zeros(m, complex)
    grad = np.zeros((m, 2), complex)
    hess = np.zeros((m, 3), complex)
    s = np.ascontiguousarray(src.T)
    refimpl.orc().oracle_l2d_direct(
        ns, W._p(s), 1, W._p(q), 1, W._p(d), W._p(np.ascontiguousarray(v.T)), 0, m,
        W._p(np.ascontiguousarray(pts[:, :m].T)), pgh, W._p(pot), W._p(grad),
        W._p(hess), 1e-300)
    return pot, grad, hess


@pytest.mark.parametrize("eps", [1e-3, 1e-6])
@pytest.mark.parametrize("dist", ["uniform", "blobs", "starfish"])
def test_mixed_within_eps(mlib, eps, dist):
    src, trg, q, d, v = inputs(40000, 20000, 7, dist)
    got, ier = W.call(mlib, "l", "st_cd_h", eps, src, q, d, v, trg)
    assert ier == 0
    m = 400
    dp, dg, dh = direct(src, q, d, v, trg, m, 3)
    assert W.rel_err(got["pottarg"][:m], dp) <= eps
    assert W.rel_err(got["gradtarg"][:m], dg) <= eps
    assert W.rel_err(got["hesstarg"][:m], dh) <= eps
    sp, sg, _ = direct(src, q, d, v, src, m, 2)
    assert W.rel_err(got["pot"][:m], sp) <= eps
    assert W.rel_err(got["grad"][:m], sg) <= eps
    want, ier = W.call(refimpl.ref(), "l", "st_cd_h", eps, src, q, d, v, trg)
    for k in ("pot", "grad", "pottarg", "gradtarg"):
        assert W.rel_err(got[k], want[k]) <= eps, k


@pytest.mark.parametrize("variant", ["s_c_p", "t_d_g", "st_cd_g", "s_c_h", "t_cd_h", "st_d_h"])
@pytest.mark.parametrize("family", ["l", "c"])
def test_mixed_variants_match_reference(mlib, family, variant):
    src, trg, q, d, v = inputs(20000, 5000, 9, "blobs")
    got, ier = W.call(mlib, family, variant, 1e-6, src, q, d, v, trg)
    want, ier2 = W.call(refimpl.ref(), family, variant, 1e-6, src, q, d, v, trg)
    assert ier == 0 and ier2 == 0
    for k in want:
        assert W.rel_err(got[k], want[k]) <= 1e-6, k


@pytest.mark.parametrize("fam,nd", [("c", 3), ("l", 2), ("c", 1)])
@pytest.mark.parametrize("m2l", ["tc", "simt"])
def test_mixed_multichannel_matches_fp64(mlib, fam, nd, m2l, monkeypatch):
    """Guru drivers with several densities (odd and even channel counts) in
    the mixed mode, both M2L paths, against the all-FP64 mode."""
    import fmm2d_c_translation_b200 as fm
    monkeypatch.setenv("FMM2D_B200_M2L", m2l)
    rng = np.random.default_rng(13)
    ns, nt = 40000, 9000
    src = rng.random((2, ns))
    trg = rng.random((2, nt))
    shp = (nd, ns) if nd > 1 else (ns,)
    q = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    d = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    kw = dict(eps=1e-6, sources=src, charges=q, dipstr=d, targets=trg, pg=2, pgt=2, nd=nd)
    f = fm.cfmm2d if fam == "c" else fm.lfmm2d
    if fam == "l":
        kw["dipvec"] = rng.standard_normal((nd, 2, ns) if nd > 1 else (2, ns))
    mixed = f(**kw)
    mlib.fmm2d_b200_set_precision(1)
    try:
        ref = f(**dict(kw, eps=1e-12))
    finally:
        mlib.fmm2d_b200_set_precision(2)
    assert W.rel_err(mixed.gradtarg, ref.gradtarg) < 1e-6
    assert W.rel_err(mixed.grad, ref.grad) < 1e-6
    if fam == "l":  # Cauchy potentials carry the branch term of log z
        assert W.rel_err(mixed.pottarg, ref.pottarg) < 1e-6


@pytest.mark.parametrize("p2p", ["flat", "group"])
@pytest.mark.parametrize("far", ["leaf", "point"])
def test_mixed_pass_forms(mlib, monkeypatch, p2p, far):
    """Both near-field forms and both far-field forms of the mixed mode stay
    within eps of the reference FMM (starfish tree: list 3 and list 4)."""
    monkeypatch.setenv("FMM2D_B200_P2P", p2p)
    monkeypatch.setenv("FMM2D_B200_FAR", far)
    src, trg, q, d, v = inputs(30000, 10000, 17, "starfish")
    got, ier = W.call(mlib, "l", "st_cd_h", 1e-6, src, q, d, v, trg)
    want, ier2 = W.call(refimpl.ref(), "l", "st_cd_h", 1e-6, src, q, d, v, trg)
    assert ier == 0 and ier2 == 0
    for k in want:
        assert W.rel_err(got[k], want[k]) <= 1e-6, k


@pytest.mark.parametrize("m2l", ["window", "tile", "simt"])
def test_mixed_charge_gradient_at_sources(mlib, monkeypatch, m2l):
    """Charges only, gradient at the sources (the far field carries a large
    share of it): every M2L form stays within eps of the direct sum at
    eps 1e-6.  The tensor-core forms pass because they recompute the
    leading local coefficients in FP32 from order 17 on."""
    if m2l != "window":
        monkeypatch.setenv("FMM2D_B200_M2L", m2l)
    rng = np.random.default_rng(101)
    ns = 100000
    src = rng.random((2, ns))
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    got, ier = W.call(mlib, "l", "s_c_g", 1e-6, src, q, None, None)
    assert ier == 0
    m = 300
    d = np.zeros(ns, complex)
    v = np.zeros((2, ns))
    pot = np.zeros(m, complex)
    grad = np.zeros((m, 2), complex)
    s = np.ascontiguousarray(src.T)
    refimpl.orc().oracle_l2d_direct(
        ns, W._p(s), 1, W._p(q), 0, W._p(d), W._p(np.ascontiguousarray(v.T)), 0, m,
        W._p(s), 2, W._p(pot), W._p(grad), None, 1e-150)
    assert W.rel_err(got["pot"][:m], pot) <= 1e-6
    assert W.rel_err(got["grad"][:m], grad) <= 1e-6
