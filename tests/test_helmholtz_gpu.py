"""Helmholtz parity on the GPU (hfmm2d_*, src/helmholtz/hfmm2dwrap.f):

* all 27 flag wrappers against the reference build on the same inputs, at
  the reference test's sizes (ns = 1000, nt = 1001, eps = 0.51e-8,
  test/helmholtz/test_hfmm2d.f:19-51) for zk = 10 and zk = 0.5 + 0.1i;
* the same wrappers against the direct sum at the first 20 points with the
  reference test's own criterion (relative l2 error < eps);
* zk = 500 (test_hfmm2d_hf.f:50), where the reference switches its coarse
  levels to the diagonal (FFT) translations and this library keeps the
  coefficient-space Graf translations (the same truncated operators);
* the guru driver with nd = 2, the ndiv driver, the bind(c) entry, and the
  GPU direct sum against the reference's h2d_direct kernels;
* the tiled M2L (both of its forms) against the per-box M2L kernel.
"""
import ctypes

import numpy as np
import pytest

import refimpl
import wrappers as W

pytestmark = pytest.mark.gpu
_P = ctypes.c_void_p
EPS = 0.51e-8
ZKS = [10.0 + 0j, 0.5 + 0.1j]


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def inputs(ns=1000, nt=1001, seed=7):
    rng = np.random.default_rng(seed)
    src = rng.random((2, ns))
    trg = rng.random((2, nt))
    q = rng.random(ns) + 1j * rng.random(ns)
    d = rng.random(ns) + 1j * rng.random(ns)
    v = rng.random((2, ns))
    return src, trg, q, d, v


@pytest.fixture(scope="module")
def glib():
    """The library in its all-FP64 mode: these are parity tests against the
    reference's FP64 FMM (the mixed mode is tested in
    test_helmholtz_mixed_gpu.py)."""
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    L.fmm2d_b200_set_precision(1)
    yield L
    L.fmm2d_b200_set_precision(0)


def h_direct(lib, zk, src, q, d, v, trg, pgh, ifc, ifd, nd=1):
    """GPU direct sum at trg (2, n): pot (n,), grad (n, 2), hess (n, 3)."""
    n = trg.shape[1]
    pot = np.zeros(n * nd, np.complex128)
    grad = np.zeros(n * nd * 2, np.complex128)
    hess = np.zeros(n * nd * 3, np.complex128)
    zka = np.array([zk.real, zk.imag])
    srcf = np.asfortranarray(src)
    trgf = np.asfortranarray(trg)
    qq = np.ascontiguousarray(q, np.complex128) if ifc else None
    dd = np.ascontiguousarray(d, np.complex128) if ifd else None
    vv = np.asfortranarray(v, np.float64) if ifd else None
    thresh = abs(zk) * 2.0 ** -51
    ier = lib.fmm2d_b200_h2d_direct(
        ctypes.c_int(nd), _p(zka), ctypes.c_int(src.shape[1]), _p(srcf), ctypes.c_int(ifc),
        _p(qq), ctypes.c_int(ifd), _p(dd), _p(vv), ctypes.c_int(n), _p(trgf),
        ctypes.c_int(pgh), _p(pot), _p(grad), _p(hess), ctypes.c_double(thresh))
    assert ier == 0
    return pot, grad.reshape(n, 2), hess.reshape(n, 3)


def _check_direct(lib, zk, variant, out, src, trg, q, d, v, ntest=20):
    st, cd, p = variant.split("_")
    pgh = {"p": 1, "g": 2, "h": 3}[p]
    ifc, ifd = int("c" in cd), int("d" in cd)
    for where, pts in (("", src), ("targ", trg)):
        if f"pot{where}" not in out:
            continue
        sub = pts[:, :ntest]
        pot, grad, hess = h_direct(lib, zk, src, q, d, v, sub, pgh, ifc, ifd)
        num = np.linalg.norm(out[f"pot{where}"][:ntest] - pot) ** 2
        den = np.linalg.norm(pot) ** 2
        if pgh >= 2:
            num += np.linalg.norm(out[f"grad{where}"][:ntest] - grad) ** 2
            den += np.linalg.norm(grad) ** 2
        if pgh >= 3:
            num += np.linalg.norm(out[f"hess{where}"][:ntest] - hess) ** 2
            den += np.linalg.norm(hess) ** 2
        err = np.sqrt(num / den)
        assert err < EPS, (variant, where, err)


@pytest.mark.parametrize("zk", ZKS, ids=["zk10", "zk0.5+0.1i"])
@pytest.mark.parametrize("variant", W.VARIANTS)
def test_hfmm2d_wrappers(glib, zk, variant):
    src, trg, q, d, v = inputs()
    out, ier = W.call(glib, "h", variant, EPS, src, q, d, v, trg, zk=zk)
    assert ier == 0
    _check_direct(glib, zk, variant, out, src, trg, q, d, v)
    if refimpl.have_ref():
        ro, rier = W.call(refimpl.ref(), "h", variant, EPS, src, q, d, v, trg, zk=zk)
        assert rier == 0
        for k in out:
            assert W.rel_err(out[k], ro[k]) < 1e-10, (variant, k, W.rel_err(out[k], ro[k]))


@pytest.mark.parametrize("variant", ["st_cd_h", "s_c_p", "t_d_g", "st_c_g"])
def test_hfmm2d_high_frequency(glib, variant):
    zk = 500.0 + 0j
    src, trg, q, d, v = inputs()
    out, ier = W.call(glib, "h", variant, EPS, src, q, d, v, trg, zk=zk)
    assert ier == 0
    _check_direct(glib, zk, variant, out, src, trg, q, d, v)
    if refimpl.have_ref():
        ro, _ = W.call(refimpl.ref(), "h", variant, EPS, src, q, d, v, trg, zk=zk)
        for k in out:
            assert W.rel_err(out[k], ro[k]) < 1e-8, (variant, k, W.rel_err(out[k], ro[k]))


@pytest.mark.parametrize("eps", [1e-3, 1e-6, 1e-12])
@pytest.mark.parametrize("zk", [30.0 + 0j, 2.0 + 3.0j, 1e-2 + 0j])
def test_hfmm2d_eps_and_zk(glib, eps, zk):
    src, trg, q, d, v = inputs(ns=3000, nt=500, seed=11)
    out, ier = W.call(glib, "h", "st_cd_g", eps, src, q, d, v, trg, zk=zk)
    assert ier == 0
    if refimpl.have_ref():
        ro, _ = W.call(refimpl.ref(), "h", "st_cd_g", eps, src, q, d, v, trg, zk=zk)
        for k in out:
            assert W.rel_err(out[k], ro[k]) < max(1e-10, 10 * eps * 1e-2), (k, W.rel_err(out[k], ro[k]))
    pot, grad, _ = h_direct(glib, zk, src, q, d, v, trg[:, :50], 2, 1, 1)
    assert W.rel_err(out["pottarg"][:50], pot) < 10 * eps
    assert W.rel_err(out["gradtarg"][:50], grad) < 100 * eps


@pytest.mark.parametrize("zk,eps", [(200.0 + 0j, 1e-6), (30.0 + 0j, 1e-9), (2.0 + 3.0j, 1e-6),
                                    (1e-3 + 0j, 1e-12)],
                         ids=["zk200", "zk30", "zk2+3i", "zk1e-3-weighted"])
def test_m2l_tile_form_matches_box_form(glib, monkeypatch, zk, eps):
    """The M2L over tiles of boxes that share their child position (the
    default; scaled Toeplitz sums, or per-term weights where the scaling
    would leave the FP64 range, as for zk = 1e-3 at eps 1e-12) against the
    per-box kernel that follows h2dmploc term by term."""
    src, trg, q, d, v = inputs(ns=20000, nt=3000, seed=5)
    out, ier = W.call(glib, "h", "st_cd_g", eps, src, q, d, v, trg, zk=zk)
    assert ier == 0
    monkeypatch.setenv("FMM2D_B200_HELM_M2L", "box")
    ob, ierb = W.call(glib, "h", "st_cd_g", eps, src, q, d, v, trg, zk=zk)
    assert ierb == 0
    for k in out:
        assert W.rel_err(out[k], ob[k]) < 1e-11, (k, W.rel_err(out[k], ob[k]))


def _guru(lib, fn_name, nd, zk, src, q, d, v, trg, ndiv=None):
    ns, nt = src.shape[1], trg.shape[1]
    pot = np.zeros((ns, nd), np.complex128)
    grad = np.zeros((ns, 2, nd), np.complex128)
    hess = np.zeros((ns, 3, nd), np.complex128)
    pt = np.zeros((nt, nd), np.complex128)
    gt = np.zeros((nt, 2, nd), np.complex128)
    ht = np.zeros((nt, 3, nd), np.complex128)
    zka = np.array([zk], np.complex128)
    ier = ctypes.c_int(-1)
    iper = ctypes.c_int(0)
    ci = lambda x: ctypes.byref(ctypes.c_int(x))  # noqa: E731
    args = [ci(nd), ctypes.byref(ctypes.c_double(1e-10)), _p(zka), ci(ns),
            _p(np.asfortranarray(src)), ci(1), _p(q), ci(1), _p(d), _p(v),
            ctypes.byref(iper), ci(3), _p(pot), _p(grad), _p(hess), ci(nt),
            _p(np.asfortranarray(trg)), ci(3), _p(pt), _p(gt), _p(ht)]
    if ndiv is not None:
        timeinfo = np.zeros(8)
        args += [ci(ndiv), ci(0), ci(1), _p(timeinfo)]
    args.append(ctypes.byref(ier))
    getattr(lib, fn_name)(*args)
    return ier.value, [pot, grad, hess, pt, gt, ht]


@pytest.mark.parametrize("fn", ["hfmm2d_", "hfmm2d_ndiv_"])
def test_hfmm2d_guru_nd2(glib, fn):
    if not refimpl.have_ref():
        pytest.skip("reference build absent")
    rng = np.random.default_rng(3)
    ns, nt, nd = 800, 300, 2
    src = rng.random((2, ns))
    trg = rng.random((2, nt))
    q = np.ascontiguousarray(rng.standard_normal((ns, nd)) + 1j * rng.standard_normal((ns, nd)))
    d = np.ascontiguousarray(rng.standard_normal((ns, nd)) + 1j * rng.standard_normal((ns, nd)))
    v = np.ascontiguousarray(rng.standard_normal((ns, 2, nd)))
    zk = 7.0 + 0.3j
    ndiv = 12 if fn == "hfmm2d_ndiv_" else None
    ier, out = _guru(glib, fn, nd, zk, src, q, d, v, trg, ndiv)
    rier, ro = _guru(refimpl.ref(), fn, nd, zk, src, q, d, v, trg, ndiv)
    assert ier == 0 and rier == 0
    for a, b in zip(out, ro):
        assert W.rel_err(a, b) < 1e-10


def test_bind_c_entry(glib):
    src, trg, q, d, v = inputs(ns=500)
    zk = 10.0 + 0j
    pot = np.zeros(500, np.complex128)
    ier = ctypes.c_int64(-1)

    class Z(ctypes.Structure):
        _fields_ = [("re", ctypes.c_double), ("im", ctypes.c_double)]

    f = glib.hfmm2d_s_c_p
    f.argtypes = [ctypes.c_double, Z, ctypes.c_int64, _P, _P, _P, ctypes.POINTER(ctypes.c_int64)]
    f(EPS, Z(zk.real, zk.imag), 500, _p(np.asfortranarray(src)), _p(q), _p(pot), ctypes.byref(ier))
    assert ier.value == 0
    out, _ = W.call(glib, "h", "s_c_p", EPS, src, q, d, v, trg, zk=zk)
    np.testing.assert_allclose(pot, out["pot"], rtol=0, atol=0)


@pytest.mark.parametrize("zk", [10.0 + 0j, 0.5 + 0.1j, 80 + 0j])
@pytest.mark.parametrize("ifc,ifd", [(1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("pgh", [1, 2, 3])
def test_h2d_direct_vs_reference(glib, zk, ifc, ifd, pgh):
    if not refimpl.have_ref():
        pytest.skip("reference build absent")
    src, trg, q, d, v = inputs(ns=300, nt=200, seed=5)
    trg[:, :3] = src[:, :3]  # coincident points exercise the threshold
    pot, grad, hess = h_direct(glib, zk, src, q, d, v, trg, pgh, ifc, ifd)
    R = refimpl.ref()
    nt = trg.shape[1]
    rp = np.zeros(nt, np.complex128)
    rg = np.zeros((nt, 2), np.complex128)
    rh = np.zeros((nt, 3), np.complex128)
    kind = {(1, 0): "c", (0, 1): "d", (1, 1): "cd"}[(ifc, ifd)] + "pgh"[pgh - 1]
    zka = np.array([zk], np.complex128)
    thresh = ctypes.byref(ctypes.c_double(abs(zk) * 2.0 ** -51))
    ci = lambda x: ctypes.byref(ctypes.c_int(x))  # noqa: E731
    args = [ci(1), _p(zka), _p(np.asfortranarray(src)), ci(src.shape[1])]
    if ifc:
        args.append(_p(q))
    if ifd:
        args += [_p(d), _p(np.asfortranarray(v))]
    args += [_p(np.asfortranarray(trg)), ci(nt), _p(rp)]
    if pgh >= 2:
        args.append(_p(rg))
    if pgh >= 3:
        args.append(_p(rh))
    args.append(thresh)
    getattr(R, f"h2d_direct{kind}_")(*args)
    assert W.rel_err(pot, rp) < 1e-13
    if pgh >= 2:
        assert W.rel_err(grad, rg) < 1e-13
    if pgh >= 3:
        assert W.rel_err(hess, rh) < 1e-13


def test_hfmm2d_zk200_against_reference(glib):
    """The zk = 200, eps = 1e-6 case (hfmm2d_s_cd_p, uniform points, complex
    charges and dipoles N(0,1), unit dipole vectors) at 2e5 sources against
    the reference's C translation on the same inputs.  The tree is the
    reference's (bit-exact), so the expansion orders -- up to p = 94 on
    level 1 here -- are the same and both sides differ only by round-off
    (all-FP64 mode)."""
    if not refimpl.have_ref():
        pytest.skip("reference build absent")
    rng = np.random.default_rng(200)
    ns = 200000
    src = rng.random((2, ns))
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    th = rng.uniform(0, 2 * np.pi, ns)
    v = np.stack([np.cos(th), np.sin(th)])
    zk = 200.0 + 0j
    out, ier = W.call(glib, "h", "s_cd_p", 1e-6, src, q, d, v, None, zk=zk)
    assert ier == 0
    ro, rier = W.call(refimpl.ref(), "h", "s_cd_p", 1e-6, src, q, d, v, None, zk=zk)
    assert rier == 0
    assert W.rel_err(out["pot"], ro["pot"]) < 1e-10, W.rel_err(out["pot"], ro["pot"])
    # and both against the direct sum at 200 sources, to the requested eps
    pot, _, _ = h_direct(glib, zk, src, q, d, v, src[:, :200], 1, 1, 1)
    assert W.rel_err(out["pot"][:200], pot) < 1e-6


@pytest.mark.parametrize("zk", [1500.0 + 0j, 900.0 + 0j])
def test_high_frequency_diagonal_m2l(glib, monkeypatch, zk):
    """Levels of more than 16 wavelengths per box take the M2L in the
    diagonal (signature) form (helm_hf.cu); it applies the same truncated
    operator as the coefficient-space shift, so the two agree to round-off,
    and both stay within eps of the direct sum."""
    src, trg, q, d, v = inputs(ns=30000, nt=4000, seed=15)
    eps = 1e-6
    out, ier = W.call(glib, "h", "st_cd_g", eps, src, q, d, v, trg, zk=zk)
    assert ier == 0
    monkeypatch.setenv("FMM2D_B200_HELM_HF", "0")
    oc, ier = W.call(glib, "h", "st_cd_g", eps, src, q, d, v, trg, zk=zk)
    assert ier == 0
    for k in out:
        assert W.rel_err(out[k], oc[k]) < 1e-11, (k, W.rel_err(out[k], oc[k]))
    pot, grad, _ = h_direct(glib, zk, src, q, d, v, trg[:, :100], 2, 1, 1)
    assert W.rel_err(out["pottarg"][:100], pot) < eps
    assert W.rel_err(out["gradtarg"][:100], grad) < eps


@pytest.mark.parametrize("zk", [200.0 + 0j, 2.0 + 3.0j])
@pytest.mark.parametrize("variant", ["st_cd_h", "s_c_p", "t_d_g"])
def test_p2p_forms_agree(glib, monkeypatch, zk, variant):
    """The near field with one warp per leaf (default for nd = 1) against one
    thread per point: the same pairs summed in another order."""
    src, trg, q, d, v = inputs(ns=20000, nt=5000, seed=23)
    out, ier = W.call(glib, "h", variant, 1e-9, src, q, d, v, trg, zk=zk)
    assert ier == 0
    monkeypatch.setenv("FMM2D_B200_HELM_P2P", "point")
    op, ier = W.call(glib, "h", variant, 1e-9, src, q, d, v, trg, zk=zk)
    assert ier == 0
    for k in out:
        assert W.rel_err(out[k], op[k]) < 1e-13, (k, W.rel_err(out[k], op[k]))
