"""The real-valued Laplace FMM (rfmm2d, src/laplace/rfmm2d.f:27) and the
vectorised wrappers {l,c,h,r}fmm2d_*_vec (src/laplace/lfmm2dwrap_vec.f,
cfmm2dwrap_vec.f, rfmm2dwrap_vec.f, src/helmholtz/hfmm2dwrap_vec.f) against
the reference's own C translation on the same inputs:

* all 27 rfmm2d wrappers against the reference's rfmm2d_ndiv_
  (c_translation/src/rfmm2d_ndiv.c:51) at the reference's leaf-capacity
  rule, at 1e-11 relative (all-FP64 mode, eps 1e-9);
* rfmm2d_ndiv_ with a caller ndiv, idivflag 0/1/2 and ifnear 0/1;
* the _vec wrappers of every family with nd = 3 against the reference's
  guru drivers (lfmm2d_, cfmm2d_, hfmm2d_, rfmm2d_ndiv_) with the flags the
  wrapper sets;
* rfmm2d in the mixed mode within eps of the FP64 direct sum.
"""
import ctypes

import numpy as np
import pytest

import refimpl
import wrappers as W

pytestmark = pytest.mark.gpu
_P = ctypes.c_void_p
EPS = 1e-9
TOL = 1e-11


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def _ci(x):
    return ctypes.byref(ctypes.c_int(x))


@pytest.fixture(scope="module")
def glib():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    L.fmm2d_b200_set_precision(1)
    yield L
    L.fmm2d_b200_set_precision(0)


def _inputs(nd, ns, nt, seed, real):
    rng = np.random.default_rng(seed)
    src, trg = rng.random((2, ns)), rng.random((2, nt))
    if real:
        q, d = rng.standard_normal((nd, ns)), rng.standard_normal((nd, ns))
    else:
        q = rng.standard_normal((nd, ns)) + 1j * rng.standard_normal((nd, ns))
        d = rng.standard_normal((nd, ns)) + 1j * rng.standard_normal((nd, ns))
    v = rng.standard_normal((nd, 2, ns))
    return src, trg, q, d, v


def ref_guru(family, nd, eps, src, q, d, v, trg, ifc, ifd, pg, pgt, zk=None, ndiv=None,
             idivflag=0, ifnear=1, lib=None):
    """The guru driver of `family` (reference build unless lib is given);
    outputs as (n, [comps,] nd) arrays like wrappers.call_nd."""
    R = lib if lib is not None else refimpl.ref()
    ns, nt = src.shape[1], trg.shape[1]
    dt = np.float64 if family == "r" else np.complex128
    gc, hc = (1, 1) if family == "c" else (2, 3)
    z = lambda n, c: np.zeros((n, c, nd) if c > 1 else (n, nd), dt)  # noqa: E731
    outs = [z(ns, 1), z(ns, gc), z(ns, hc), z(nt, 1), z(nt, gc), z(nt, hc)]
    qq = np.ascontiguousarray(np.asarray(q, dt).reshape(nd, ns).T)
    dd = np.ascontiguousarray(np.asarray(d, dt).reshape(nd, ns).T)
    vv = np.ascontiguousarray(np.transpose(np.asarray(v).reshape(nd, 2, ns), (2, 1, 0)))
    ier = ctypes.c_int(-1)
    iper = ctypes.c_int(0)
    args = [_ci(nd), ctypes.byref(ctypes.c_double(eps))]
    if family == "h":
        zka = np.array([zk], np.complex128)
        args.append(_p(zka))
    args += [_ci(ns), _p(np.asfortranarray(src)), _ci(ifc), _p(qq), _ci(ifd), _p(dd)]
    if family != "c":
        args.append(_p(vv))
    args += [ctypes.byref(iper), _ci(pg), _p(outs[0]), _p(outs[1]), _p(outs[2]), _ci(nt),
             _p(np.asfortranarray(trg)), _ci(pgt), _p(outs[3]), _p(outs[4]), _p(outs[5])]
    name = f"{family}fmm2d_"
    if family == "r" or ndiv is not None:
        if ndiv is None:
            import fmm2d_c_translation_b200 as fm
            ndiv = fm.lib().fmm2d_b200_leaf_capacity(ctypes.c_double(eps), ns, nt)
        timeinfo = np.zeros(8)
        args += [_ci(ndiv), _ci(idivflag), _ci(ifnear), _p(timeinfo)]
        name = f"{family}fmm2d_ndiv_"
    args.append(ctypes.byref(ier))
    getattr(R, name)(*args)
    keys = ["pot", "grad", "hess", "pottarg", "gradtarg", "hesstarg"]
    res = {}
    for k, o in zip(keys, outs):
        if (k.endswith("targ") and pgt >= 1 + ("grad" in k) + 2 * ("hess" in k)) or \
           (not k.endswith("targ") and pg >= 1 + ("grad" in k) + 2 * ("hess" in k)):
            res[k] = o
    return res, ier.value


def _flags(variant):
    st, cd, p = variant.split("_")
    lvl = {"p": 1, "g": 2, "h": 3}[p]
    return int("c" in cd and cd != "d"), int("d" in cd), lvl if "s" in st else 0, \
        lvl if "t" in st else 0


@pytest.mark.parametrize("variant", W.VARIANTS)
def test_rfmm2d_wrappers_match_reference(glib, variant):
    if not refimpl.have_ref():
        pytest.skip("reference build absent")
    src, trg, q, d, v = _inputs(1, 3000, 1200, 3, True)
    got, ier = W.call_nd(glib, "r", variant, EPS, src, 1, False, q[0], d[0], v[0], trg)
    assert ier == 0
    ifc, ifd, pg, pgt = _flags(variant)
    want, rier = ref_guru("r", 1, EPS, src, q, d, v, trg, ifc, ifd, pg, pgt)
    assert rier == 0
    for k, w in want.items():
        assert W.rel_err(got[k].reshape(w.shape), w) <= TOL, (k, W.rel_err(got[k].reshape(w.shape), w))


@pytest.mark.parametrize("idivflag", [0, 1, 2])
@pytest.mark.parametrize("ifnear", [1, 0])
def test_rfmm2d_ndiv_matches_reference(glib, idivflag, ifnear):
    if not refimpl.have_ref():
        pytest.skip("reference build absent")
    nd = 2
    src, trg, q, d, v = _inputs(nd, 2500, 1700, 5 + idivflag, True)
    src[:, :1200] = 0.5 + 0.05 * (src[:, :1200] - 0.5)  # a cluster
    kw = dict(ndiv=9, idivflag=idivflag, ifnear=ifnear)
    got, ier = ref_guru("r", nd, EPS, src, q, d, v, trg, 1, 1, 3, 3, lib=glib, **kw)
    want, rier = ref_guru("r", nd, EPS, src, q, d, v, trg, 1, 1, 3, 3, **kw)
    assert ier == 0 and rier == 0
    for k in want:
        assert W.rel_err(got[k], want[k]) <= TOL, k


@pytest.mark.parametrize("family", ["l", "c", "h", "r"])
@pytest.mark.parametrize("variant", ["s_c_p", "t_d_g", "st_cd_h", "st_c_g", "s_cd_h"])
def test_vec_wrappers_match_reference_guru(glib, family, variant):
    if not refimpl.have_ref():
        pytest.skip("reference build absent")
    nd = 3
    src, trg, q, d, v = _inputs(nd, 2000, 900, 7, family == "r")
    zk = 8.0 + 0.5j if family == "h" else None
    got, ier = W.call_nd(glib, family, variant, EPS, src, nd, True, q, d, v, trg, zk=zk)
    assert ier == 0
    ifc, ifd, pg, pgt = _flags(variant)
    want, rier = ref_guru(family, nd, EPS, src, q, d, v, trg, ifc, ifd, pg, pgt, zk=zk)
    assert rier == 0
    tol = 1e-10 if family == "h" else TOL
    for k, w in want.items():
        g = got[k].reshape(w.shape)
        assert W.rel_err(g, w) <= tol, (k, W.rel_err(g, w))


def test_rfmm2d_mixed_within_eps(glib):
    """rfmm2d at eps 1e-6 in the mixed mode: potential and gradient at the
    targets within eps of the FP64 direct sum (the real parts of the
    complex-Laplace sums with real strengths)."""
    glib.fmm2d_b200_set_precision(2)
    try:
        src, trg, q, d, v = _inputs(1, 40000, 10000, 9, True)
        got, ier = W.call_nd(glib, "r", "st_cd_g", 1e-6, src, 1, False, q[0], d[0], v[0], trg)
    finally:
        glib.fmm2d_b200_set_precision(1)
    assert ier == 0
    m = 300
    ns = src.shape[1]
    pot = np.zeros(m, complex)
    grad = np.zeros((m, 2), complex)
    qc = q[0].astype(complex)
    dc = d[0].astype(complex)
    refimpl.orc().oracle_l2d_direct(
        ns, W._p(np.ascontiguousarray(src.T)), 1, W._p(qc), 1, W._p(dc),
        W._p(np.ascontiguousarray(v[0].T)), 0, m, W._p(np.ascontiguousarray(trg[:, :m].T)), 2,
        W._p(pot), W._p(grad), None, 1e-300)
    assert W.rel_err(got["pottarg"][:m, 0], pot.real) <= 1e-6
    assert W.rel_err(got["gradtarg"][:m, :, 0], grad.real) <= 1e-6
