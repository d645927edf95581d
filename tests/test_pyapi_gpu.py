"""The fmm2dpy-compatible Python front end (python/fmm2dpy/fmm2d.py:20,
459, 715) against the flag wrappers of the same library and, for nd > 1,
against one call per density."""
import numpy as np
import pytest

import wrappers as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fm():
    import fmm2d_c_translation_b200 as m
    return m


def _inputs(ns=2000, nt=700, nd=1, seed=4):
    rng = np.random.default_rng(seed)
    src = rng.random((2, ns))
    trg = rng.random((2, nt))
    shp = (ns,) if nd == 1 else (nd, ns)
    q = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    d = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    v = rng.standard_normal((2, ns) if nd == 1 else (nd, 2, ns))
    return src, trg, q, d, v


@pytest.mark.parametrize("fam", ["l", "c", "h"])
@pytest.mark.parametrize("pg,pgt", [(1, 0), (2, 2), (0, 1), (3, 3)])
def test_front_end_matches_wrappers(fm, fam, pg, pgt):
    src, trg, q, d, v = _inputs()
    kw = dict(eps=1e-9, sources=src, charges=q, dipstr=d, pg=pg, pgt=pgt)
    if fam != "c":
        kw["dipvec"] = v
    if pgt:
        kw["targets"] = trg
    zk = 6.0 + 0.2j
    if fam == "h":
        kw["zk"] = zk
    out = {"l": fm.lfmm2d, "c": fm.cfmm2d, "h": fm.hfmm2d}[fam](**kw)
    assert out.ier == 0
    st = ("s" if pg else "") + ("t" if pgt else "")
    var = f"{st}_cd_{'pgh'[max(pg, pgt) - 1]}"
    ref, ier = W.call(fm.lib(), fam, var, 1e-9, src, q, d, v, trg, zk=zk if fam == "h" else None)
    assert ier == 0
    gc = 1 if fam == "c" else 2
    if pg:
        np.testing.assert_array_equal(out.pot, ref["pot"])
        if pg >= 2:
            g = out.grad if gc == 1 else out.grad.T
            np.testing.assert_array_equal(g, ref["grad"])
    if pgt:
        np.testing.assert_array_equal(out.pottarg, ref["pottarg"])
        if pgt >= 3:
            h = out.hesstarg if gc == 1 else out.hesstarg.T
            np.testing.assert_array_equal(h, ref["hesstarg"])


@pytest.mark.parametrize("fam", ["l", "h"])
def test_front_end_nd(fm, fam):
    nd = 3
    src, trg, q, d, v = _inputs(nd=nd, seed=9)
    kw = dict(eps=1e-10, sources=src, charges=q, dipstr=d, dipvec=v, targets=trg, pg=2, pgt=2,
              nd=nd)
    if fam == "h":
        kw["zk"] = 3.0
    f = fm.lfmm2d if fam == "l" else fm.hfmm2d
    out = f(**kw)
    assert out.pot.shape == (nd, src.shape[1]) and out.grad.shape == (nd, 2, src.shape[1])
    for j in range(nd):
        kj = dict(kw, charges=q[j], dipstr=d[j], dipvec=v[j], nd=1)
        oj = f(**kj)
        assert W.rel_err(out.pot[j], oj.pot) < 1e-12
        assert W.rel_err(out.gradtarg[j], oj.gradtarg) < 1e-12


def test_rfmm2d_front_end(fm):
    """fmm2dpy-style rfmm2d: real outputs equal the rfmm2d wrappers'."""
    rng = np.random.default_rng(31)
    ns, nt = 3000, 700
    src, trg = rng.random((2, ns)), rng.random((2, nt))
    q, d = rng.standard_normal(ns), rng.standard_normal(ns)
    v = rng.standard_normal((2, ns))
    out = fm.rfmm2d(eps=1e-9, sources=src, charges=q, dipstr=d, dipvec=v, targets=trg, pg=2,
                    pgt=3)
    assert out.ier == 0 and out.pot.dtype == np.float64
    ref, ier = W.call_nd(fm.lib(), "r", "st_cd_h", 1e-9, src, 1, False, q, d, v, trg)
    assert ier == 0
    np.testing.assert_array_equal(out.pot, ref["pot"][:, 0])
    np.testing.assert_array_equal(out.grad.T, ref["grad"][:, :, 0])
    np.testing.assert_array_equal(out.hesstarg.T, ref["hesstarg"][:, :, 0])
