"""The MATLAB/MEX entry points lfmm2d_ndiv_ and cfmm2d_ndiv_
(matlab/fmm2d.c:1256-1286; c_translation/src/lfmm2d_ndiv.c:57,
c_translation/src/cfmm2d_ndiv.c:94) against the reference's own C
translation on the same inputs.

They take the caller's leaf capacity ndiv, the subdivision rule idivflag
(0: split a box with more than ndiv sources, 1: more than ndiv targets,
2: more than ndiv of either; pts_tree2d.c:212-214) and ifnear (0 drops the
list-1 direct interactions).  The GPU tree is bit-exact against the
reference's for every rule, so the outputs agree to FP64 round-off
(relative l2 difference <= 1e-11 at eps 1e-10).  Also checks the timeinfo
array: the reference's C translation leaves it zero, the GPU library fills
it with the device time of each FMM step in seconds.
"""
import ctypes

import numpy as np
import pytest

import refimpl
import wrappers as W

pytestmark = pytest.mark.gpu

_P = ctypes.c_void_p
EPS = 1e-10
TOL = 1e-11


def _p(a):
    return a.ctypes.data_as(_P)


def _ci(x):
    return ctypes.byref(ctypes.c_int(x))


def _inputs(ns, nt, nd, seed):
    rng = np.random.default_rng(seed)
    # clustered sources and uniform targets, so the three rules give
    # different trees
    src = np.clip(0.5 + 0.08 * rng.standard_normal((2, ns)), 0, 1)
    trg = rng.random((2, nt))
    cz = lambda *s: np.ascontiguousarray(rng.standard_normal(s) + 1j * rng.standard_normal(s))
    return (np.asfortranarray(src), np.asfortranarray(trg), cz(ns, nd), cz(ns, nd),
            np.ascontiguousarray(rng.standard_normal((ns, 2, nd))))


def _call(lib, fam, nd, src, q, d, v, trg, ndiv, idivflag, ifnear, pg=3, pgt=3):
    ns, nt = src.shape[1], trg.shape[1]
    gc, hc = (2, 3) if fam == "l" else (1, 1)
    z = lambda n, c: np.zeros((n, c, nd) if c > 1 else (n, nd), np.complex128)
    outs = [z(ns, 1), z(ns, gc), z(ns, hc), z(nt, 1), z(nt, gc), z(nt, hc)]
    timeinfo = np.full(8, -1.0)
    ier = ctypes.c_int(-1)
    iper = ctypes.c_int(0)
    args = [_ci(nd), ctypes.byref(ctypes.c_double(EPS)), _ci(ns), _p(src), _ci(1), _p(q),
            _ci(1), _p(d)]
    if fam == "l":
        args.append(_p(v))
    args += [ctypes.byref(iper), _ci(pg), _p(outs[0]), _p(outs[1]), _p(outs[2]), _ci(nt),
             _p(trg), _ci(pgt), _p(outs[3]), _p(outs[4]), _p(outs[5]), _ci(ndiv),
             _ci(idivflag), _ci(ifnear), _p(timeinfo), ctypes.byref(ier)]
    getattr(lib, f"{fam}fmm2d_ndiv_")(*args)
    return ier.value, outs, timeinfo


@pytest.fixture(scope="module")
def glib():
    import fmm2d_c_translation_b200 as fm
    return fm.lib()


@pytest.mark.parametrize("fam", ["l", "c"])
@pytest.mark.parametrize("idivflag", [0, 1, 2])
@pytest.mark.parametrize("ifnear", [1, 0])
@pytest.mark.parametrize("ndiv", [7, 40])
def test_ndiv_driver_matches_reference(glib, fam, idivflag, ifnear, ndiv):
    if not refimpl.have_ref():
        pytest.skip("reference build absent")
    nd = 2 if ndiv == 7 else 1
    src, trg, q, d, v = _inputs(3000, 1700, nd, 11 + idivflag)
    ier, got, ti = _call(glib, fam, nd, src, q, d, v, trg, ndiv, idivflag, ifnear)
    rier, want, rti = _call(refimpl.ref(), fam, nd, src, q, d, v, trg, ndiv, idivflag, ifnear)
    assert ier == 0 and rier == 0
    for g, w in zip(got, want):
        assert W.rel_err(g, w) <= TOL
    # the reference's C translation reports zeros; the GPU library reports
    # the device time of each step (seconds), nonnegative, P2P only with ifnear
    assert np.all(rti == 0.0)
    assert np.all(ti >= 0.0) and ti.sum() > 0.0
    assert ti[3] > 0.0  # M2L ran
    if ifnear:
        assert ti[7] > 0.0


def test_ndiv_matches_default_driver_at_the_rule(glib):
    """With ndiv equal to the rule's leaf capacity (lndiv2d) and idivflag 0,
    the ndiv driver gives the guru driver's outputs (same tree, same kernels;
    only round-off from the order of independent sums may differ)."""
    import fmm2d_c_translation_b200 as fm
    src, trg, q, d, v = _inputs(2000, 900, 1, 5)
    nd = 1
    ndiv = glib.fmm2d_b200_leaf_capacity(ctypes.c_double(EPS), 2000, 900)
    ier, got, _ = _call(glib, "l", nd, src, q, d, v, trg, ndiv, 0, 1)
    assert ier == 0, fm.last_error()
    want, ier2 = W.call(glib, "l", "st_cd_h", EPS, src, q[:, 0], d[:, 0], v[:, :, 0].T, trg)
    assert ier2 == 0
    assert W.rel_err(got[0][:, 0], want["pot"]) <= 1e-14
    assert W.rel_err(got[3][:, 0], want["pottarg"]) <= 1e-14
    assert W.rel_err(got[4][:, :, 0], want["gradtarg"]) <= 1e-14
    assert W.rel_err(got[5][:, :, 0], want["hesstarg"]) <= 1e-14
