"""M2L of the mixed mode over runs of same-row boxes (windowed tcgen05
kernel) against the slot-table tensor-core kernel it replaces on dense
levels (FMM2D_B200_M2L=tile) and against the FP64 direct sum.

The two kernels apply the same truncated shifts (src/laplace/cfmm2d.f,
l2dmploc in c_translation/src/laprouts2d.c:886-994) with the same 3 x TF32
split, so their results agree far below eps; each stays within eps of the
direct sum.  Cases cover the three operand widths of the mixed orders (eps
1e-3, 1e-5, 1e-6), two channels per row (lfmm2d, nd = 1 and 2), one channel
per row (cfmm2d), and uniform and clustered points (dense levels in
windows, sparse ones on the slot tables)."""
import ctypes
import os

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


def _profile(L):
    buf = ctypes.create_string_buffer(1 << 16)
    L.fmm2d_b200_last_profile(buf, len(buf))
    out = {}
    for item in buf.value.decode().split(";"):
        if "=" in item:
            k, v = item.split("=", 1)
            out[k] = float(v)
    return out


class _M2LMode:
    """Sets FMM2D_B200_M2L (None = default) and phase profiling for a block."""

    def __init__(self, L, mode):
        self.L, self.mode = L, mode

    def __enter__(self):
        self.old = os.environ.get("FMM2D_B200_M2L")
        if self.mode is None:
            os.environ.pop("FMM2D_B200_M2L", None)
        else:
            os.environ["FMM2D_B200_M2L"] = self.mode
        self.L.fmm2d_b200_set_profiling(1)
        return self

    def __exit__(self, *exc):
        self.prof = _profile(self.L)
        self.L.fmm2d_b200_set_profiling(0)
        if self.old is None:
            os.environ.pop("FMM2D_B200_M2L", None)
        else:
            os.environ["FMM2D_B200_M2L"] = self.old
        return False


def _inputs(ns, nt, seed, dist):
    rng = np.random.default_rng(seed)
    if dist == "uniform":
        src, trg = ps.uniform(ns, seed), ps.uniform(nt, seed + 1)
    else:
        src, trg = ps.blobs(ns, seed), ps.blobs(nt, seed + 1)
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    th = rng.uniform(0, 2 * np.pi, ns)
    v = np.stack([np.cos(th), np.sin(th)])
    return src, trg, q, d, v


def _call(L, family, variant, eps, src, q, d, v, trg, mode):
    with _M2LMode(L, mode) as m:
        out, ier = W.call(L, family, variant, eps, src, q, d, v, trg)
    assert ier == 0
    return out, m.prof


@pytest.mark.parametrize("eps", [1e-3, 1e-5, 1e-6])
@pytest.mark.parametrize("dist", ["uniform", "blobs"])
def test_window_matches_slot_tables(mlib, eps, dist):
    src, trg, q, d, v = _inputs(300000, 200000, 5, dist)
    win, prof = _call(mlib, "l", "st_cd_g", eps, src, q, d, v, trg, None)
    assert prof.get("#m2l_window_levels", 0) >= 1, prof
    tile, prof_t = _call(mlib, "l", "st_cd_g", eps, src, q, d, v, trg, "tile")
    assert prof_t.get("#m2l_window_levels", 0) == 0
    for k in ("pot", "grad", "pottarg", "gradtarg"):
        # the same operators and split, summed in another order: well below eps
        assert W.rel_err(win[k], tile[k]) <= 0.2 * eps, (k, W.rel_err(win[k], tile[k]))
    m = 300
    pot = np.zeros(m, np.complex128)
    grad = np.zeros((m, 2), np.complex128)
    refimpl.orc().oracle_l2d_direct(
        src.shape[1], W._p(np.ascontiguousarray(src.T)), 1, W._p(q), 1, W._p(d),
        W._p(np.ascontiguousarray(v.T)), 0, m, W._p(np.ascontiguousarray(trg[:, :m].T)), 2,
        W._p(pot), W._p(grad), None, 1e-300)
    assert W.rel_err(win["pottarg"][:m], pot) <= eps
    assert W.rel_err(win["gradtarg"][:m], grad) <= eps


def test_window_two_densities(mlib):
    # nd = 2: four Cauchy channels, two launches of two channels per row
    nd, ns, nt = 2, 200000, 100000
    rng = np.random.default_rng(8)
    src, trg = ps.uniform(ns, 8), ps.uniform(nt, 9)
    q = np.asfortranarray(rng.standard_normal((nd, ns)) + 1j * rng.standard_normal((nd, ns)))
    d = np.asfortranarray(rng.standard_normal((nd, ns)) + 1j * rng.standard_normal((nd, ns)))
    v = np.asfortranarray(rng.standard_normal((nd, 2, ns)))
    res = []
    for mode in (None, "tile"):
        pot = np.zeros((nd, ns), np.complex128, order="F")
        grad = np.zeros((nd, 2, ns), np.complex128, order="F")
        pt = np.zeros((nd, nt), np.complex128, order="F")
        gt = np.zeros((nd, 2, nt), np.complex128, order="F")
        ier = ctypes.c_int(-1)
        I = lambda x: ctypes.byref(ctypes.c_int(x))  # noqa: E731
        with _M2LMode(mlib, mode) as m:
            mlib.lfmm2d_(I(nd), ctypes.byref(ctypes.c_double(1e-6)), I(ns), W._p(src),
                         I(1), W._p(q), I(1), W._p(d), W._p(v), I(0), I(2),
                         W._p(pot), W._p(grad), None, I(nt), W._p(trg), I(2),
                         W._p(pt), W._p(gt), None, ctypes.byref(ier))
        assert ier.value == 0
        if mode is None:
            assert m.prof.get("#m2l_window_levels", 0) >= 1, m.prof
        res.append((pot, grad, pt, gt))
    for a, b in zip(*res):
        assert W.rel_err(a, b) <= 2e-7


@pytest.mark.parametrize("variant", ["st_cd_g", "t_c_p"])
def test_window_cauchy_one_channel(mlib, variant):
    # cfmm2d: one Cauchy channel, 128 parents per run
    src, trg, q, d, v = _inputs(300000, 200000, 9, "uniform")
    win, prof = _call(mlib, "c", variant, 1e-6, src, q, d, v, trg, None)
    assert prof.get("#m2l_window_levels", 0) >= 1, prof
    tile, _ = _call(mlib, "c", variant, 1e-6, src, q, d, v, trg, "tile")
    for k in win:
        assert W.rel_err(win[k], tile[k]) <= 2e-7, (k, W.rel_err(win[k], tile[k]))
