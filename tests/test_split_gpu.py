"""Split-precision M2L (precision mode 3): every Laplace / Cauchy pass in
FP64 except the multipole-to-local shift's terms of high total order
i + j, which run as TF32 x 3 slot GEMMs on the tcgen05 tensor cores and are
added to the FP64 triangle i + j < NT (m2l.cu, m2l_split_fp64; the shift is
the reference's l2dmploc, c_translation/src/laprouts2d.c:886-994).

* at eps 1e-9 and 1e-10, on uniform, clustered and starfish (boundary
  curve, deep tree) points, every output within eps of the all-FP64 mode,
  and its error against the FP64 direct sum and the reference FMM at most
  eps above the all-FP64 mode's own;
* at eps 1e-12 (order 37) the split keeps the FP64 M2L: the results equal
  the all-FP64 mode's to the bit;
* the split path is the one that ran (its triangle order is reported in
  the call's profile);
* Cauchy wrappers and several channels;
* two calls give the same bits.
"""
import ctypes
import os

import numpy as np
import pytest

import pointsets as ps
import refimpl
import wrappers as W
from test_mixed_gpu import direct, inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def slib():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    L.fmm2d_b200_set_precision(3)
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


@pytest.mark.parametrize("eps", [1e-9, 1e-10])
@pytest.mark.parametrize("dist", ["uniform", "blobs", "starfish"])
def test_split_within_eps(slib, eps, dist):
    """The split adds at most eps to the all-FP64 mode's own error against
    the FP64 direct sum and against the reference FMM (gradients and
    Hessians of clustered points carry FMM errors above eps in both modes),
    and stays within eps of the all-FP64 result."""
    src, trg, q, d, v = inputs(60000, 20000, 11, dist)
    slib.fmm2d_b200_set_profiling(1)
    try:
        got, ier = W.call(slib, "l", "st_cd_h", eps, src, q, d, v, trg)
        prof = _profile(slib)
    finally:
        slib.fmm2d_b200_set_profiling(0)
    assert ier == 0
    assert prof.get("#m2l_split_nt", 0) >= 8  # the split M2L ran
    slib.fmm2d_b200_set_precision(1)
    try:
        f64, ier = W.call(slib, "l", "st_cd_h", eps, src, q, d, v, trg)
    finally:
        slib.fmm2d_b200_set_precision(3)
    assert ier == 0
    m = 400
    dp, dg, dh = direct(src, q, d, v, trg, m, 3)
    sp, sg, sh = direct(src, q, d, v, src, m, 3)
    ref = {"pottarg": dp, "gradtarg": dg, "hesstarg": dh, "pot": sp, "grad": sg, "hess": sh}
    for k, want in ref.items():
        e_split = W.rel_err(got[k][:m], want)
        e_64 = W.rel_err(f64[k][:m], want)
        assert e_split <= e_64 + eps, (k, e_split, e_64)
    for k in f64:
        assert W.rel_err(got[k], f64[k]) <= eps, (k, W.rel_err(got[k], f64[k]))
    if refimpl.have_ref():
        want, rier = W.call(refimpl.ref(), "l", "st_cd_h", eps, src, q, d, v, trg)
        assert rier == 0
        for k in want:
            e_split, e_64 = W.rel_err(got[k], want[k]), W.rel_err(f64[k], want[k])
            assert e_split <= e_64 + eps, (k, e_split, e_64)


def test_split_keeps_fp64_at_high_order(slib):
    src, trg, q, d, v = inputs(30000, 10000, 23, "blobs")
    slib.fmm2d_b200_set_profiling(1)
    try:
        got, ier = W.call(slib, "l", "st_cd_h", 1e-12, src, q, d, v, trg)
        prof = _profile(slib)
    finally:
        slib.fmm2d_b200_set_profiling(0)
    assert ier == 0
    assert "#m2l_split_nt" not in prof
    slib.fmm2d_b200_set_precision(1)
    try:
        want, ier = W.call(slib, "l", "st_cd_h", 1e-12, src, q, d, v, trg)
    finally:
        slib.fmm2d_b200_set_precision(3)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k])


def test_split_matches_fp64_mode(slib):
    """Same tree and passes, only the M2L's tail differs: the split result
    stays within eps 1e-9 of the all-FP64 one."""
    src, trg, q, d, v = inputs(80000, 30000, 13, "starfish")
    got, ier = W.call(slib, "l", "st_cd_g", 1e-9, src, q, d, v, trg)
    assert ier == 0
    slib.fmm2d_b200_set_precision(1)
    try:
        want, ier = W.call(slib, "l", "st_cd_g", 1e-9, src, q, d, v, trg)
    finally:
        slib.fmm2d_b200_set_precision(3)
    assert ier == 0
    for k in want:
        assert W.rel_err(got[k], want[k]) <= 1e-9, (k, W.rel_err(got[k], want[k]))


@pytest.mark.parametrize("variant", ["s_c_g", "t_d_p", "st_cd_h"])
def test_split_cauchy_matches_reference(slib, variant):
    src, trg, q, d, v = inputs(30000, 8000, 15, "blobs")
    got, ier = W.call(slib, "c", variant, 1e-9, src, q, d, v, trg)
    assert ier == 0
    if not refimpl.have_ref():
        pytest.skip("reference build absent")
    want, rier = W.call(refimpl.ref(), "c", variant, 1e-9, src, q, d, v, trg)
    assert rier == 0
    for k in want:
        assert W.rel_err(got[k], want[k]) <= 1e-9, (k, W.rel_err(got[k], want[k]))


def test_split_several_channels(slib):
    import fmm2d_c_translation_b200 as fm
    rng = np.random.default_rng(17)
    nd, ns, nt = 3, 30000, 6000
    src = rng.random((2, ns))
    trg = rng.random((2, nt))
    q = rng.standard_normal((nd, ns)) + 1j * rng.standard_normal((nd, ns))
    kw = dict(eps=1e-9, sources=src, charges=q, targets=trg, pg=2, pgt=2, nd=nd)
    out = fm.lfmm2d(**kw)
    for j in range(nd):
        oj = fm.lfmm2d(**dict(kw, charges=q[j], nd=1))
        assert W.rel_err(out.pot[j], oj.pot) <= 1e-9
        assert W.rel_err(out.gradtarg[j], oj.gradtarg) <= 1e-9


def test_split_is_deterministic(slib):
    src, trg, q, d, v = inputs(40000, 0, 19, "uniform")
    a, _ = W.call(slib, "l", "s_cd_g", 1e-9, src, q, d, v, None)
    b, _ = W.call(slib, "l", "s_cd_g", 1e-9, src, q, d, v, None)
    np.testing.assert_array_equal(a["pot"], b["pot"])
    np.testing.assert_array_equal(a["grad"], b["grad"])


@pytest.mark.parametrize("nt_order", ["8", "24"])
def test_split_triangle_orders(slib, monkeypatch, nt_order):
    """Triangles set by FMM2D_B200_SPLIT_NT (which also lifts the order
    limit): at eps 1e-12 (order 37) both stay within 1e-9 of the FP64
    direct sum (the smaller triangle leaves more of the shift to the
    TF32 x 3 tail)."""
    monkeypatch.setenv("FMM2D_B200_SPLIT_NT", nt_order)
    src, trg, q, d, v = inputs(30000, 10000, 21, "uniform")
    got, ier = W.call(slib, "l", "st_c_g", 1e-12, src, q, None, None, trg)
    assert ier == 0
    m = 300
    dp, dg, _ = direct(src, q, np.zeros_like(q), v, trg, m, 2)
    tol = 1e-12 if nt_order == "24" else 1e-9
    assert W.rel_err(got["pottarg"][:m], dp) <= tol
    assert W.rel_err(got["gradtarg"][:m], dg) <= tol
