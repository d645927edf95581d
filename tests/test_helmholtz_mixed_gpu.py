"""Helmholtz FMM in the mixed mode: the M2L of the levels of order <= 23 as
TF32 x 3 contractions on the tcgen05 tensor cores (helm_m2l_tc.cu), the
rest in FP64 (H0/H1, P2P, expansions, rescaling).

* every result within the requested eps of the FP64 direct sum (relative
  l2 over sampled points) and of the reference's FP64 FMM on the same
  inputs, at zk = 10, 200 and 2 + 3i (complex wavenumber), eps 1e-3 and 1e-6;
* the same evaluation with the FP64 CUDA-core M2L (FMM2D_B200_HELM_M2L=tile)
  agrees to the TF32 x 3 level;
* several channels (guru driver, nd = 3) against nd single-channel calls;
* results are deterministic (two calls give the same bits).
"""
import ctypes

import numpy as np
import pytest

import refimpl
import wrappers as W
from test_helmholtz_gpu import h_direct

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mlib():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    L.fmm2d_b200_set_precision(2)
    yield L
    L.fmm2d_b200_set_precision(0)


def _inputs(ns, nt, seed):
    rng = np.random.default_rng(seed)
    src = rng.random((2, ns))
    trg = rng.random((2, nt))
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    th = rng.uniform(0, 2 * np.pi, ns)
    v = np.stack([np.cos(th), np.sin(th)])
    return src, trg, q, d, v


CASES = [(10.0 + 0j, 1e-6), (200.0 + 0j, 1e-6), (2.0 + 3.0j, 1e-6), (10.0 + 0j, 1e-3),
         (200.0 + 0j, 1e-3)]


@pytest.mark.parametrize("zk,eps", CASES, ids=[f"zk{z}-eps{e:g}" for z, e in CASES])
def test_mixed_within_eps_of_direct_and_reference(mlib, zk, eps):
    src, trg, q, d, v = _inputs(60000, 20000, 3)
    got, ier = W.call(mlib, "h", "st_cd_g", eps, src, q, d, v, trg, zk=zk)
    assert ier == 0
    m = 300
    pot, grad, _ = h_direct(mlib, zk, src, q, d, v, trg[:, :m], 2, 1, 1)
    assert W.rel_err(got["pottarg"][:m], pot) <= eps
    assert W.rel_err(got["gradtarg"][:m], grad) <= eps
    pot, grad, _ = h_direct(mlib, zk, src, q, d, v, src[:, :m], 2, 1, 1)
    assert W.rel_err(got["pot"][:m], pot) <= eps
    assert W.rel_err(got["grad"][:m], grad) <= eps
    if refimpl.have_ref():
        want, rier = W.call(refimpl.ref(), "h", "st_cd_g", eps, src, q, d, v, trg, zk=zk)
        assert rier == 0
        for k in want:
            assert W.rel_err(got[k], want[k]) <= eps, (k, W.rel_err(got[k], want[k]))


@pytest.mark.parametrize("zk", [10.0 + 0j, 200.0 + 0j, 2.0 + 3.0j])
def test_tensor_core_m2l_matches_fp64_m2l(mlib, monkeypatch, zk):
    """Same tree and passes, only the M2L differs: the difference is the
    TF32 x 3 rounding (about 2^-22 = 2.4e-7 relative per product; measured
    2.6e-7 and 3.2e-7 in the potential at zk 10 and 200), held to 5e-7."""
    src, trg, q, d, v = _inputs(40000, 10000, 5)
    tc, ier = W.call(mlib, "h", "st_cd_g", 1e-6, src, q, d, v, trg, zk=zk)
    assert ier == 0
    monkeypatch.setenv("FMM2D_B200_HELM_M2L", "tile")
    f64, ier = W.call(mlib, "h", "st_cd_g", 1e-6, src, q, d, v, trg, zk=zk)
    assert ier == 0
    for k in tc:
        assert W.rel_err(tc[k], f64[k]) <= 5e-7, (k, W.rel_err(tc[k], f64[k]))


def test_mixed_is_deterministic(mlib):
    src, trg, q, d, v = _inputs(30000, 0, 8)
    a, _ = W.call(mlib, "h", "s_cd_p", 1e-6, src, q, d, v, None, zk=200.0 + 0j)
    b, _ = W.call(mlib, "h", "s_cd_p", 1e-6, src, q, d, v, None, zk=200.0 + 0j)
    np.testing.assert_array_equal(a["pot"], b["pot"])


def test_mixed_zk200_config_shape(mlib):
    """hfmm2d_s_cd_p at zk = 200 and eps = 1e-6 (the 2e6-point configuration's
    arithmetic) at 2e5 sources: within eps of the reference FMM and of the
    direct sum."""
    rng = np.random.default_rng(200)
    ns = 200000
    src = rng.random((2, ns))
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    th = rng.uniform(0, 2 * np.pi, ns)
    v = np.stack([np.cos(th), np.sin(th)])
    zk = 200.0 + 0j
    out, ier = W.call(mlib, "h", "s_cd_p", 1e-6, src, q, d, v, None, zk=zk)
    assert ier == 0
    pot, _, _ = h_direct(mlib, zk, src, q, d, v, src[:, :300], 1, 1, 1)
    assert W.rel_err(out["pot"][:300], pot) <= 1e-6
    if refimpl.have_ref():
        ro, rier = W.call(refimpl.ref(), "h", "s_cd_p", 1e-6, src, q, d, v, None, zk=zk)
        assert rier == 0
        assert W.rel_err(out["pot"], ro["pot"]) <= 1e-6


def test_mixed_several_channels(mlib):
    import fmm2d_c_translation_b200 as fm
    rng = np.random.default_rng(21)
    nd, ns, nt = 3, 30000, 5000
    src = rng.random((2, ns))
    trg = rng.random((2, nt))
    q = rng.standard_normal((nd, ns)) + 1j * rng.standard_normal((nd, ns))
    kw = dict(eps=1e-6, zk=40.0, sources=src, charges=q, targets=trg, pg=2, pgt=2, nd=nd)
    out = fm.hfmm2d(**kw)
    for j in range(nd):
        oj = fm.hfmm2d(**dict(kw, charges=q[j], nd=1))
        assert W.rel_err(out.pot[j], oj.pot) <= 1e-6
        assert W.rel_err(out.gradtarg[j], oj.gradtarg) <= 1e-6
