"""The autotuner of the mixed-precision path (csrc/autotune.cu): the
per-order M2L-form table on the host, and -- on a GPU -- a tuning run whose
choice is kept for later calls, which stay within eps of the reference."""
import ctypes

import numpy as np
import pytest

import refimpl
import wrappers as W


@pytest.fixture(scope="module")
def L():
    import fmm2d_c_translation_b200 as fm
    return fm.lib()


def test_m2l_form_table(L, monkeypatch):
    monkeypatch.delenv("FMM2D_B200_M2L", raising=False)
    assert L.fmm2d_b200_m2l_form(18) == 0
    assert L.fmm2d_b200_set_m2l_form(18, 2) == 0
    assert L.fmm2d_b200_m2l_form(18) == 2
    monkeypatch.setenv("FMM2D_B200_M2L", "tile")
    assert L.fmm2d_b200_m2l_form(18) == 1          # the environment wins
    monkeypatch.delenv("FMM2D_B200_M2L")
    assert L.fmm2d_b200_set_m2l_form(18, 0) == 0
    assert L.fmm2d_b200_set_m2l_form(18, 3) == 4   # no such form
    assert L.fmm2d_b200_set_m2l_form(200, 0) == 4  # no such order


def test_autotune_rejects_bad_workload(L):
    nd, fm_, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
    ier = L.fmm2d_b200_autotune(0, ctypes.c_double(1e-6), 0, None, 0, None, 1, 0, 1, 0,
                                ctypes.byref(nd), ctypes.byref(fm_), ctypes.byref(ms))
    assert ier == 4


@pytest.mark.gpu
def test_autotune_choice_is_kept_and_accurate(L, monkeypatch):
    import fmm2d_c_translation_b200 as fm
    monkeypatch.delenv("FMM2D_B200_MIXED_NDIV", raising=False)
    monkeypatch.delenv("FMM2D_B200_M2L", raising=False)
    eps = 1e-6
    p = L.fmm2d_b200_laplace_nterms(ctypes.c_double(eps))
    try:
        ndiv, form, ms = fm.autotune("l", eps=eps, ns=60000, nt=30000, dipoles=True, pg=2, pgt=2)
        assert ndiv in (12, 16, 20, 24, 32, 40, 48, 64)
        assert form in (0, 1, 2) and ms > 0
        assert L.fmm2d_b200_m2l_form(p) == form
        assert L.fmm2d_b200_mixed_leaf_capacity(ctypes.c_double(eps), 100, 0) == ndiv
        rng = np.random.default_rng(3)
        ns, nt = 30000, 10000
        src, trg = rng.random((2, ns)), rng.random((2, nt))
        q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
        d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
        th = rng.uniform(0, 2 * np.pi, ns)
        v = np.stack([np.cos(th), np.sin(th)])
        L.fmm2d_b200_set_precision(2)
        got, ier = W.call(L, "l", "st_cd_g", eps, src, q, d, v, trg)
        want, ier2 = W.call(refimpl.ref(), "l", "st_cd_g", eps, src, q, d, v, trg)
        assert ier == 0 and ier2 == 0
        for k in want:
            assert W.rel_err(got[k], want[k]) <= eps, k
    finally:
        L.fmm2d_b200_set_precision(0)
        L.fmm2d_b200_set_leaf_capacity(p, 0)
        L.fmm2d_b200_set_m2l_form(p, 0)
