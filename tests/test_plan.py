"""Resident geometry (csrc/plan.cu): evaluations of new strengths on a plan
equal the one-shot drivers' results on the same points, call after call,
in both precision modes."""
import ctypes

import numpy as np
import pytest

import pointsets as ps
import wrappers as W


def test_plan_rejects_bad_arguments():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    h = ctypes.c_void_p()
    src = np.zeros((2, 10))
    # Helmholtz has no plan; ns = 0 is invalid: both fail before any device work
    assert L.fmm2d_b200_plan_create(2, 1, ctypes.c_double(1e-6), 10,
                                    src.ctypes.data_as(ctypes.c_void_p), 1, 0, 1, 0, None, 0,
                                    ctypes.byref(h)) == 4
    assert L.fmm2d_b200_plan_create(0, 1, ctypes.c_double(1e-6), 0,
                                    src.ctypes.data_as(ctypes.c_void_p), 1, 0, 1, 0, None, 0,
                                    ctypes.byref(h)) == 4
    assert not h.value
    assert L.fmm2d_b200_plan_eval(None, *([None] * 9)) == 4
    assert L.fmm2d_b200_plan_destroy(None) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("graph", ["on", "off"])
@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("kernel", ["l", "c"])
def test_plan_matches_one_shot(kernel, precision, graph, monkeypatch):
    """Evaluation 1 runs eagerly, 2 and 3 replay the captured CUDA graph
    (or stay eager with FMM2D_B200_PLAN_GRAPH=0); all equal the one-shot
    drivers' results on the same points."""
    import fmm2d_c_translation_b200 as fm
    if graph == "off":
        monkeypatch.setenv("FMM2D_B200_PLAN_GRAPH", "0")
    else:
        monkeypatch.delenv("FMM2D_B200_PLAN_GRAPH", raising=False)
    L = fm.lib()
    L.fmm2d_b200_set_precision(precision)
    try:
        rng = np.random.default_rng(8)
        ns, nt = 30000, 12000
        src, trg = ps.blobs(ns, 3), ps.uniform(nt, 4)
        eps = 1e-9 if precision == 1 else 1e-6
        plan = fm.Plan(kernel, eps=eps, sources=src, targets=trg, charges=True, dipoles=True,
                       pg=2, pgt=3)
        f = fm.lfmm2d if kernel == "l" else fm.cfmm2d
        for it in range(3):
            q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
            d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
            kw = dict(charges=q, dipstr=d)
            if kernel == "l":
                kw["dipvec"] = rng.standard_normal((2, ns))
            got = plan.eval(**kw)
            want = f(eps=eps, sources=src, targets=trg, pg=2, pgt=3, **kw)
            for k in ("pot", "grad", "pottarg", "gradtarg", "hesstarg"):
                assert W.rel_err(getattr(got, k), getattr(want, k)) <= 1e-14, (it, k)
            assert plan.uses_graph == (graph == "on" and it >= 1), it
        plan.close()
    finally:
        L.fmm2d_b200_set_precision(0)
