"""Batches of independent problems evaluated as one forest
(fmm2d_b200_fmm2d_batch): argument checks on the host, and -- on a GPU --
every problem's outputs against the same problem run alone, in FP64 and in
the mixed mode, for uneven sizes, extents and positions."""
import ctypes

import numpy as np
import pytest

import pointsets as ps
import wrappers as W


def test_batch_rejects_bad_arguments():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    ns = (ctypes.c_int * 1)(10)
    # no problems; no strengths; missing output lists: all refused on the host
    assert L.fmm2d_b200_fmm2d_batch(0, 0, ctypes.c_double(1e-6), ns, None, None, None, None,
                                    0, None, None, None, None, None, 0, None, None, None) == 4
    srcs = (ctypes.c_void_p * 1)(None)
    assert L.fmm2d_b200_fmm2d_batch(0, 1, ctypes.c_double(1e-6), ns, srcs, None, None, None,
                                    1, None, None, None, None, None, 0, None, None, None) == 4


def _problems(seed, kernel, with_targets):
    rng = np.random.default_rng(seed)
    sizes = [37, 500, 3000, 20000, 1200, 8000, 150]
    probs = []
    for k, n in enumerate(sizes):
        scale, shift = 10.0 ** rng.uniform(-2, 1), rng.uniform(-5, 5, (2, 1))
        pts = ps.blobs(n, seed + k) if k % 2 else ps.uniform(n, seed + k)
        p = {"sources": shift + scale * pts,
             "charges": rng.standard_normal(n) + 1j * rng.standard_normal(n),
             "dipstr": rng.standard_normal(n) + 1j * rng.standard_normal(n)}
        if kernel == "l":
            th = rng.uniform(0, 2 * np.pi, n)
            p["dipvec"] = np.stack([np.cos(th), np.sin(th)])
        if with_targets and k % 3 != 1:
            p["targets"] = shift + scale * ps.uniform(n // 2 + 1, seed + 100 + k)
        probs.append(p)
    return probs


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["l", "c"])
@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_batch_matches_single_calls(kernel, mode):
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    probs = _problems(7, kernel, True)
    f = fm.lfmm2d if kernel == "l" else fm.cfmm2d
    eps = 1e-12 if mode == "fp64" else 1e-6
    L.fmm2d_b200_set_precision(1 if mode == "fp64" else 2)
    try:
        outs = fm.fmm2d_batch(kernel, eps=eps, problems=probs, pg=2, pgt=2)
    finally:
        L.fmm2d_b200_set_precision(1)
    try:
        for p, o in zip(probs, outs):
            kw = {k: v for k, v in p.items()}
            want = f(eps=1e-12, pg=2, pgt=2 if "targets" in p else 0, **kw)
            tol = 1e-10 if mode == "fp64" else 1e-6
            keys = ["grad", "gradtarg"] if kernel == "c" else ["pot", "grad", "pottarg", "gradtarg"]
            for k in keys:
                if getattr(want, k) is None:
                    continue
                assert W.rel_err(getattr(o, k), getattr(want, k)) <= tol, (len(p["charges"]), k)
    finally:
        L.fmm2d_b200_set_precision(0)
