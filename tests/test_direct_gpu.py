"""GPU direct sums (fmm2d_b200_l2d_direct / c2d_direct) against the oracle's
FP64 direct sums, with host and with device arrays."""
import ctypes

import numpy as np
import pytest

import refimpl
import wrappers as W

pytestmark = pytest.mark.gpu


def setup(ns, nt, nd, seed):
    rng = np.random.default_rng(seed)
    src = rng.random((ns, 2))
    trg = np.concatenate([rng.random((nt - 2, 2)), src[:2]])  # two coincident
    cz = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    return src, trg, cz(ns, nd), cz(ns, nd), rng.standard_normal((ns, 2, nd))


@pytest.mark.parametrize("form", ["l", "c"])
@pytest.mark.parametrize("cd", ["c", "d", "cd"])
@pytest.mark.parametrize("pgh", [1, 2, 3])
def test_direct_matches_oracle(form, cd, pgh):
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    ns, nt, nd = 5000, 700, 1
    src, trg, q, d, v = setup(ns, nt, nd, 3)
    gc, hc = (2, 3) if form == "l" else (1, 1)
    pot = np.zeros((nt, nd), complex)
    grad = np.zeros((nt, gc, nd), complex)
    hess = np.zeros((nt, hc, nd), complex)
    thr = 1e-14
    fn = L.fmm2d_b200_l2d_direct if form == "l" else L.fmm2d_b200_c2d_direct
    args = [nd, ns, W._p(src), int("c" in cd), W._p(q), int("d" in cd), W._p(d)]
    if form == "l":
        args.append(W._p(v))
    args += [nt, W._p(trg), pgh, W._p(pot), W._p(grad), W._p(hess),
             ctypes.c_double(thr)]
    assert fn(*args) == 0, fm.last_error()
    op = np.zeros(nt, complex)
    og = np.zeros((nt, gc), complex)
    oh = np.zeros((nt, hc), complex)
    vv = np.ascontiguousarray(v[:, :, 0])
    if form == "l":
        refimpl.orc().oracle_l2d_direct(
            ns, W._p(src), int("c" in cd), W._p(np.ascontiguousarray(q[:, 0])),
            int("d" in cd), W._p(np.ascontiguousarray(d[:, 0])), W._p(vv), 0, nt,
            W._p(trg), pgh, W._p(op), W._p(og), W._p(oh), thr)
    else:
        refimpl.orc().oracle_c2d_direct(
            ns, W._p(src), int("c" in cd), W._p(np.ascontiguousarray(q[:, 0])),
            int("d" in cd), W._p(np.ascontiguousarray(d[:, 0])), 0, nt,
            W._p(trg), pgh, W._p(op), W._p(og), W._p(oh), thr)
    assert W.rel_err(pot[:, 0], op) < 1e-12
    if pgh >= 2:
        assert W.rel_err(grad[:, :, 0], og) < 1e-12
    if pgh >= 3:
        assert W.rel_err(hess[:, :, 0], oh) < 1e-12


def test_direct_device_arrays_nd2():
    import torch
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    ns, nt, nd = 200000, 3000, 2
    src, trg, q, d, v = setup(ns, nt, nd, 4)
    outs_h = [np.zeros((nt, nd), complex), np.zeros((nt, 2, nd), complex),
              np.zeros((nt, 3, nd), complex)]
    args_h = [W._p(src), W._p(q), W._p(d), W._p(v), W._p(trg)]
    assert L.fmm2d_b200_l2d_direct(nd, ns, args_h[0], 1, args_h[1], 1, args_h[2],
                                   args_h[3], nt, args_h[4], 3,
                                   *[W._p(o) for o in outs_h],
                                   ctypes.c_double(1e-14)) == 0
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.float64)).cuda()
    dsrc, dq, dd, dv, dtrg = map(dev, (src, q, d, v, trg))
    douts = [torch.zeros(o.size * 2, dtype=torch.float64, device="cuda") for o in outs_h]
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    assert L.fmm2d_b200_l2d_direct(nd, ns, P(dsrc), 1, P(dq), 1, P(dd), P(dv),
                                   nt, P(dtrg), 3, *[P(o) for o in douts],
                                   ctypes.c_double(1e-14)) == 0
    torch.cuda.synchronize()
    for h, dv_ in zip(outs_h, douts):
        got = dv_.cpu().numpy().view(complex).reshape(h.shape)
        np.testing.assert_array_equal(got, h)
