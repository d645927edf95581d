"""The no-allocation direct sum, fmm2d_b200_l2d_direct_noalloc.

It exists for callers that cannot have device memory allocated on their
behalf: applications whose GPU memory belongs to another allocator or to a
budget reserved up front, and latency-critical callers for which an
allocation call (which can synchronize the device) is not acceptable.  It
keeps its partial sums in a fixed 4 MiB device array instead of allocating.

This test calls it through the C ABI twice in a row, on device arrays, and
checks each result against the allocating entry point fmm2d_b200_l2d_direct
on the same inputs.  It also checks the two refusals that happen on the
host before any GPU work: host arrays, and a problem too large for the
scratch array.  The file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

import wrappers as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _setup(ns, nt, nd, seed):
    rng = np.random.default_rng(seed)
    src = rng.random((ns, 2))
    trg = np.concatenate([rng.random((nt - 2, 2)), src[:2]])  # two coincident points
    cz = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    return src, trg, cz(ns, nd), cz(ns, nd), rng.standard_normal((ns, 2, nd))


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    import fmm2d_c_translation_b200 as fm

    L = fm.lib()
    L.fmm2d_b200_l2d_direct_noalloc.argtypes = (
        [ctypes.c_int] * 2 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                              ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        + [ctypes.c_void_p] * 3 + [ctypes.c_double, ctypes.c_void_p])
    ns, nt, nd, pgh = 40000, 1200, 1, 3
    src, trg, q, d, v = _setup(ns, nt, nd, 11)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.float64)).cuda()
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    dsrc, dtrg, dq, dd, dv = map(dev, (src, trg, q, d, v))
    shapes = [(nt, nd), (nt, 2, nd), (nt, 3, nd)]
    zeros = lambda: [torch.zeros(int(np.prod(s)) * 2, dtype=torch.float64,
                                 device="cuda") for s in shapes]

    want = zeros()
    assert L.fmm2d_b200_l2d_direct(nd, ns, P(dsrc), 1, P(dq), 1, P(dd), P(dv),
                                   nt, P(dtrg), pgh, *[P(o) for o in want],
                                   ctypes.c_double(1e-14)) == 0, fm.last_error()
    torch.cuda.synchronize()
    want = [w.cpu().numpy().view(complex) for w in want]

    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        got = zeros()
        ier = L.fmm2d_b200_l2d_direct_noalloc(
            nd, ns, P(dsrc), 1, P(dq), 1, P(dd), P(dv), nt, P(dtrg), pgh,
            *[P(o) for o in got], 1e-14, ctypes.c_void_p(stream))
        assert ier == 0, fm.last_error()
        torch.cuda.synchronize()
        for g, w in zip(got, want):
            assert W.rel_err(g.cpu().numpy().view(complex), w) <= TOL


def test_noalloc_refuses_what_it_cannot_do():
    import torch
    import fmm2d_c_translation_b200 as fm

    L = fm.lib()
    ns, nt, nd = 1000, 200, 1
    src, trg, q, d, v = _setup(ns, nt, nd, 12)
    pot = np.zeros((nt, nd), complex)
    # host arrays are refused before any GPU work
    ier = L.fmm2d_b200_l2d_direct_noalloc(
        nd, ns, W._p(src), 1, W._p(q), 0, None, None, nt, W._p(trg), 1,
        W._p(pot), None, None, ctypes.c_double(1e-14), None)
    assert ier == 4 and "device arrays" in fm.last_error()
    # a problem whose per-chunk partials exceed the 4 MiB scratch is refused
    big = 50000  # 50000 targets x 6 outputs > 262144 values
    dsrc = torch.zeros(2 * ns, dtype=torch.float64, device="cuda")
    dq = torch.zeros(2 * ns, dtype=torch.float64, device="cuda")
    dtrg = torch.zeros(2 * big, dtype=torch.float64, device="cuda")
    outs = [torch.zeros(2 * big * k, dtype=torch.float64, device="cuda") for k in (1, 2, 3)]
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    ier = L.fmm2d_b200_l2d_direct_noalloc(
        nd, ns, P(dsrc), 1, P(dq), 0, None, None, big, P(dtrg), 3,
        *[P(o) for o in outs], ctypes.c_double(1e-14), None)
    assert ier == 4 and "exceeds" in fm.last_error()
