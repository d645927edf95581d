"""Failure detection without a GPU fault.

The reference reports exactly one failure to its callers: ier = 4 when a
workspace allocation fails (src/helmholtz/hfmm2d.f:374-381,
src/laplace/cfmm2d.f).  The B200 library adds bounded waits inside its
tensor-core kernels.  Both are exercised here by host-side injection:

* an allocation failure injected at several points of a call: the call
  returns ier = 4 with a message, releases every device allocation it made,
  and the next call succeeds with the same results as before;
* a stalled tensor-core issuer (it issues and commits nothing) with a 1 ms
  wait limit: the other roles' bounded waits run out, the kernel sets its
  error flag and returns, the call reports ier = 4, and the next call
  succeeds.  No kernel traps or faults; the context stays usable.
"""
import ctypes

import numpy as np
import pytest

import wrappers as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    import fmm2d_c_translation_b200 as fm
    lib = fm.lib()
    lib.fmm2d_b200_inject_alloc_failure.argtypes = [ctypes.c_longlong]
    lib.fmm2d_b200_inject_tc_stall.argtypes = [ctypes.c_int, ctypes.c_double]
    yield lib
    lib.fmm2d_b200_inject_alloc_failure(0)
    lib.fmm2d_b200_inject_tc_stall(0, 0.0)
    lib.fmm2d_b200_set_precision(0)


def _inputs(ns, nt, seed=4):
    rng = np.random.default_rng(seed)
    src, trg = rng.random((2, ns)), rng.random((2, nt))
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    th = rng.uniform(0, 2 * np.pi, ns)
    return src, trg, q, d, np.stack([np.cos(th), np.sin(th)])


def _in_use(L):
    import torch
    torch.cuda.synchronize()
    b = ctypes.c_ulonglong(0)
    assert L.fmm2d_b200_device_bytes_in_use(ctypes.byref(b)) == 0
    return b.value


@pytest.mark.parametrize("fam", ["l", "h"])
@pytest.mark.parametrize("nth", [1, 2, 5, 11, 23])
def test_injected_allocation_failure(L, fam, nth):
    import fmm2d_c_translation_b200 as fm
    L.fmm2d_b200_set_precision(1)
    src, trg, q, d, v = _inputs(20000, 5000)
    zk = 15.0 + 0j if fam == "h" else None
    want, ier = W.call(L, fam, "st_cd_g", 1e-9, src, q, d, v, trg, zk=zk)
    assert ier == 0
    before = _in_use(L)
    L.fmm2d_b200_inject_alloc_failure(nth)
    got, ier = W.call(L, fam, "st_cd_g", 1e-9, src, q, d, v, trg, zk=zk)
    L.fmm2d_b200_inject_alloc_failure(0)
    assert ier == 4
    assert "allocation" in fm.last_error()
    assert _in_use(L) == before  # everything the failed call allocated was released
    again, ier = W.call(L, fam, "st_cd_g", 1e-9, src, q, d, v, trg, zk=zk)
    assert ier == 0
    for k in want:
        assert W.rel_err(again[k], want[k]) <= 1e-14, k


@pytest.mark.parametrize("fam", ["l", "h"])
def test_stalled_tensor_core_wait_runs_out(L, fam):
    import fmm2d_c_translation_b200 as fm
    L.fmm2d_b200_set_precision(2)
    src, trg, q, d, v = _inputs(200000, 50000, 6)
    zk = 40.0 + 0j if fam == "h" else None
    want, ier = W.call(L, fam, "st_cd_g", 1e-6, src, q, d, v, trg, zk=zk)
    assert ier == 0
    L.fmm2d_b200_inject_tc_stall(1, 1.0)
    try:
        _, ier = W.call(L, fam, "st_cd_g", 1e-6, src, q, d, v, trg, zk=zk)
    finally:
        L.fmm2d_b200_inject_tc_stall(0, 0.0)
    assert ier == 4
    assert "timed out" in fm.last_error()
    again, ier = W.call(L, fam, "st_cd_g", 1e-6, src, q, d, v, trg, zk=zk)
    assert ier == 0
    for k in want:
        assert W.rel_err(again[k], want[k]) <= 1e-14, k
