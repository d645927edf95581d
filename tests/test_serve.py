"""The request loop (csrc/serve.cu): admission by the HBM budget, tickets,
and -- on a GPU -- that every result in a mixed stream equals the same
request run alone."""
import numpy as np
import pytest

import wrappers as W


@pytest.fixture(scope="module")
def fm():
    import fmm2d_c_translation_b200 as m
    return m


def _req(fm, kernel, n, seed, eps=1e-6, zk=5.0, pgt=0, precision=0):
    rng = np.random.default_rng(seed)
    src = rng.random((2, n))
    q = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    trg = rng.random((2, n // 2)) if pgt else None
    return fm.make_request(kernel, eps=eps, sources=src, charges=q, targets=trg, pg=2,
                           pgt=pgt, zk=zk, precision=precision)


def test_oversize_request_is_rejected(fm):
    srv = fm.Server(slots=2, hbm_budget=1e6)
    r, keep = _req(fm, "l", 100000, 1)
    assert srv.request_bytes(r) > 1e6
    t = srv.submit(r, keep)
    ier, times = srv.wait(t)
    assert ier == 4 and times[2] == 0.0
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_footprint_grows_with_size(fm):
    srv = fm.Server(slots=1, hbm_budget=1e12)
    small, _ = _req(fm, "l", 1000, 2)
    big, _ = _req(fm, "l", 100000, 2)
    helm, _ = _req(fm, "h", 100000, 2, zk=50.0)
    assert srv.request_bytes(small) < srv.request_bytes(big) < srv.request_bytes(helm)
    srv.close()


@pytest.mark.gpu
def test_mixed_stream_matches_alone(fm, monkeypatch):
    # (without batching: every request runs on its own tree, as alone)
    monkeypatch.setenv("FMM2D_B200_SERVE_BATCH", "0")
    specs = [("l", 20000, 1e-6, 0), ("h", 8000, 1e-6, 1), ("c", 15000, 1e-9, 0),
             ("l", 3000, 1e-3, 1), ("h", 30000, 1e-9, 0), ("l", 60000, 1e-9, 1),
             ("c", 1000, 1e-3, 1), ("h", 2000, 1e-6, 1)] * 3
    # alone: one request at a time through a single-slot server
    alone = []
    srv1 = fm.Server(slots=1, hbm_budget=100e9)
    for i, (k, n, eps, pgt) in enumerate(specs):
        r, keep = _req(fm, k, n, 100 + i, eps=eps, zk=3.0 + i, pgt=pgt)
        t = srv1.submit(r, keep)
        ier, _ = srv1.wait(t)
        assert ier == 0
        alone.append(keep)
    srv1.close()
    # mixed: everything submitted at once into 6 slots and a budget that
    # admits only part of the stream at a time
    budget = 3e9
    srv = fm.Server(slots=6, hbm_budget=budget)
    tickets = []
    for i, (k, n, eps, pgt) in enumerate(specs):
        r, keep = _req(fm, k, n, 100 + i, eps=eps, zk=3.0 + i, pgt=pgt)
        tickets.append((srv.submit(r, keep), keep))
    for (t, keep), ref in zip(tickets, alone):
        ier, _ = srv.wait(t)
        assert ier == 0
        for key in ref:
            if key.startswith(("pot", "grad")):
                assert W.rel_err(keep[key], ref[key]) <= 1e-14, key
    st = srv.stats()
    assert st["peak_bytes"] <= budget
    assert st["peak_running"] >= 2
    srv.close()


@pytest.mark.gpu
def test_concurrent_orders_all_succeed(fm):
    # Requests of different expansion orders run the same kernels with
    # different shared-memory sizes on concurrent worker threads; every one
    # of them must launch (a kernel's shared-memory limit is only raised,
    # never lowered under another thread's launch).
    srv = fm.Server(slots=8, hbm_budget=100e9)
    tickets = []
    for i in range(96):
        eps = (1e-3, 1e-6, 1e-9, 1e-12)[i % 4]
        kern = "lch"[i % 3]
        r, keep = _req(fm, kern, 2000 + 97 * i, 500 + i, eps=eps, zk=2.0 + i % 7, pgt=i % 2)
        tickets.append(srv.submit(r, keep))
    iers = [srv.wait(t)[0] for t in tickets]
    srv.close()
    assert iers == [0] * len(iers), fm.last_error()


@pytest.mark.gpu
def test_batched_stream_matches_alone(fm, monkeypatch):
    """Small lfmm2d requests queued together run in batches (one forest per
    batch); each result agrees with the request run alone to its eps."""
    monkeypatch.delenv("FMM2D_B200_SERVE_BATCH", raising=False)
    specs = [(500 + 331 * i, 1e-6 if i % 2 else 1e-9, i % 3 == 0) for i in range(40)]
    alone = []
    for i, (n, eps, pgt) in enumerate(specs):
        r, keep = _req(fm, "l", n, 700 + i, eps=eps, pgt=int(pgt))
        srv1 = fm.Server(slots=1, hbm_budget=100e9)
        t = srv1.submit(r, keep)
        assert srv1.wait(t)[0] == 0
        srv1.close()
        alone.append((keep, eps))
    srv = fm.Server(slots=2, hbm_budget=100e9)
    tickets = []
    for i, (n, eps, pgt) in enumerate(specs):
        r, keep = _req(fm, "l", n, 700 + i, eps=eps, pgt=int(pgt))
        tickets.append((srv.submit(r, keep), keep))
    for (t, keep), (ref, eps) in zip(tickets, alone):
        assert srv.wait(t)[0] == 0
        for key in ref:
            if key.startswith(("pot", "grad")):
                assert W.rel_err(keep[key], ref[key]) <= max(2 * eps, 1e-12), key
    assert srv.stats()["batched"] >= 2
    srv.close()


@pytest.mark.gpu
def test_batch_across_eps_of_one_arithmetic(fm, monkeypatch):
    """Mixed-mode requests at eps 1e-3 and 1e-6 batch together and run at
    1e-6; each result is within its own eps of its alone run."""
    monkeypatch.delenv("FMM2D_B200_SERVE_BATCH", raising=False)
    specs = [(800 + 97 * i, 1e-3 if i % 2 else 1e-6) for i in range(24)]
    alone = []
    for i, (n, eps) in enumerate(specs):
        r, keep = _req(fm, "l", n, 900 + i, eps=eps)
        srv1 = fm.Server(slots=1, hbm_budget=100e9)
        t = srv1.submit(r, keep)
        assert srv1.wait(t)[0] == 0
        srv1.close()
        alone.append((keep, eps))
    srv = fm.Server(slots=1, hbm_budget=100e9)
    tickets = []
    for i, (n, eps) in enumerate(specs):
        r, keep = _req(fm, "l", n, 900 + i, eps=eps)
        tickets.append((srv.submit(r, keep), keep))
    for (t, keep), (ref, eps) in zip(tickets, alone):
        assert srv.wait(t)[0] == 0
        for key in ref:
            if key.startswith(("pot", "grad")):
                assert W.rel_err(keep[key], ref[key]) <= 2 * eps, key
    assert srv.stats()["batched"] >= 4
    srv.close()
