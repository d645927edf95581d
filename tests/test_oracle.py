"""The oracle (oracle/fmm2d_oracle.c) is pinned against the reference's own
direct kernels and rules, compiled from the reference sources into
oracle/_ref/ (lapkernels2d.c:19-494, cauchykernels2d.c:31-442,
l2dterms.c:26-67, hndiv2d.c:15-48)."""
import ctypes

import numpy as np
import pytest

import refimpl
import wrappers as W

pytestmark = pytest.mark.skipif(not refimpl.have_ref(),
                                reason="reference build absent")
I = lambda v: ctypes.byref(ctypes.c_int(v))
D = lambda v: ctypes.byref(ctypes.c_double(v))


def data(ns, nt, seed):
    rng = np.random.default_rng(seed)
    src = rng.random((2, ns))
    trg = np.concatenate([rng.random((2, nt - 3)), src[:, :3]], axis=1)  # coincident
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    v = rng.standard_normal((2, ns))
    return src, trg, q, d, v


@pytest.mark.parametrize("cd", ["c", "d", "cd"])
@pytest.mark.parametrize("pgh", [1, 2, 3])
def test_l2d_direct_matches_reference(cd, pgh):
    ns, nt = 300, 120
    src, trg, q, d, v = data(ns, nt, 1)
    thr = 1e-14
    name = f"l2d_direct{cd}{'pgh'[pgh - 1]}_"
    outs = [np.zeros(nt, complex), np.zeros((nt, 2), complex), np.zeros((nt, 3), complex)]
    args = [I(1), W._p(np.asfortranarray(src)), I(ns)]
    if "c" in cd:
        args.append(W._p(q))
    if "d" in cd:
        args += [W._p(d), W._p(np.asfortranarray(v))]
    args += [W._p(np.asfortranarray(trg)), I(nt)] + [W._p(o) for o in outs[:pgh]] + [D(thr)]
    getattr(refimpl.ref(), name)(*args)
    mine = [np.zeros(nt, complex), np.zeros((nt, 2), complex), np.zeros((nt, 3), complex)]
    refimpl.orc().oracle_l2d_direct(
        ns, W._p(np.ascontiguousarray(src.T)), int("c" in cd), W._p(q),
        int("d" in cd), W._p(d), W._p(np.ascontiguousarray(v.T)), 0, nt,
        W._p(np.ascontiguousarray(trg.T)), pgh, W._p(mine[0]), W._p(mine[1]),
        W._p(mine[2]), thr)
    for a, b in zip(mine[:pgh], outs[:pgh]):
        assert W.rel_err(a, b) < 1e-13


@pytest.mark.parametrize("cd", ["c", "d", "cd"])
@pytest.mark.parametrize("pgh", [1, 2, 3])
def test_c2d_direct_matches_reference(cd, pgh):
    ns, nt = 300, 120
    src, trg, q, d, v = data(ns, nt, 2)
    thr = 1e-14
    name = f"c2d_direct{cd}{'pgh'[pgh - 1]}_"
    outs = [np.zeros(nt, complex) for _ in range(3)]
    args = [I(1), W._p(np.asfortranarray(src)), I(ns)]
    if "c" in cd:
        args.append(W._p(q))
    if "d" in cd:
        args.append(W._p(d))
    args += [W._p(np.asfortranarray(trg)), I(nt)] + [W._p(o) for o in outs[:pgh]] + [D(thr)]
    getattr(refimpl.ref(), name)(*args)
    mine = [np.zeros(nt, complex) for _ in range(3)]
    refimpl.orc().oracle_c2d_direct(
        ns, W._p(np.ascontiguousarray(src.T)), int("c" in cd), W._p(q),
        int("d" in cd), W._p(d), 0, nt, W._p(np.ascontiguousarray(trg.T)), pgh,
        W._p(mine[0]), W._p(mine[1]), W._p(mine[2]), thr)
    for a, b in zip(mine[:pgh], outs[:pgh]):
        assert W.rel_err(a, b) < 1e-13


def test_rules_match_reference():
    O, R = refimpl.orc(), refimpl.ref()
    for eps in 10.0 ** -np.linspace(0.5, 15.5, 151):
        nt, ier = ctypes.c_int(0), ctypes.c_int(0)
        R.l2dterms_(D(eps), ctypes.byref(nt), ctypes.byref(ier))
        assert O.oracle_l2dterms(eps) == nt.value
        nd, idf = ctypes.c_int(0), ctypes.c_int(0)
        R.hndiv2d_(D(eps), I(10), I(5), I(1), I(0), I(1), I(0),
                   ctypes.byref(nd), ctypes.byref(idf))
        assert O.oracle_lndiv2d(eps, 10, 5) == nd.value


@pytest.mark.parametrize("zk", [10.0 + 0j, 0.5 + 0.1j, 80.0 + 0j, 3.0 + 6.0j])
@pytest.mark.parametrize("cd", ["c", "d", "cd"])
@pytest.mark.parametrize("pgh", [1, 2, 3])
def test_h2d_direct_matches_reference(zk, cd, pgh):
    ns, nt = 200, 90
    src, trg, q, d, v = data(ns, nt, 2)
    thr = abs(zk) * 2.0 ** -51
    ifc, ifd = int("c" in cd), int("d" in cd)
    O = refimpl.orc()
    O.oracle_h2d_direct.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_double]
    mine = [np.zeros(nt, complex), np.zeros((nt, 2), complex), np.zeros((nt, 3), complex)]
    O.oracle_h2d_direct(zk.real, zk.imag, ns, W._p(np.asfortranarray(src)), ifc, W._p(q), ifd,
                        W._p(d), W._p(np.asfortranarray(v)), nt, W._p(np.asfortranarray(trg)),
                        pgh, W._p(mine[0]), W._p(mine[1]), W._p(mine[2]), thr)
    outs = [np.zeros(nt, complex), np.zeros((nt, 2), complex), np.zeros((nt, 3), complex)]
    zka = np.array([zk])
    args = [I(1), W._p(zka), W._p(np.asfortranarray(src)), I(ns)]
    if ifc:
        args.append(W._p(q))
    if ifd:
        args += [W._p(d), W._p(np.asfortranarray(v))]
    args += [W._p(np.asfortranarray(trg)), I(nt)] + [W._p(o) for o in outs[:pgh]] + [D(thr)]
    getattr(refimpl.ref(), f"h2d_direct{cd}{'pgh'[pgh - 1]}_")(*args)
    for k in range(pgh):
        assert W.rel_err(mine[k], outs[k]) < 1e-13, (k, W.rel_err(mine[k], outs[k]))


def test_oracle_hankel_matches_hank103():
    rng = np.random.default_rng(5)
    r = np.exp(rng.uniform(np.log(1e-6), np.log(1e3), 3000))
    a = rng.uniform(-np.pi / 2, np.pi, 3000)
    z = np.ascontiguousarray(r * np.exp(1j * a))
    out = np.zeros(4 * len(z))
    O = refimpl.orc()
    O.oracle_hankel01.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    O.oracle_hankel01(len(z), W._p(z), W._p(out))
    h0 = out[0::4] + 1j * out[1::4]
    one = ctypes.c_int(1)
    worst = 0.0
    for k in range(len(z)):
        zz = np.array([z[k]])
        a0 = np.zeros(1, complex)
        a1 = np.zeros(1, complex)
        refimpl.ref().hank103_(W._p(zz), W._p(a0), W._p(a1), ctypes.byref(one))
        if np.isfinite(a0[0]) and 1e-290 < abs(a0[0]) < 1e290:
            worst = max(worst, abs(h0[k] - a0[0]) / abs(a0[0]))
    assert worst < 2e-14
