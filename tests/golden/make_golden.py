"""Generates the golden fixtures in this directory from the reference's own
C translation (oracle/_ref/libfmm2d_ref.so, built by oracle/Makefile from
the reference sources).  Run from the repository root:

    python tests/golden/make_golden.py

Fixtures (seeded inputs, the reference's test sizes ns = 200, nt = 100,
eps = 1e-6, as in c_translation/test/test_lfmm2d_ndiv.f:25,49):
  tree_200_100.npz      pts_tree_build / pts_tree_sort / computelists output
  fmm_<fam>_<variant>.npz  inputs and outputs of lfmm2d_st_* and cfmm2d_st_*
  fmm_h1_<variant>.npz, fmm_h2_<variant>.npz  hfmm2d_st_* with zk = 10 and
      zk = 0.5 + 0.1i (the values of test/helmholtz/test_hfmm2d.f:48-49),
      eps = 0.51e-8 (:51)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import refimpl  # noqa: E402
import wrappers as W  # noqa: E402


def inputs(seed=2024, ns=200, nt=100):
    rng = np.random.default_rng(seed)
    src = rng.random((2, ns))
    trg = rng.random((2, nt))
    q = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    d = rng.standard_normal(ns) + 1j * rng.standard_normal(ns)
    th = rng.uniform(0, 2 * np.pi, ns)
    v = np.stack([np.cos(th), np.sin(th)])
    return src, trg, q, d, v


def main():
    src, trg, q, d, v = inputs()
    t = refimpl.ref_tree(src, trg, ndiv=15, idivflag=0)
    np.savez_compressed(os.path.join(HERE, "tree_200_100.npz"), src=src, trg=trg,
                        **{k: np.asarray(x) for k, x in t.items()})
    for fam in ("l", "c"):
        for cd in ("c", "d", "cd"):
            for p in "pgh":
                var = f"st_{cd}_{p}"
                out, ier = W.call(refimpl.ref(), fam, var, 1e-6, src, q, d, v, trg)
                assert ier == 0
                np.savez_compressed(os.path.join(HERE, f"fmm_{fam}_{var}.npz"),
                                    src=src, trg=trg, charge=q, dipstr=d,
                                    dipvec=v, eps=1e-6, **out)
    for tag, zk in (("h1", 10.0 + 0j), ("h2", 0.5 + 0.1j)):
        for cd in ("c", "d", "cd"):
            for p in "pgh":
                var = f"st_{cd}_{p}"
                out, ier = W.call(refimpl.ref(), "h", var, 0.51e-8, src, q, d, v, trg, zk=zk)
                assert ier == 0
                np.savez_compressed(os.path.join(HERE, f"fmm_{tag}_{var}.npz"),
                                    src=src, trg=trg, charge=q, dipstr=d, dipvec=v,
                                    eps=0.51e-8, zk=zk, family="h", **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
