"""The GPU library reproduces the golden outputs of the reference (tests/
golden/, no reference build needed): the quadtree bit for bit, the FMM
outputs to 1e-11 in all-FP64 mode (Laplace, Cauchy) and to 1e-10 (Helmholtz,
whose Bessel and Hankel values come from different algorithms)."""
import glob
import os

import numpy as np
import pytest

import wrappers as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(GOLD, "fmm_*.npz")))


@pytest.fixture(scope="module")
def glib():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    L.fmm2d_b200_set_precision(1)
    yield L
    L.fmm2d_b200_set_precision(0)


def test_tree_golden():
    import fmm2d_c_translation_b200 as fm
    g = np.load(os.path.join(GOLD, "tree_200_100.npz"))
    t = fm.tree_build(g["src"], g["trg"], ndiv=15, idivflag=0)
    for k in ("itree", "iptr", "centers", "boxsize", "isrc", "isrcse", "itarg",
              "itargse"):
        np.testing.assert_array_equal(t[k], g[k], err_msg=k)
    for k in (1, 2, 3, 4):
        np.testing.assert_array_equal(t[f"nlist{k}"], g[f"nlist{k}"])
        m = min(t[f"list{k}"].shape[1], g[f"list{k}"].shape[1])
        np.testing.assert_array_equal(t[f"list{k}"][:, :m], g[f"list{k}"][:, :m])


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_fmm_golden(glib, path):
    name = os.path.basename(path)[4:-4]
    fam, variant = name.split("_", 1)
    g = np.load(path)
    zk = None
    if "family" in g.files:  # Helmholtz fixtures carry their wavenumber
        fam, zk = str(g["family"]), complex(g["zk"])
    out, ier = W.call(glib, fam, variant, float(g["eps"]), g["src"], g["charge"],
                      g["dipstr"], g["dipvec"], g["trg"], zk=zk)
    assert ier == 0
    tol = 1e-10 if zk is not None else 1e-11
    for k in out:
        assert W.rel_err(out[k], g[k]) < tol, (name, k)
