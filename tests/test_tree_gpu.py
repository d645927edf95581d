"""The device-built quadtree is bit-identical to the reference's
(pts_tree_mem/pts_tree_build/pts_tree_sort/computelists,
src/common/pts_tree2d.f, src/common/tree_routs2d.f) on the same inputs:
box arrays, centers, box sizes, point permutations and ranges; the
interaction lists hold the same boxes in the same order."""
import numpy as np
import pytest

import pointsets as ps
import refimpl

pytestmark = pytest.mark.gpu

CASES = {
    "uniform_200_100": lambda: (ps.uniform(200, 1), ps.uniform(100, 2), 15, 0),
    "uniform_20000": lambda: (ps.uniform(20000, 3), None, 15, 0),
    "blobs_30000_8000": lambda: (ps.blobs(30000, 4), ps.blobs(8000, 5), 10, 0),
    "starfish_20000": lambda: (ps.starfish(20000, 0)[0],
                               ps.near_curve_targets(20000, 6), 20, 0),
    "grid_lines_65": lambda: (ps.grid_lines(64), ps.grid_lines(32), 8, 0),
    "duplicates_deep": lambda: (ps.with_duplicates(1000, 7, 40), None, 15, 0),
    "single_box": lambda: (ps.uniform(10, 8), ps.uniform(5, 9), 15, 0),
    "targets_rule": lambda: (ps.uniform(3000, 10), ps.blobs(6000, 11), 12, 1),
    "max_rule": lambda: (ps.blobs(3000, 12), ps.uniform(6000, 13), 12, 2),
    # deeper than the first guess of the key depth (20+ levels)
    "tight_blobs": lambda: (ps.blobs(20000, 14, nblob=4, sigma=1e-6),
                            ps.blobs(5000, 15, nblob=4, sigma=1e-5), 10, 0),
    # enough points per set for the multi-block sort passes
    "uniform_300000": lambda: (ps.uniform(300000, 16), ps.uniform(200000, 17), 24, 0),
    # target leaves of 33..256 points (shared-memory leaf sort) and of more
    # than 256 points (the global sort)
    "targets_per_leaf_40": lambda: (ps.uniform(20000, 18), ps.uniform(100000, 19), 15, 0),
    "targets_per_leaf_1000": lambda: (ps.uniform(1000, 20), ps.uniform(150000, 21), 15, 0),
}


@pytest.fixture(params=["keys", "keys_sync", "levelwise"])
def builder(request, monkeypatch):
    """keys: path keys with the refinement counts of every level taken from
    the sorted keys (one host synchronisation); keys_sync: path keys with a
    synchronisation per level; levelwise: the reference's level-by-level
    point partition."""
    monkeypatch.delenv("FMM2D_B200_TREE_SYNC", raising=False)
    if request.param == "levelwise":
        monkeypatch.setenv("FMM2D_B200_TREE", "levelwise")
    else:
        monkeypatch.delenv("FMM2D_B200_TREE", raising=False)
        if request.param == "keys_sync":
            monkeypatch.setenv("FMM2D_B200_TREE_SYNC", "1")
    return request.param


@pytest.mark.parametrize("name", sorted(CASES))
def test_tree_bit_exact(name, builder):
    import fmm2d_c_translation_b200 as fm
    src, trg, ndiv, idiv = CASES[name]()
    got = fm.tree_build(src, trg, ndiv=ndiv, idivflag=idiv)
    want = refimpl.ref_tree(src, trg, ndiv=ndiv, idivflag=idiv)
    for k in ("nlevels", "nboxes", "ltree"):
        assert got[k] == want[k], k
    for k in ("iptr", "itree", "centers", "boxsize", "isrc", "isrcse",
              "itarg", "itargse"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    for k in (1, 2, 3, 4):
        np.testing.assert_array_equal(got[f"nlist{k}"], want[f"nlist{k}"],
                                      err_msg=f"nlist{k}")
        m = min(got[f"list{k}"].shape[1], want[f"list{k}"].shape[1])
        np.testing.assert_array_equal(got[f"list{k}"][:, :m],
                                      want[f"list{k}"][:, :m],
                                      err_msg=f"list{k}")
