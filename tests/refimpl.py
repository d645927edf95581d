"""ctypes access to the checkers under oracle/_ref/ (test infrastructure).

* ``oracle/_ref/libfmm2d_ref.so``: the reference's own C translation,
  compiled unmodified by ``oracle/Makefile`` (plus the Fortran-only driver
  pieces restated in ``oracle/ref_harness.c``).
* ``oracle/_ref/liboracle.so``: ``oracle/fmm2d_oracle.c``, independent FP64
  direct sums.

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU baseline use
this module.
"""
import ctypes
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(REPO, "oracle", "_ref", "libfmm2d_ref.so")
ORACLE_SO = os.path.join(REPO, "oracle", "_ref", "liboracle.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_ref = None
_orc = None


def have_ref():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO, mode=os.RTLD_LOCAL | os.RTLD_NOW)
    return _ref


def orc():
    global _orc
    if _orc is None:
        _orc = ctypes.CDLL(ORACLE_SO, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        _orc.oracle_l2d_direct.argtypes = [_I, _P, _I, _P, _I, _P, _P, _I, _I,
                                           _P, _I, _P, _P, _P, ctypes.c_double]
        _orc.oracle_c2d_direct.argtypes = [_I, _P, _I, _P, _I, _P, _I, _I, _P,
                                           _I, _P, _P, _P, ctypes.c_double]
        _orc.oracle_lndiv2d.argtypes = [ctypes.c_double, _I, _I]
        _orc.oracle_l2dterms.argtypes = [ctypes.c_double]
    return _orc


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def _ri(v):
    return ctypes.byref(_I(v))


def ref_tree(sources, targets=None, ndiv=15, idivflag=0, lists=True):
    """The reference's pts_tree_mem / pts_tree_build / pts_tree_sort /
    computelists on the same inputs, in the same dict layout as
    fmm2d_c_translation_b200.tree_build."""
    R = ref()
    src = np.asfortranarray(np.asarray(sources, np.float64))
    ns = src.shape[1]
    trg = (np.zeros((2, 1)) if targets is None
           else np.asfortranarray(np.asarray(targets, np.float64)))
    nt = 0 if targets is None else trg.shape[1]
    nlevels, nboxes, ltree = _I(), _I(), _I()
    nlmin, nlmax, ifunif, iper = _I(0), _I(51), _I(0), _I(0)
    R.pts_tree_mem_(_p(src), _ri(ns), _p(trg), _ri(nt), _ri(idivflag),
                    _ri(ndiv), ctypes.byref(nlmin), ctypes.byref(nlmax),
                    ctypes.byref(ifunif), ctypes.byref(iper),
                    ctypes.byref(nlevels), ctypes.byref(nboxes),
                    ctypes.byref(ltree))
    nl, nb, lt = nlevels.value, nboxes.value, ltree.value
    itree = np.zeros(lt, np.int32)
    iptr = np.zeros(8, np.int32)
    centers = np.zeros((2, nb), order="F")
    boxsize = np.zeros(nl + 1)
    R.pts_tree_build_(_p(src), _ri(ns), _p(trg), _ri(nt), _ri(idivflag),
                      _ri(ndiv), ctypes.byref(nlmin), ctypes.byref(nlmax),
                      ctypes.byref(ifunif), ctypes.byref(iper),
                      ctypes.byref(nlevels), _ri(nb), _ri(lt), _p(itree),
                      _p(iptr), _p(centers), _p(boxsize))
    isrc = np.zeros(max(ns, 1), np.int32)
    isrcse = np.zeros((2, nb), np.int32, order="F")
    itarg = np.zeros(max(nt, 1), np.int32)
    itargse = np.zeros((2, nb), np.int32, order="F")
    R.pts_tree_sort_(_ri(ns), _p(src), _p(itree), _ri(lt), _ri(nb), _ri(nl),
                     _p(iptr), _p(centers), _p(isrc), _p(isrcse))
    R.pts_tree_sort_(_ri(nt), _p(trg), _p(itree), _ri(lt), _ri(nb), _ri(nl),
                     _p(iptr), _p(centers), _p(itarg), _p(itargse))
    out = dict(nlevels=nl, nboxes=nb, ltree=lt, itree=itree, iptr=iptr,
               centers=np.ascontiguousarray(centers), boxsize=boxsize,
               isrc=isrc[:ns], isrcse=np.ascontiguousarray(isrcse),
               itarg=itarg[:nt], itargse=np.ascontiguousarray(itargse))
    if lists:
        mn = [_I() for _ in range(4)]
        R.computemnlists_(_ri(nl), _ri(nb), _p(itree), _ri(lt), _p(iptr),
                          _p(centers), _p(boxsize), ctypes.byref(iper),
                          *[ctypes.byref(m) for m in mn])
        arrs = []
        for k, m in enumerate(mn):
            n_k = np.zeros(nb, np.int32)
            l_k = np.zeros((nb, m.value), np.int32)
            out[f"nlist{k + 1}"] = n_k
            out[f"list{k + 1}"] = l_k
            arrs += [ctypes.byref(m), _p(n_k), _p(l_k)]
        R.computelists_(_ri(nl), _ri(nb), _p(itree), _ri(lt), _p(iptr),
                        _p(centers), _p(boxsize), ctypes.byref(iper), *arrs)
        for k in range(1, 5):
            n_k, l_k = out[f"nlist{k}"], out[f"list{k}"]
            mask = np.arange(l_k.shape[1])[None, :] < n_k[:, None]
            out[f"list{k}"] = np.where(mask, l_k, 0)
    return out
