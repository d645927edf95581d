"""fmm2d_c_translation_b200 -- B200-native evaluation path of fmm2d.

The product is the C-ABI shared library ``libfmm2d_b200.so`` built from
``csrc/``: it exports the reference's gfortran-convention entry points
(``lfmm2d_*``, ``cfmm2d_*``, ``hfmm2d_*``, the guru drivers and the
``*_ndiv`` variants), so C, Fortran and MATLAB callers link it in place of
the reference library.  This module is the Python host layer over that
library: it loads it with ctypes and mirrors the reference's Python
interface (``python/fmm2dpy/fmm2d.py``: ``lfmm2d``, ``cfmm2d``, ``hfmm2d``
with the same keyword arguments, array shapes and ``Output`` fields).

There is no CPU fallback: if the library is missing or no CUDA device is
present, every call raises.
"""
import ctypes
import os

import numpy as np

__all__ = ["Output", "lfmm2d", "cfmm2d", "hfmm2d", "lib", "lib_path",
           "last_error", "tree_build", "FmmError"]

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
lib_path = os.path.join(_PKG_DIR, "libfmm2d_b200.so")
_lib = None


class FmmError(RuntimeError):
    """Raised when an entry point returns a nonzero ``ier``."""


def lib():
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(lib_path):
            raise ImportError(
                "libfmm2d_b200.so is not built; run "
                "`python -m fmm2d_c_translation_b200.build` (needs nvcc)")
        # RTLD_LOCAL: the reference library exports the same symbol names.
        _lib = ctypes.CDLL(lib_path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        _declare(_lib)
    return _lib


_P = ctypes.c_void_p
_I = ctypes.c_int


def _declare(L):
    L.fmm2d_b200_version.restype = ctypes.c_char_p
    L.fmm2d_b200_last_error.argtypes = [ctypes.c_char_p, _I]
    L.fmm2d_b200_tree_build.argtypes = [_P, _I, _P, _I, _I, _I,
                                        ctypes.POINTER(_P)]
    L.fmm2d_b200_tree_sizes.argtypes = [_P, _P, _P, _P]
    L.fmm2d_b200_tree_export.argtypes = [_P] * 9
    L.fmm2d_b200_tree_lists.argtypes = [_P] * 9
    L.fmm2d_b200_tree_free.argtypes = [_P]
    L.fmm2d_b200_tree_free.restype = None


def last_error():
    buf = ctypes.create_string_buffer(2048)
    lib().fmm2d_b200_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def _check(ier, what):
    if ier != 0:
        raise FmmError(f"{what} failed (ier={ier}): {last_error()}")


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


class Output:
    """Results of one evaluation (fields as in fmm2dpy.Output)."""
    pot = None
    grad = None
    hess = None
    pottarg = None
    gradtarg = None
    hesstarg = None
    ier = 0


def tree_build(sources, targets=None, ndiv=15, idivflag=0, lists=True):
    """Builds the quadtree on the GPU and returns it in the reference's
    layout (1-based, as pts_tree_build / pts_tree_sort / computelists
    produce): dict with nlevels, nboxes, ltree, itree, iptr, centers(2,nb),
    boxsize, isrc, isrcse(2,nb), itarg, itargse and, with lists=True,
    nlist1..4 / list1..4 (list_k(mnlist_k, nboxes), zero-padded)."""
    L = lib()
    src = np.ascontiguousarray(np.asarray(sources, dtype=np.float64).T)
    ns = src.shape[0]
    if targets is None:
        trg = np.zeros((0, 2))
    else:
        trg = np.ascontiguousarray(np.asarray(targets, dtype=np.float64).T)
    nt = trg.shape[0]
    h = _P()
    _check(L.fmm2d_b200_tree_build(_ptr(src), ns, _ptr(trg) if nt else None,
                                   nt, ndiv, idivflag, ctypes.byref(h)),
           "tree_build")
    try:
        nl, nb, lt = _I(), _I(), _I()
        L.fmm2d_b200_tree_sizes(h, ctypes.byref(nl), ctypes.byref(nb),
                                ctypes.byref(lt))
        nl, nb, lt = nl.value, nb.value, lt.value
        out = dict(nlevels=nl, nboxes=nb, ltree=lt,
                   itree=np.zeros(lt, np.int32), iptr=np.zeros(8, np.int32),
                   centers=np.zeros((nb, 2)), boxsize=np.zeros(nl + 1),
                   isrc=np.zeros(max(ns, 1), np.int32),
                   isrcse=np.zeros((nb, 2), np.int32),
                   itarg=np.zeros(max(nt, 1), np.int32),
                   itargse=np.zeros((nb, 2), np.int32))
        _check(L.fmm2d_b200_tree_export(
            h, _ptr(out["itree"]), _ptr(out["iptr"]), _ptr(out["centers"]),
            _ptr(out["boxsize"]), _ptr(out["isrc"]), _ptr(out["isrcse"]),
            _ptr(out["itarg"]), _ptr(out["itargse"])), "tree_export")
        out["isrc"] = out["isrc"][:ns]
        out["itarg"] = out["itarg"][:nt]
        out["centers"] = out["centers"].T.copy()
        out["isrcse"] = out["isrcse"].T.copy()
        out["itargse"] = out["itargse"].T.copy()
        if lists:
            for k, m in ((1, 13), (2, 27), (3, 20), (4, 5)):
                out[f"nlist{k}"] = np.zeros(nb, np.int32)
                out[f"list{k}"] = np.zeros((nb, m), np.int32)
            _check(L.fmm2d_b200_tree_lists(
                h, *[_ptr(out[f"{p}{k}"]) for k in (1, 2, 3, 4)
                     for p in ("nlist", "list")]), "tree_lists")
        return out
    finally:
        L.fmm2d_b200_tree_free(h)
