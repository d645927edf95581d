"""The C-ABI library: it loads without a GPU, exports every entry point
include/fmm2d_b200.h declares, and its host-side rules (expansion order,
leaf capacity) agree with the reference's l2dterms / hndiv2d."""
import ctypes
import os
import re

import numpy as np
import pytest

import refimpl

REPO = refimpl.REPO
HEADER = os.path.join(REPO, "include", "fmm2d_b200.h")


def declared_names():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(\w+)\s*\(", txt)) - {"if", "defined"})


def test_header_declares_the_reference_surface():
    names = declared_names()
    for fam in "lchr":
        for st in ("s", "t", "st"):
            for cd in ("c", "d", "cd"):
                for p in "pgh":
                    assert f"{fam}fmm2d_{st}_{cd}_{p}_" in names
                    assert f"{fam}fmm2d_{st}_{cd}_{p}_vec_" in names
    for g in ("lfmm2d_", "cfmm2d_", "hfmm2d_", "rfmm2d_", "lfmm2d_ndiv_", "cfmm2d_ndiv_",
              "hfmm2d_ndiv_", "rfmm2d_ndiv_"):
        assert g in names


def test_library_exports_every_declared_symbol():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    missing = [n for n in declared_names() if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_no_device_error_path():
    import fmm2d_c_translation_b200 as fm
    assert fm.lib().fmm2d_b200_version().startswith(b"fmm2d-b200")


@pytest.mark.skipif(not refimpl.have_ref(), reason="reference build absent")
def test_nterms_matches_reference_l2dterms():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    R = refimpl.ref()
    for eps in np.concatenate([10.0 ** -np.linspace(0.5, 15.5, 301),
                               [1e-3, 1e-6, 1e-9, 1e-12, 0.5e-6]]):
        nt, ier = ctypes.c_int(0), ctypes.c_int(0)
        R.l2dterms_(ctypes.byref(ctypes.c_double(eps)), ctypes.byref(nt),
                    ctypes.byref(ier))
        assert L.fmm2d_b200_laplace_nterms(ctypes.c_double(eps)) == nt.value, eps


@pytest.mark.skipif(not refimpl.have_ref(), reason="reference build absent")
def test_leaf_capacity_matches_reference_hndiv2d():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    R = refimpl.ref()
    I = lambda v: ctypes.byref(ctypes.c_int(v))
    for eps in [0.9, 0.5, 0.1, 0.05, 1e-2, 5e-3, 1e-3, 5e-4, 1e-6, 5e-7,
                1e-9, 5e-10, 1e-12, 5e-13, 1e-15, 5e-16, 1e-17]:
        nd, idf = ctypes.c_int(0), ctypes.c_int(0)
        R.hndiv2d_(ctypes.byref(ctypes.c_double(eps)), I(100), I(50), I(1),
                   I(0), I(1), I(0), ctypes.byref(nd), ctypes.byref(idf))
        assert L.fmm2d_b200_leaf_capacity(ctypes.c_double(eps), 100, 50) == nd.value
        assert idf.value == 0


def _direct_argtypes(L):
    base = ([ctypes.c_int] * 2 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
            + [ctypes.c_void_p] * 3 + [ctypes.c_double])
    L.fmm2d_b200_l2d_direct.argtypes = base
    L.fmm2d_b200_l2d_direct_noalloc.argtypes = base + [ctypes.c_void_p]


@pytest.mark.parametrize("missing", ["charge", "dipstr", "dipvec", "grad", "hess",
                                     "sources", "targ", "pot"])
@pytest.mark.parametrize("entry", ["l2d_direct", "l2d_direct_noalloc"])
def test_direct_refuses_null_required_arrays(entry, missing):
    """A NULL array that the flags require is refused with ier = 4 on the
    host, before any device work (no GPU is touched)."""
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    _direct_argtypes(L)
    ns, nt = 10, 5
    a = {k: np.zeros(n) for k, n in [("sources", 2 * ns), ("charge", 2 * ns),
                                      ("dipstr", 2 * ns), ("dipvec", 2 * ns),
                                      ("targ", 2 * nt), ("pot", 2 * nt),
                                      ("grad", 4 * nt), ("hess", 6 * nt)]}
    P = {k: (None if k == missing else v.ctypes.data_as(ctypes.c_void_p))
         for k, v in a.items()}
    args = [1, ns, P["sources"], 1, P["charge"], 1, P["dipstr"], P["dipvec"], nt,
            P["targ"], 3, P["pot"], P["grad"], P["hess"], 1e-14]
    if entry.endswith("noalloc"):
        args.append(None)
    ier = getattr(L, "fmm2d_b200_" + entry)(*args)
    assert ier == 4
    assert missing in fm.last_error() and "NULL" in fm.last_error()
