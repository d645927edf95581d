"""Host-side Helmholtz rules and special functions (no GPU needed):

* H0, H1 of the library's Hankel routine against the reference's hank103
  (c_translation/src/hank103.c:66) over the complex plane;
* the scaled sequences (h2dall, jbessel2d) the translation tables are
  built from, against the reference's own routines;
* the expansion order rule h2dterms (c_translation/src/h2dterms.c:19)
  for the wavenumbers of the reference tests and more.
"""
import ctypes

import numpy as np
import pytest

import refimpl

_P = ctypes.c_void_p


def _p(a):
    return a.ctypes.data_as(_P)


@pytest.fixture(scope="module")
def lib():
    import fmm2d_c_translation_b200 as fm
    L = fm.lib()
    L.fmm2d_b200_helm_nterms.restype = ctypes.c_int
    L.fmm2d_b200_helm_nterms.argtypes = [ctypes.c_double] * 4
    L.fmm2d_b200_helm_hvec.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, _P]
    L.fmm2d_b200_helm_jvec.argtypes = L.fmm2d_b200_helm_hvec.argtypes
    return L


needs_ref = pytest.mark.skipif(not refimpl.have_ref(), reason="reference build absent")


def _hankel(lib, z):
    z = np.ascontiguousarray(z, np.complex128)
    out = np.zeros(4 * len(z))
    lib.fmm2d_b200_hankel01(ctypes.c_int(len(z)), _p(z), _p(out))
    return out[0::4] + 1j * out[1::4], out[2::4] + 1j * out[3::4]


@needs_ref
def test_hankel01_vs_hank103(lib):
    rng = np.random.default_rng(0)
    r = np.exp(rng.uniform(np.log(1e-6), np.log(2e3), 4000))
    a = rng.uniform(-np.pi / 2, np.pi, 4000)
    z = np.concatenate([r * np.exp(1j * a), np.exp(np.linspace(-12, 8, 500)) + 0j])
    h0, h1 = _hankel(lib, z)
    R = refimpl.ref()
    one = ctypes.c_int(1)
    r0 = np.zeros(len(z), complex)
    r1 = np.zeros(len(z), complex)
    for k in range(len(z)):
        zz = np.array([z[k]])
        a0 = np.zeros(1, complex)
        a1 = np.zeros(1, complex)
        R.hank103_(_p(zz), _p(a0), _p(a1), ctypes.byref(one))
        r0[k], r1[k] = a0[0], a1[0]
    ok = np.isfinite(r0) & (np.abs(r0) > 1e-290) & (np.abs(r0) < 1e290)
    assert ok.sum() > 4000
    e0 = np.abs(h0 - r0)[ok] / np.abs(r0)[ok]
    e1 = np.abs(h1 - r1)[ok] / np.abs(r1)[ok]
    assert e0.max() < 2e-14 and e1.max() < 2e-14, (e0.max(), e1.max())


def test_hankel01_vs_scipy(lib):
    sp = pytest.importorskip("scipy.special")
    rng = np.random.default_rng(1)
    r = np.exp(rng.uniform(np.log(1e-8), np.log(1e3), 5000))
    a = rng.uniform(-np.pi / 2, np.pi, 5000)
    z = r * np.exp(1j * a)
    h0, h1 = _hankel(lib, z)
    r0, r1 = sp.hankel1(0, z), sp.hankel1(1, z)
    ok = np.isfinite(r0) & (np.abs(r0) > 1e-290) & (np.abs(r0) < 1e290)
    assert np.max(np.abs(h0 - r0)[ok] / np.abs(r0)[ok]) < 2e-14
    assert np.max(np.abs(h1 - r1)[ok] / np.abs(r1)[ok]) < 2e-14


@needs_ref
@pytest.mark.parametrize("which", ["h", "j"])
def test_scaled_sequences(lib, which):
    R = refimpl.ref()
    zero = ctypes.c_int(0)
    for z, rs, n in [(3.0 + 0j, 0.5, 40), (0.2 + 0.05j, 0.03, 30), (40 + 0j, 1.0, 80),
                     (5 - 1j, 0.8, 25), (1e-3 + 0j, 1e-3, 20), (17 + 9j, 1.0, 60)]:
        mine = np.zeros(n + 1, np.complex128)
        getattr(lib, f"fmm2d_b200_helm_{which}vec")(n, z.real, z.imag, rs, _p(mine))
        ref = np.zeros(n + 8, np.complex128)
        der = np.zeros(n + 8, np.complex128)
        zz = np.array([z])
        fn = R.h2dall_ if which == "h" else R.jbessel2d_
        fn(ctypes.byref(ctypes.c_int(n)), _p(zz), ctypes.byref(ctypes.c_double(rs)), _p(ref),
           ctypes.byref(zero), _p(der))
        ref = ref[: n + 1]
        scale = np.maximum(np.abs(ref), 1e-300)
        err = np.abs(mine - ref) / scale
        assert np.all(err < 1e-11), (z, rs, which, err.max())


@needs_ref
def test_helm_nterms_vs_h2dterms(lib):
    R = refimpl.ref()
    for zk in [10, 0.5 + 0.1j, 500, 1e-3, 30 + 5j, 100, 3j]:
        for eps in [0.51e-8, 1e-3, 1e-6, 1e-12, 1e-15]:
            for bs in [1.0, 0.5, 0.25, 0.125, 1 / 64, 1 / 1024, 2.3, 1e-5]:
                zka = np.array([complex(zk)])
                n = ctypes.c_int(0)
                ier = ctypes.c_int(0)
                R.h2dterms_(ctypes.byref(ctypes.c_double(bs)), _p(zka),
                            ctypes.byref(ctypes.c_double(eps)), ctypes.byref(n),
                            ctypes.byref(ier))
                mine = lib.fmm2d_b200_helm_nterms(bs, complex(zk).real, complex(zk).imag, eps)
                if ier.value == 13:
                    assert mine == -1
                else:
                    assert mine == n.value, (zk, eps, bs, mine, n.value)
