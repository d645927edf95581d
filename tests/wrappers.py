"""Calls any of the 81 flag wrappers (lfmm2d_*, cfmm2d_*, hfmm2d_*) of a
library loaded with ctypes -- the GPU library or the reference build --
with the argument list the Fortran wrapper declares
(src/laplace/lfmm2dwrap.f, cfmm2dwrap.f, src/helmholtz/hfmm2dwrap.f)."""
import ctypes

import numpy as np

_P = ctypes.c_void_p

VARIANTS = [f"{st}_{cd}_{p}" for st in ("s", "t", "st")
            for cd in ("c", "d", "cd") for p in ("p", "g", "h")]


def _p(a):
    return a.ctypes.data_as(_P)


def call(lib, family, variant, eps, sources, charge=None, dipstr=None,
         dipvec=None, targ=None, zk=None):
    """sources (2, ns); charge/dipstr (ns,) complex; dipvec (2, ns);
    targ (2, nt).  Returns (dict of outputs, ier)."""
    st, cd, pgh = variant.split("_")
    npgh = {"p": 1, "g": 2, "h": 3}[pgh]
    src = np.asfortranarray(sources, dtype=np.float64)
    ns = src.shape[1]
    keep = [src]
    args = [ctypes.byref(ctypes.c_double(eps))]
    if family == "h":
        zka = np.array([zk], dtype=np.complex128)
        keep.append(zka)
        args.append(_p(zka))
    args += [ctypes.byref(ctypes.c_int(ns)), _p(src)]
    if "c" in cd:
        q = np.ascontiguousarray(charge, dtype=np.complex128)
        keep.append(q)
        args.append(_p(q))
    if "d" in cd:
        d = np.ascontiguousarray(dipstr, dtype=np.complex128)
        keep.append(d)
        args.append(_p(d))
        if family != "c":
            v = np.asfortranarray(dipvec, dtype=np.float64)
            keep.append(v)
            args.append(_p(v))
    gc, hc = (1, 1) if family == "c" else (2, 3)
    out = {}

    def outputs(prefix, n):
        out[f"pot{prefix}"] = np.zeros(n, np.complex128)
        args.append(_p(out[f"pot{prefix}"]))
        if npgh >= 2:
            out[f"grad{prefix}"] = np.zeros((n, gc) if gc > 1 else n, np.complex128)
            args.append(_p(out[f"grad{prefix}"]))
        if npgh >= 3:
            out[f"hess{prefix}"] = np.zeros((n, hc) if hc > 1 else n, np.complex128)
            args.append(_p(out[f"hess{prefix}"]))

    if "s" in st:
        outputs("", ns)
    if "t" in st:
        t = np.asfortranarray(targ, dtype=np.float64)
        keep.append(t)
        args += [ctypes.byref(ctypes.c_int(t.shape[1])), _p(t)]
        outputs("targ", t.shape[1])
    ier = ctypes.c_int(-1)
    args.append(ctypes.byref(ier))
    getattr(lib, f"{family}fmm2d_{variant}_")(*args)
    return out, ier.value


def rel_err(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def call_nd(lib, family, variant, eps, sources, nd=1, vec=False, charge=None, dipstr=None,
            dipvec=None, targ=None, zk=None):
    """Any flag wrapper of the four families (l, c, h, r), plain (nd = 1)
    or _vec (leading nd argument).  charge/dipstr: (ns,) or (nd, ns) --
    complex, or real for rfmm2d; dipvec: (2, ns) or (nd, 2, ns).  Outputs
    come back in the Fortran layouts as (n, [comps,] nd) arrays."""
    st, cd, pgh = variant.split("_")
    npgh = {"p": 1, "g": 2, "h": 3}[pgh]
    dt = np.float64 if family == "r" else np.complex128
    src = np.asfortranarray(sources, dtype=np.float64)
    ns = src.shape[1]
    keep = [src]
    args = []
    if vec:
        args.append(ctypes.byref(ctypes.c_int(nd)))
    args.append(ctypes.byref(ctypes.c_double(eps)))
    if family == "h":
        zka = np.array([zk], dtype=np.complex128)
        keep.append(zka)
        args.append(_p(zka))
    args += [ctypes.byref(ctypes.c_int(ns)), _p(src)]

    def strength(a):
        # Fortran (nd, ns): element (j, i) at j + nd * i
        a = np.asarray(a, dtype=dt)
        a = a.reshape(nd, ns) if a.ndim == 2 else a.reshape(1, ns)
        out = np.ascontiguousarray(a.T)
        keep.append(out)
        return _p(out)

    if "c" in cd:
        args.append(strength(charge))
    if "d" in cd:
        args.append(strength(dipstr))
        if family != "c":
            v = np.asarray(dipvec, dtype=np.float64).reshape(nd, 2, ns)
            vf = np.ascontiguousarray(np.transpose(v, (2, 1, 0)))  # (ns, 2, nd) C order
            keep.append(vf)
            args.append(_p(vf))
    gc, hc = (1, 1) if family == "c" else (2, 3)
    out = {}

    def outputs(prefix, n):
        out[f"pot{prefix}"] = np.zeros((n, nd), dt)
        args.append(_p(out[f"pot{prefix}"]))
        if npgh >= 2:
            out[f"grad{prefix}"] = np.zeros((n, gc, nd), dt)
            args.append(_p(out[f"grad{prefix}"]))
        if npgh >= 3:
            out[f"hess{prefix}"] = np.zeros((n, hc, nd), dt)
            args.append(_p(out[f"hess{prefix}"]))

    if "s" in st:
        outputs("", ns)
    if "t" in st:
        t = np.asfortranarray(targ, dtype=np.float64)
        keep.append(t)
        args += [ctypes.byref(ctypes.c_int(t.shape[1])), _p(t)]
        outputs("targ", t.shape[1])
    ier = ctypes.c_int(-1)
    args.append(ctypes.byref(ier))
    name = f"{family}fmm2d_{variant}_" + ("vec_" if vec else "")
    getattr(lib, name)(*args)
    return out, ier.value
