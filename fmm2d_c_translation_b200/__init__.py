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

__all__ = ["Output", "lfmm2d", "cfmm2d", "hfmm2d", "rfmm2d", "lib", "lib_path",
           "last_error", "tree_build", "FmmError", "Server", "Request",
           "make_request"]

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


# ---------------------------------------------------------------------------
# fmm2dpy-compatible front end (python/fmm2dpy/fmm2d.py:20 hfmm2d, :201
# rfmm2d, :459 lfmm2d, :715 cfmm2d): same keyword arguments, array shapes
# and Output fields.  Every call goes through the guru drivers of the C ABI.
# ---------------------------------------------------------------------------
def _as_f(a, dtype):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


def _run(kernel, *, eps, zk, sources, charges, dipstr, dipvec, targets, pg, pgt, nd):
    out = Output()
    # strengths and outputs: complex, or real for the real-valued Laplace FMM
    cdt = np.float64 if kernel == "r" else np.complex128
    sources = np.asarray(sources, dtype=np.float64)
    assert sources.shape[0] == 2, "The first dimension of sources must be 2"
    ns = sources.shape[1] if sources.ndim == 2 else 1
    src = _as_f(sources.reshape(2, ns), np.float64)
    if pg == 0 and pgt == 0:
        print("Nothing to compute, set either pg or pgt to non-zero")
        return out
    ifcharge = int(charges is not None)
    ifdipole = int(dipstr is not None or dipvec is not None)
    if ifcharge:
        q = _as_f(charges, cdt)
        assert q.size == nd * ns, "Charges must be of shape [nd,ns] (or [ns] for nd = 1)"
    else:
        q = np.zeros(nd * ns, cdt)
    if ifdipole:
        d = _as_f(dipstr, cdt)
        assert d.size == nd * ns, "Dipole strengths must be of shape [nd,ns] (or [ns])"
        if kernel != "c":
            v = _as_f(dipvec, np.float64)
            assert v.size == nd * 2 * ns, "Dipole vectors must be of shape [nd,2,ns] (or [2,ns])"
        else:
            v = np.zeros(1)
    else:
        d = np.zeros(nd * ns, cdt)
        v = np.zeros(nd * 2 * ns)
    if targets is not None:
        targets = np.asarray(targets, dtype=np.float64)
        assert targets.shape[0] == 2, "The first dimension of targets must be 2"
        nt = targets.shape[1] if targets.ndim == 2 else 1
        trg = _as_f(targets.reshape(2, nt), np.float64)
    else:
        nt, trg, pgt = 0, np.zeros((2, 1), order="F"), 0
    gc, hc = (1, 1) if kernel == "c" else (2, 3)

    def alloc(n, comps):
        shape = (nd, n) if comps == 1 else (nd, comps, n)
        return np.zeros(shape, cdt, order="F")

    pot, grad, hess = alloc(ns, 1), alloc(ns, gc), alloc(ns, hc)
    pt, gt, ht = alloc(max(nt, 1), 1), alloc(max(nt, 1), gc), alloc(max(nt, 1), hc)
    ier = _I(0)
    iper = _I(0)
    args = [ctypes.byref(_I(nd)), ctypes.byref(ctypes.c_double(eps))]
    if kernel == "h":
        zka = np.array([complex(zk)], np.complex128)
        args.append(_ptr(zka))
    args += [ctypes.byref(_I(ns)), _ptr(src), ctypes.byref(_I(ifcharge)), _ptr(q),
             ctypes.byref(_I(ifdipole)), _ptr(d)]
    if kernel != "c":
        args.append(_ptr(v))
    args += [ctypes.byref(iper), ctypes.byref(_I(pg)), _ptr(pot), _ptr(grad), _ptr(hess),
             ctypes.byref(_I(nt)), _ptr(trg), ctypes.byref(_I(pgt)), _ptr(pt), _ptr(gt),
             _ptr(ht), ctypes.byref(ier)]
    getattr(lib(), f"{kernel}fmm2d_")(*args)
    out.ier = ier.value
    _check(out.ier, f"{kernel}fmm2d")

    def shaped(a):
        return a[0] if nd == 1 else a

    if pg >= 1:
        out.pot = shaped(pot)
    if pg >= 2:
        out.grad = shaped(grad)
    if pg >= 3:
        out.hess = shaped(hess)
    if pgt >= 1:
        out.pottarg = shaped(pt[..., :nt])
    if pgt >= 2:
        out.gradtarg = shaped(gt[..., :nt])
    if pgt >= 3:
        out.hesstarg = shaped(ht[..., :nt])
    return out


def hfmm2d(*, eps, zk, sources, charges=None, dipstr=None, dipvec=None, targets=None, pg=0,
           pgt=0, nd=1):
    """Helmholtz FMM, u(x) = (i/4) sum_j [c_j H0(k|x - x_j|) + k d_j
    (v_j . (x - x_j)) / |x - x_j| H1(k|x - x_j|)] (fmm2dpy.hfmm2d).
    pg / pgt: 1 potential, 2 + gradient, 3 + Hessian at sources / targets.
    Returns Output with pot (n) or (nd, n), grad (2, n) or (nd, 2, n), hess
    (3, n) or (nd, 3, n) and the same for targets."""
    return _run("h", eps=eps, zk=zk, sources=sources, charges=charges, dipstr=dipstr,
                dipvec=dipvec, targets=targets, pg=pg, pgt=pgt, nd=nd)


def lfmm2d(*, eps, sources, charges=None, dipstr=None, dipvec=None, targets=None, pg=0,
           pgt=0, nd=1):
    """Complex-Laplace FMM with the kernels the reference computes,
    u(x) = sum_j [c_j log|x - x_j| - d_j (v_j . (x - x_j)) / |x - x_j|^2]
    (fmm2dpy.lfmm2d); arguments and outputs as for hfmm2d."""
    return _run("l", eps=eps, zk=None, sources=sources, charges=charges, dipstr=dipstr,
                dipvec=dipvec, targets=targets, pg=pg, pgt=pgt, nd=nd)


def rfmm2d(*, eps, sources, charges=None, dipstr=None, dipvec=None, targets=None, pg=0,
           pgt=0, nd=1):
    """Real-valued Laplace FMM (fmm2dpy.rfmm2d, python/fmm2dpy/fmm2d.py:201),
    u(x) = sum_j [c_j log|x - x_j| - d_j (v_j . (x - x_j)) / |x - x_j|^2] with
    real charges c_j, dipole strengths d_j and dipole vectors v_j; real pot
    (n) or (nd, n), grad (2, n) or (nd, 2, n), hess (3, n) or (nd, 3, n)."""
    return _run("r", eps=eps, zk=None, sources=sources, charges=charges, dipstr=dipstr,
                dipvec=dipvec, targets=targets, pg=pg, pgt=pgt, nd=nd)


def cfmm2d(*, eps, sources, charges=None, dipstr=None, targets=None, pg=0, pgt=0, nd=1):
    """Cauchy-kernel FMM with the reference's conventions (fmm2dpy.cfmm2d):
    u(z) = sum_j [c_j log(z - xi_j) + d_j / (z - xi_j)], the near field
    taking log|z - xi_j| for the logarithm as the reference's direct kernels
    do; grad = du/dz and hess = d2u/dz2, shape (n) or (nd, n)."""
    return _run("c", eps=eps, zk=None, sources=sources, charges=charges, dipstr=dipstr,
                dipvec=None, targets=targets, pg=pg, pgt=pgt, nd=nd)


def fmm2d_batch(kernel="l", *, eps, problems, pg=1, pgt=0):
    """Many independent lfmm2d / cfmm2d problems (nd = 1) with the same eps
    and flags, evaluated as one forest (fmm2d_b200_fmm2d_batch).  Each
    problem is a dict with "sources" (2, n), optional "charges" / "dipstr"
    (n,) complex, "dipvec" (2, n) and "targets" (2, m); every problem must
    have the same kinds of strengths.  Returns a list of Output."""
    L = lib()
    n = len(problems)
    L.fmm2d_b200_fmm2d_batch.argtypes = [_I, _I, ctypes.c_double, _P, _P, _P, _P, _P, _I, _P, _P,
                                         _P, _P, _P, _I, _P, _P, _P]
    keep = []

    def arr(a, dtype):
        x = np.asfortranarray(np.asarray(a, dtype=dtype))
        keep.append(x)
        return x

    def plist(xs):
        if xs is None:
            return None
        v = (ctypes.c_void_p * n)(*[None if x is None else x.ctypes.data for x in xs])
        keep.append(v)
        return ctypes.cast(v, _P)

    src = [arr(p["sources"], np.float64) for p in problems]
    ns = np.array([x.shape[1] for x in src], np.int32)
    has_c = "charges" in problems[0] and problems[0]["charges"] is not None
    has_d = "dipstr" in problems[0] and problems[0]["dipstr"] is not None
    q = [arr(p["charges"], np.complex128) for p in problems] if has_c else None
    d = [arr(p["dipstr"], np.complex128) for p in problems] if has_d else None
    v = [arr(p["dipvec"], np.float64) for p in problems] if (has_d and kernel == "l") else None
    trg = [arr(p["targets"], np.float64) if p.get("targets") is not None else None
           for p in problems]
    nt = np.array([0 if t is None else t.shape[1] for t in trg], np.int32)
    if nt.sum() == 0:
        pgt = 0
    gc, hc = (1, 1) if kernel == "c" else (2, 3)
    outs = [Output() for _ in problems]

    def alloc(count, comps, need):
        if not need:
            return None
        return [np.zeros((comps, k) if comps > 1 else (k,), np.complex128, order="F")
                for k in count]

    pot, grad, hess = alloc(ns, 1, pg >= 1), alloc(ns, gc, pg >= 2), alloc(ns, hc, pg >= 3)
    pt, gt, ht = alloc(nt, 1, pgt >= 1), alloc(nt, gc, pgt >= 2), alloc(nt, hc, pgt >= 3)
    ier = L.fmm2d_b200_fmm2d_batch({"l": 0, "c": 1}[kernel], n, eps, _ptr(ns), plist(src),
                                   plist(q), plist(d), plist(v), pg, plist(pot), plist(grad),
                                   plist(hess), _ptr(nt), plist(trg), pgt, plist(pt),
                                   plist(gt), plist(ht))
    _check(ier, "fmm2d_b200_fmm2d_batch")
    for k, o in enumerate(outs):
        o.pot = pot[k] if pot else None
        o.grad = grad[k] if grad else None
        o.hess = hess[k] if hess else None
        if nt[k] > 0:
            o.pottarg = pt[k] if pt else None
            o.gradtarg = gt[k] if gt else None
            o.hesstarg = ht[k] if ht else None
    return outs


class Plan:
    """Resident geometry for repeated lfmm2d / cfmm2d evaluations on the same
    points (plan.cu): the tree, its lists and the sorted points stay on the
    device; each eval() only brings new strengths.  Outputs as lfmm2d /
    cfmm2d return them."""

    def __init__(self, kernel="l", *, eps, sources, targets=None, charges=True, dipoles=False,
                 pg=1, pgt=0, nd=1):
        L = lib()
        L.fmm2d_b200_plan_create.argtypes = [_I, _I, ctypes.c_double, _I, _P, _I, _I, _I, _I,
                                             _P, _I, ctypes.POINTER(_P)]
        L.fmm2d_b200_plan_eval.argtypes = [_P] * 10
        L.fmm2d_b200_plan_destroy.argtypes = [_P]
        self.kernel, self.nd, self.pg = kernel, nd, pg
        sources = np.asarray(sources, dtype=np.float64)
        self.ns = sources.shape[1]
        src = _as_f(sources, np.float64)
        if targets is not None:
            trg = _as_f(targets, np.float64)
            self.nt = trg.shape[1]
        else:
            trg, self.nt, pgt = None, 0, 0
        self.pgt = pgt
        self.ifcharge, self.ifdipole = int(bool(charges)), int(bool(dipoles))
        h = _P()
        ier = L.fmm2d_b200_plan_create({"l": 0, "c": 1}[kernel], nd, eps, self.ns, _ptr(src),
                                       self.ifcharge, self.ifdipole, pg, self.nt, _ptr(trg),
                                       pgt, ctypes.byref(h))
        _check(ier, "fmm2d_b200_plan_create")
        self._h = h

    def eval(self, charges=None, dipstr=None, dipvec=None):
        nd, ns, nt = self.nd, self.ns, self.nt
        q = _as_f(charges, np.complex128) if self.ifcharge else None
        d = _as_f(dipstr, np.complex128) if self.ifdipole else None
        v = _as_f(dipvec, np.float64) if (self.ifdipole and self.kernel == "l") else None
        gc, hc = (1, 1) if self.kernel == "c" else (2, 3)

        def alloc(n, comps, need):
            if not need or n == 0:
                return None
            shape = (nd, n) if comps == 1 else (nd, comps, n)
            return np.zeros(shape, np.complex128, order="F")

        pg, pgt = self.pg, self.pgt
        outs = [alloc(ns, 1, pg >= 1), alloc(ns, gc, pg >= 2), alloc(ns, hc, pg >= 3),
                alloc(nt, 1, pgt >= 1), alloc(nt, gc, pgt >= 2), alloc(nt, hc, pgt >= 3)]
        ier = lib().fmm2d_b200_plan_eval(self._h, _ptr(q), _ptr(d), _ptr(v),
                                         *[_ptr(o) for o in outs])
        _check(ier, "fmm2d_b200_plan_eval")
        out = Output()
        shaped = (lambda a: a if a is None or nd > 1 else a[0])
        out.pot, out.grad, out.hess, out.pottarg, out.gradtarg, out.hesstarg = map(shaped, outs)
        return out

    @property
    def uses_graph(self):
        """True once evaluations replay the captured CUDA graph."""
        L = lib()
        L.fmm2d_b200_plan_uses_graph.argtypes = [_P]
        return bool(L.fmm2d_b200_plan_uses_graph(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().fmm2d_b200_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Request loop (serve.cu): continuous admission of independent evaluations.
# ---------------------------------------------------------------------------
def autotune(kernel="l", *, eps, ns, nt=0, sources=None, targets=None, charges=True,
             dipoles=False, pg=1, pgt=0):
    """Autotunes the mixed-precision path for the order of `eps` on a
    workload of this shape (the given points, or seeded uniform ones) and
    keeps the choice for later calls.  Returns (leaf capacity, M2L form,
    ms per evaluation)."""
    L = lib()
    L.fmm2d_b200_autotune.argtypes = [_I, ctypes.c_double, _I, _P, _I, _P, _I, _I, _I, _I,
                                      _P, _P, _P]
    src = None if sources is None else _as_f(sources, np.float64)
    trg = None if targets is None else _as_f(targets, np.float64)
    nd_, fm_, ms_ = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
    ier = L.fmm2d_b200_autotune({"l": 0, "c": 1}[kernel], eps, ns,
                                None if src is None else _ptr(src), nt,
                                None if trg is None else _ptr(trg), int(bool(charges)),
                                int(bool(dipoles)), pg, pgt, ctypes.byref(nd_),
                                ctypes.byref(fm_), ctypes.byref(ms_))
    _check(ier, "fmm2d_b200_autotune")
    return nd_.value, fm_.value, ms_.value


class Request(ctypes.Structure):
    """fmm2d_b200_request: the guru drivers' arguments of one evaluation."""
    _fields_ = [("kernel", _I), ("nd", _I), ("eps", ctypes.c_double),
                ("zk", ctypes.c_double * 2), ("ns", _I), ("sources", _P),
                ("ifcharge", _I), ("charge", _P), ("ifdipole", _I), ("dipstr", _P),
                ("dipvec", _P), ("ifpgh", _I), ("pot", _P), ("grad", _P), ("hess", _P),
                ("nt", _I), ("targ", _P), ("ifpghtarg", _I), ("pottarg", _P),
                ("gradtarg", _P), ("hesstarg", _P), ("precision", _I)]


class Server:
    """A request loop on the current device: `slots` concurrent
    evaluations within `hbm_budget` bytes of estimated footprint.  submit()
    keeps the request's arrays alive until wait() returns its ticket."""

    def __init__(self, slots=4, hbm_budget=120e9):
        L = lib()
        L.fmm2d_b200_server_create.restype = _P
        L.fmm2d_b200_server_create.argtypes = [_I, ctypes.c_double]
        L.fmm2d_b200_server_submit.restype = ctypes.c_longlong
        L.fmm2d_b200_server_submit.argtypes = [_P, ctypes.POINTER(Request)]
        L.fmm2d_b200_server_wait.argtypes = [_P, ctypes.c_longlong, _P]
        L.fmm2d_b200_server_stats.argtypes = [_P, _P]
        L.fmm2d_b200_server_stats.restype = None
        L.fmm2d_b200_server_destroy.argtypes = [_P]
        L.fmm2d_b200_server_destroy.restype = None
        L.fmm2d_b200_request_bytes.restype = ctypes.c_double
        L.fmm2d_b200_request_bytes.argtypes = [ctypes.POINTER(Request)]
        self._L = L
        self._h = L.fmm2d_b200_server_create(int(slots), float(hbm_budget))
        if not self._h:
            raise FmmError("server_create failed")
        self._keep = {}

    def submit(self, req, keep=()):
        t = self._L.fmm2d_b200_server_submit(self._h, ctypes.byref(req))
        if t < 0:
            raise FmmError("invalid request")
        self._keep[t] = (req, keep)
        return t

    def wait(self, ticket):
        """(ier, (queue_ms, run_ms, total_ms))."""
        times = np.zeros(3)
        ier = self._L.fmm2d_b200_server_wait(self._h, ticket, _ptr(times))
        self._keep.pop(ticket, None)
        return ier, tuple(times)

    def stats(self):
        out = np.zeros(6)
        self._L.fmm2d_b200_server_stats(self._h, _ptr(out))
        self._L.fmm2d_b200_server_batched.restype = ctypes.c_longlong
        self._L.fmm2d_b200_server_batched.argtypes = [_P]
        return dict(bytes_in_use=out[0], peak_bytes=out[1], queued=int(out[2]),
                    running=int(out[3]), rejected=int(out[4]), peak_running=int(out[5]),
                    batched=int(self._L.fmm2d_b200_server_batched(self._h)))

    def request_bytes(self, req):
        return self._L.fmm2d_b200_request_bytes(ctypes.byref(req))

    def close(self):
        if self._h:
            self._L.fmm2d_b200_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_request(kernel, *, eps, sources, charges=None, dipstr=None, dipvec=None,
                 targets=None, pg=1, pgt=0, zk=0.0, precision=0):
    """A Request for nd = 1 with freshly allocated outputs.  Returns
    (Request, arrays) where arrays holds every buffer the request points to
    (pass it to Server.submit as `keep`); outputs are arrays["pot"], ...,
    grad as (n, 2) rows and hess as (n, 3) rows for lfmm2d / hfmm2d."""
    kid = {"l": 0, "c": 1, "h": 2}[kernel]
    src = _as_f(sources, np.float64)
    ns = src.shape[1]
    arrs = {"src": src}
    r = Request()
    r.kernel, r.nd, r.eps = kid, 1, float(eps)
    zk = complex(zk)
    r.zk[0], r.zk[1] = zk.real, zk.imag
    r.ns, r.sources = ns, src.ctypes.data
    r.precision = int(precision)
    if charges is not None:
        arrs["q"] = np.ascontiguousarray(charges, np.complex128)
        r.ifcharge, r.charge = 1, arrs["q"].ctypes.data
    if dipstr is not None:
        arrs["d"] = np.ascontiguousarray(dipstr, np.complex128)
        r.ifdipole, r.dipstr = 1, arrs["d"].ctypes.data
        if kernel != "c":
            arrs["v"] = _as_f(dipvec, np.float64)
            r.dipvec = arrs["v"].ctypes.data
    gc, hc = (1, 1) if kernel == "c" else (2, 3)

    def outs(prefix, n, flag):
        arrs["pot" + prefix] = np.zeros(n, np.complex128)
        ptrs = [arrs["pot" + prefix].ctypes.data, None, None]
        if flag >= 2:
            arrs["grad" + prefix] = np.zeros((n, gc) if gc > 1 else n, np.complex128)
            ptrs[1] = arrs["grad" + prefix].ctypes.data
        if flag >= 3:
            arrs["hess" + prefix] = np.zeros((n, hc) if hc > 1 else n, np.complex128)
            ptrs[2] = arrs["hess" + prefix].ctypes.data
        return ptrs

    if pg:
        r.ifpgh = pg
        r.pot, r.grad, r.hess = outs("", ns, pg)
    if targets is not None and pgt:
        trg = _as_f(targets, np.float64)
        arrs["trg"] = trg
        r.nt, r.targ, r.ifpghtarg = trg.shape[1], trg.ctypes.data, pgt
        r.pottarg, r.gradtarg, r.hesstarg = outs("targ", trg.shape[1], pgt)
    return r, arrs
