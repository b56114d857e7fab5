"""Oracle access for the tests (test infrastructure only; never shipped or measured).

``oracle/_ref/libref_iga.so`` is IGAP4STANDARD's own assembly code compiled in
place by oracle/build_ref.py.  It exposes the reference callbacks through the
case builder (same C API as igap4standard_b200.case) and the reference's
point functions: ge_residual/ge_tangent (phys/ge), getime_residual/
getime_tangent (phys/getime), eval_Bspline (mesh/nurbs/eval_Bspline.c),
evalN (mesh/nurbs/evalN.c), legendre_handle (src/quadrature.c),
iga_dirichlet (src/iga_dirichlet.c), iga_intdensity (src/iga_intdensity.c),
nurbs_knotinsert (mesh/nurbs/nurbs_knotinsert.c), write_solution / read_solution
(src/ioutil.c).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libref_iga.so")

_lib = None


def available():
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError("oracle/_ref/libref_iga.so is not built (python oracle/build_ref.py)")
        from igap4standard_b200 import native
        L = ctypes.CDLL(REF_LIB, mode=ctypes.RTLD_LOCAL)
        native.bind(L, native.CASE_API)
        vp = ctypes.c_void_p
        for f in ("ge_residual", "ge_tangent", "getime_residual", "getime_tangent"):
            getattr(L, f).argtypes = [vp, vp, vp]
            getattr(L, f).restype = None
        L.eval_Bspline.argtypes = [vp, vp, ctypes.c_int, vp]
        L.eval_Bspline.restype = None
        L.evalN.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.evalN.restype = ctypes.c_double
        L.legendre_handle.argtypes = [vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.legendre_handle.restype = None
        L.iga_dirichlet.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp, ctypes.c_int,
                                    ctypes.c_int]
        L.iga_dirichlet.restype = None
        L.iga_intdensity.argtypes = [vp, vp]
        L.iga_intdensity.restype = None
        L.nurbs_knotinsert.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
        L.nurbs_knotinsert.restype = None
        L.write_solution.argtypes = [ctypes.c_char_p, vp, vp, ctypes.c_int, ctypes.c_int]
        L.write_solution.restype = None
        L.read_solution.argtypes = [ctypes.c_char_p, vp, vp, ctypes.c_int, ctypes.c_int]
        L.read_solution.restype = None
        L.oracle_scale_install.argtypes = [vp, vp, ctypes.c_long]
        L.oracle_scale_install.restype = None
        L.oracle_scale_remove.argtypes = [vp]
        L.oracle_scale_remove.restype = None
        L.oracle_scale_reset.argtypes = []
        L.oracle_scale_reset.restype = None
        L.oracle_scale_calls.restype = ctypes.c_long
        L.oracle_scale_overflow.restype = ctypes.c_long
        L.layout_probe_reference.argtypes = [vp]
        L.layout_probe_ours.argtypes = [vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def case(*args, **kw):
    """A case whose callbacks are the reference's own CPU assembly."""
    from igap4standard_b200.case import Case
    return Case(lib(), *args, **kw)


def ge_residual(u, par):
    u = np.ascontiguousarray(u, dtype=np.float64)
    par = np.ascontiguousarray(par, dtype=np.float64)
    r = np.empty(30)
    lib().ge_residual(_p(r), _p(u), _p(par))
    return r


def ge_tangent(u, par):
    u = np.ascontiguousarray(u, dtype=np.float64)
    par = np.ascontiguousarray(par, dtype=np.float64)
    t = np.empty(900)
    lib().ge_tangent(_p(t), _p(u), _p(par))
    return t.reshape(30, 30)


def getime_residual(u90, par):
    u = np.ascontiguousarray(u90, dtype=np.float64)
    par = np.ascontiguousarray(par, dtype=np.float64)
    r = np.empty(30)
    lib().getime_residual(_p(r), _p(u), _p(par))
    return r


def getime_tangent(u90, par):
    u = np.ascontiguousarray(u90, dtype=np.float64)
    par = np.ascontiguousarray(par, dtype=np.float64)
    t = np.empty(900)
    lib().getime_tangent(_p(t), _p(u), _p(par))
    return t.reshape(30, 30)


def gauss(n=4):
    x = np.empty(n)
    w = np.empty(n)
    lib().legendre_handle(_p(x), _p(w), n, 0.0, 1.0)
    return x, w


def eval_bspline(kv_windows, xq):
    """kv_windows: three 6-knot windows; returns N[27][10]."""
    wins = [np.ascontiguousarray(k, dtype=np.float64) for k in kv_windows]
    ptrs = (ctypes.c_void_p * 3)(*[w.ctypes.data for w in wins])
    x = np.ascontiguousarray(xq, dtype=np.float64)
    N = np.empty(270)
    lib().eval_Bspline(_p(N), ptrs, 2, _p(x))
    return N.reshape(27, 10)


def evalN(kv, k, i, x, p=2):
    kv = np.ascontiguousarray(kv, dtype=np.float64)
    return lib().evalN(_p(kv), int(kv.size), int(k), int(i), int(p), float(x))


def layouts():
    a = np.zeros(128, dtype=np.int64)
    b = np.zeros(128, dtype=np.int64)
    na = lib().layout_probe_reference(_p(a))
    nb = lib().layout_probe_ours(_p(b))
    return a[:na], b[:nb]


class ScaledCase:
    """A reference case whose element integrands are multiplied by s_e = exp(g_e)
    (oracle/elem_scale.c).  residual()/tangent() as Case."""

    def __init__(self, case, g):
        self.case = case
        self.ndof = case.ndof
        self.s = np.ascontiguousarray(np.exp(np.asarray(g, dtype=np.float64)))
        lib().oracle_scale_install(case.app, _p(self.s), int(self.s.size))

    def _checked(self, fn, *a):
        L = lib()
        L.oracle_scale_reset()
        out = fn(*a)
        if L.oracle_scale_overflow() != 0 or L.oracle_scale_calls() != 64 * self.s.size:
            raise RuntimeError("integrand call count does not match the element count")
        return out

    def residual(self, U):
        return self._checked(self.case.residual, U)

    def tangent(self, U):
        return self._checked(self.case.tangent, U)

    def close(self):
        lib().oracle_scale_remove(self.case.app)
