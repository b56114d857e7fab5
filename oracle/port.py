"""CPU restatement oracle (oracle/port/oracle_port.cpp) -- test infrastructure only.

Usable wherever g++ is present (builds on first use into oracle/_build/); the
tests pin it against the reference itself (oracle/_ref) and the committed
golden vectors, and fall back to it where the reference library is absent."""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        sys.path.insert(0, HERE)
        import build_port
        path = build_port.build()
        L = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        vp = ctypes.c_void_p
        L.port_case_create.restype = vp
        L.port_case_create.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_int]
        L.port_case_destroy.argtypes = [vp]
        L.port_ndof.restype = ctypes.c_long
        L.port_ndof.argtypes = [vp]
        L.port_nnz.restype = ctypes.c_long
        L.port_nnz.argtypes = [vp]
        L.port_residual.argtypes = [vp, vp, vp]
        L.port_tangent.argtypes = [vp, vp, vp, vp, vp]
        L.port_ge_point.argtypes = [vp, vp, vp, vp]
        L.port_gauss.argtypes = [vp, vp]
        L.port_bspline_window.argtypes = [vp, ctypes.c_double, vp]
        L.port_bspline_any.restype = ctypes.c_double
        L.port_bspline_any.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class PortCase:
    def __init__(self, nelem, knots, par_mat, bc_type, par_periodic=None, par_dirichlet=None, par_neumann=None):
        L = lib()
        self._a = [np.ascontiguousarray(nelem, dtype=np.int32), np.ascontiguousarray(knots, dtype=np.float64),
                   np.ascontiguousarray(par_mat, dtype=np.float64), np.ascontiguousarray(bc_type, dtype=np.int32),
                   np.ascontiguousarray(par_periodic if par_periodic is not None else np.zeros(9), dtype=np.float64),
                   np.ascontiguousarray(par_dirichlet if par_dirichlet is not None else np.zeros(9), dtype=np.float64),
                   np.ascontiguousarray(par_neumann if par_neumann is not None else np.zeros(39), dtype=np.float64)]
        self.h = L.port_case_create(*[_p(a) for a in self._a], int(self._a[6].size))
        self.ndof = L.port_ndof(self.h)
        self.nnz = L.port_nnz(self.h)

    def __del__(self):
        try:
            lib().port_case_destroy(self.h)
        except Exception:
            pass

    def set_par_neumann(self, pn):
        """Change the traction parameters (the case is rebuilt with them)."""
        L = lib()
        L.port_case_destroy(self.h)
        self._a[6] = np.ascontiguousarray(pn, dtype=np.float64)
        self.h = L.port_case_create(*[_p(a) for a in self._a], int(self._a[6].size))

    def residual(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.empty(self.ndof)
        lib().port_residual(self.h, _p(U), _p(R))
        return R

    def tangent(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        rp = np.empty(self.ndof + 1, dtype=np.int32)
        cols = np.empty(self.nnz, dtype=np.int32)
        vals = np.empty(self.nnz)
        lib().port_tangent(self.h, _p(U), _p(rp), _p(cols), _p(vals))
        return rp, cols, vals


def ge_point(u, par):
    u = np.ascontiguousarray(u, dtype=np.float64)
    par = np.ascontiguousarray(par, dtype=np.float64)
    r = np.empty(30)
    D = np.empty(900)
    lib().port_ge_point(_p(u), _p(par), _p(r), _p(D))
    return r, D.reshape(30, 30)


def gauss():
    x = np.empty(4)
    w = np.empty(4)
    lib().port_gauss(_p(x), _p(w))
    return x, w


def bspline_window(kv6, x):
    kv6 = np.ascontiguousarray(kv6, dtype=np.float64)
    out = np.empty(9)
    lib().port_bspline_window(_p(kv6), float(x), _p(out))
    return out.reshape(3, 3)


def bspline_any(kv, k, i, x, p=2):
    kv = np.ascontiguousarray(kv, dtype=np.float64)
    return lib().port_bspline_any(_p(kv), int(kv.size), int(k), int(i), int(p), float(x))
