"""Python face of the single-rank case builder (include/iga_case.h).

The same C source is linked into libsnesiga_b200 (GPU callbacks) and into the
CPU oracle library, so one wrapper drives both through identical PETSc-style
objects."""
import ctypes
import numpy as np

from . import native
from .native import vp

KIND = {"ge": 0, "getime": 1}


def _p(a):
    return a.ctypes.data_as(vp)


class Case:
    def __init__(self, lib, phys, nelem, knots, par_mat, bc_type, par_periodic=None, par_dirichlet=None,
                 par_neumann=None, bc_periodic=(0, 0, 0)):
        self.lib = lib
        self._nel = np.ascontiguousarray(nelem, dtype=np.int32)
        self._kn = np.ascontiguousarray(knots, dtype=np.float64)
        self._pm = np.ascontiguousarray(par_mat, dtype=np.float64)
        self._bc = np.ascontiguousarray(bc_type, dtype=np.int32)
        self._pp = np.ascontiguousarray(par_periodic if par_periodic is not None else np.zeros(9), dtype=np.float64)
        self._pd = np.ascontiguousarray(par_dirichlet if par_dirichlet is not None else np.zeros(9), dtype=np.float64)
        pn = np.ascontiguousarray(par_neumann if par_neumann is not None else np.zeros(39), dtype=np.float64)
        self._pn = pn
        self._per = np.ascontiguousarray(bc_periodic, dtype=np.int32)
        h = lib.iga_case_create_periodic(KIND[phys], _p(self._nel), _p(self._kn), _p(self._pm), _p(self._bc),
                                         _p(self._pp), _p(self._pd), _p(pn), int(pn.size), _p(self._per))
        if not h:
            raise RuntimeError("iga_case_create failed")
        self.h = h
        self.ndof = lib.iga_case_ndof(h)
        self.phys = phys

    def close(self):
        if getattr(self, "h", None):
            self.lib.iga_case_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def residual(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = np.empty(self.ndof)
        rc = self.lib.iga_case_residual(self.h, _p(U), _p(R))
        if rc:
            raise RuntimeError("residual callback returned %d" % rc)
        return R

    def tangent(self, U):
        """Returns (rowptr, cols, vals) of the assembled AIJ matrix."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        rc = self.lib.iga_case_tangent(self.h, _p(U))
        if rc:
            raise RuntimeError("tangent callback returned %d" % rc)
        nnz = self.lib.iga_case_tangent_nnz(self.h)
        rowptr = np.empty(self.ndof + 1, dtype=np.int32)
        cols = np.empty(nnz, dtype=np.int32)
        vals = np.empty(nnz)
        self.lib.iga_case_tangent_csr(self.h, _p(rowptr), _p(cols), _p(vals))
        return rowptr, cols, vals

    def index_maps(self):
        """(selfIdx, sendIdx, recvIdx, globalIdx) as the linked snesiga_init left them."""
        n = np.zeros(3, dtype=np.int32)
        self.lib.iga_case_index_maps(self.h, _p(n), None, None, None, None)
        a = [np.empty(int(k), dtype=np.int32) for k in (n[0], n[1], n[2], n[0] + n[2])]
        self.lib.iga_case_index_maps(self.h, _p(n), *[_p(x) for x in a])
        return tuple(a)

    def set_history(self, level, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        if self.lib.iga_case_set_history(self.h, int(level), _p(U)):
            raise ValueError("bad history level")

    def get_history(self, level):
        U = np.empty(self.ndof)
        if self.lib.iga_case_get_history(self.h, int(level), _p(U)):
            raise ValueError("bad history level")
        return U

    def set_par_neumann(self, pn):
        a = np.ascontiguousarray(pn, dtype=np.float64)
        self._pn_live = a
        if self.lib.iga_case_set_par_neumann(self.h, _p(a), int(a.size)):
            raise ValueError("par_neumann too long")

    def set_par_dirichlet(self, pd):
        a = np.ascontiguousarray(pd, dtype=np.float64)
        self.lib.iga_case_set_par_dirichlet(self.h, _p(a))

    def set_par_mat(self, pm):
        a = np.ascontiguousarray(pm, dtype=np.float64)
        self.lib.iga_case_set_par_mat(self.h, _p(a))

    def solve(self, U0):
        """The linked library's snes_solve from U0; returns (converged, U)."""
        U = np.array(U0, dtype=np.float64, copy=True)
        rc = self.lib.iga_case_solve(self.h, _p(U))
        if rc < 0:
            raise RuntimeError("no snes_solve in this library")
        return rc == 0, U

    @property
    def app(self):
        return self.lib.iga_case_app(self.h)

    def intdensity(self, nd):
        """This library's iga_intdensity (src/iga_intdensity.c:10) on U_hist as it
        stands: nd integrated densities (13 for phys/ge, 2 for phys/getime)."""
        HH = np.zeros(nd)
        self.lib.iga_intdensity(_p(HH), vp(self.app))
        return HH


def gpu_case(*args, **kw):
    """A case whose callbacks are the B200 drop-in (libsnesiga_b200)."""
    return Case(native.lib_dropin(), *args, **kw)
