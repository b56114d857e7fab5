"""The allocation-free residual entry point (igab_residual_noalloc).

For callers that cannot let the library allocate device memory (device memory
fully reserved by another allocator, or a fixed device-memory budget inside a
solver callback): the entry point stages U and R in a static device array.
Collected last so that a failure here never hides another test's result."""
import ctypes

import numpy as np
import pytest

from cases import make_case, neumann_values, residual_tolerance

pytestmark = pytest.mark.gpu


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _assembly(name):
    from igap4standard_b200 import Assembly
    c = make_case(name)
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"])
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, c["par_neumann"]))
    return A, c


def test_noalloc_matches_residual_twice(built):
    from igap4standard_b200.native import lib_cuda
    lib = lib_cuda()
    A, c = _assembly("perturbed_lame")
    rng = np.random.default_rng(11)
    for call in range(2):
        U = c["U"] if call == 0 else rng.uniform(-1e-2, 1e-2, A.ndof)
        R_ref = A.residual(U)
        R = np.full(A.ndof, np.nan)
        rc = lib.igab_residual_noalloc(A.h, _p(np.ascontiguousarray(U)), _p(R))
        assert rc == 0, lib.igab_last_error()
        assert np.all(np.abs(R - R_ref) <= residual_tolerance(R_ref))
    A.close()


def test_noalloc_rejects_oversize_mesh(built):
    from igap4standard_b200 import Assembly, knots_for, PAR_MAT_DEFAULT, bc_config0
    from igap4standard_b200.native import lib_cuda
    lib = lib_cuda()
    nelem = (100, 100, 33)   # 1,092,420 dofs > 1,048,576
    bc, pd = bc_config0()
    A = Assembly(nelem, knots_for(nelem), PAR_MAT_DEFAULT, bc, pd)
    U = np.zeros(A.ndof)
    R = np.zeros(A.ndof)
    rc = lib.igab_residual_noalloc(A.h, _p(U), _p(R))
    assert rc == 1
    assert b"exceed" in lib.igab_last_error()
    A.close()
