"""The allocation-free residual entry point (igab_residual_noalloc).

Some callers cannot let the library allocate device memory: their device
memory is already reserved in full by another allocator, or the residual runs
inside a solver callback under a fixed device-memory budget.  For them
igab_residual_noalloc stages U and R in a static device array instead of the
context buffers that igab_residual allocates on first use.

The first test works on a fresh context: the no-alloc calls come before any
igab_residual, match the reference's own CPU residual, leave the context
without staging buffers, and then agree with igab_residual on the same states,
two calls in a row.  Collected last so that a failure here never hides another
test's result."""
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


def _staging_bytes(lib, A):
    n = ctypes.c_size_t()
    assert lib.igab_staging_bytes(A.h, ctypes.byref(n)) == 0, lib.igab_last_error()
    return n.value


def test_noalloc_fresh_context_matches_reference_and_residual(built, checker):
    from igap4standard_b200.native import lib_cuda
    lib = lib_cuda()
    A, c = _assembly("perturbed_lame")
    rng = np.random.default_rng(11)
    states = [c["U"], rng.uniform(-1e-2, 1e-2, A.ndof)]
    R_noalloc = []
    for U in states:                       # before any igab_residual on this context
        R = np.full(A.ndof, np.nan)
        rc = lib.igab_residual_noalloc(A.h, _p(np.ascontiguousarray(U)), _p(R))
        assert rc == 0, lib.igab_last_error()
        R_noalloc.append(R)
        assert _staging_bytes(lib, A) == 0   # no context staging was allocated
    ref = checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                  c["par_dirichlet"], c["par_neumann"])
    for U, R in zip(states, R_noalloc):
        R_ref = ref.residual(U)
        assert np.all(np.abs(R - R_ref) <= residual_tolerance(R_ref))
    for U, R in zip(states, R_noalloc):   # the existing entry point, same states
        R_res = A.residual(U)
        assert np.all(np.abs(R - R_res) <= residual_tolerance(R_res))
    assert _staging_bytes(lib, A) == 2 * A.ndof * 8
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
    assert _staging_bytes(lib, A) == 0
    A.close()
