"""GPU parity of the transient physics (phys/getime) against the reference's
own CPU assembly: residual and tangent with two history levels."""
import numpy as np
import pytest

from cases import make_transient_case, neumann_values, residual_tolerance, tangent_tolerance

pytestmark = pytest.mark.gpu

CASES = ["getime_small", "getime_config2"]


def _ref(oracle_lib, c):
    C = oracle_lib.case("getime", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                        c["par_dirichlet"], c["par_neumann"])
    C.set_history(1, c["U1"])
    C.set_history(2, c["U0"])
    return C


def _assembly(c):
    from igap4standard_b200 import Assembly
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"],
                 phys="getime")
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, c["par_neumann"]))
    A.set_history(1, c["U1"])
    A.set_history(2, c["U0"])
    return A


@pytest.mark.parametrize("name", CASES)
def test_getime_residual(built, oracle_lib, name):
    c = make_transient_case(name)
    R_ref = _ref(oracle_lib, c).residual(c["U"])
    R = _assembly(c).residual(c["U"])
    tol = residual_tolerance(R_ref)
    assert np.max(np.abs(R - R_ref) / tol) <= 1.0


@pytest.mark.parametrize("name", CASES)
def test_getime_tangent(built, oracle_lib, name):
    c = make_transient_case(name)
    rp, cols, v_ref = _ref(oracle_lib, c).tangent(c["U"])
    A = _assembly(c)
    v = A.tangent(c["U"], "fp64")
    assert np.max(np.abs(v - v_ref) / tangent_tolerance(rp, v_ref)) <= 1.0
    v32 = A.tangent(c["U"], "fp32").astype(np.float64)
    rowmax = np.maximum.reduceat(np.abs(v_ref), rp[:-1])
    err = np.maximum.reduceat(np.abs(v32 - v_ref), rp[:-1])
    assert np.all(err <= 1e-5 * rowmax)


def test_getime_dropin_history(built, oracle_lib):
    """The drop-in reads U_hist levels 1 and 2 from the IGA struct, as the reference callback does."""
    from igap4standard_b200 import gpu_case
    c = make_transient_case("getime_config2")
    args = ("getime", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"], c["par_dirichlet"],
            c["par_neumann"])
    ref = oracle_lib.case(*args)
    gpu = gpu_case(*args)
    for C in (ref, gpu):
        C.set_history(1, c["U1"])
        C.set_history(2, c["U0"])
    R_ref = ref.residual(c["U"])
    R = gpu.residual(c["U"])
    assert np.max(np.abs(R - R_ref) / residual_tolerance(R_ref)) <= 1.0
    rp, cols, v_ref = ref.tangent(c["U"])
    rp2, cols2, v = gpu.tangent(c["U"])
    assert np.array_equal(cols, cols2)
    assert np.max(np.abs(v - v_ref) / tangent_tolerance(rp, v_ref)) <= 1.0
