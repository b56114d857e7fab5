"""GPU parity: the B200 assembly against IGAP4STANDARD's own CPU assembly.

Both sides run on the same mesh, state and parameters; the reference side is
the unmodified reference code (oracle/_ref) driven through the same case
builder.  Criterion (residual and tangent): every entry within 1e-12
relative, with the cancellation floor of tests/cases.py."""
import numpy as np
import pytest

from cases import make_case, neumann_values, residual_tolerance, tangent_tolerance

pytestmark = pytest.mark.gpu

CASES = ["tiny_default", "ragged_config0", "perturbed_lame", "mixed_bc"]


def _assembly(c):
    from igap4standard_b200 import Assembly
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"])
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, c["par_neumann"]))
    return A


def _ref_case(checker, c):
    return checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                   c["par_dirichlet"], c["par_neumann"])


def _report(name, err, tol):
    worst = np.max(err / np.maximum(tol, 1e-300)) if err.size else 0.0
    print("%s: max |diff| %.3e, worst diff/tol %.3f" % (name, err.max() if err.size else 0.0, worst))
    return worst


@pytest.mark.parametrize("name", CASES + ["config0_8"])
def test_residual_parity(built, checker, name):
    c = make_case(name)
    R_ref = _ref_case(checker, c).residual(c["U"])
    A = _assembly(c)
    R = A.residual(c["U"])
    err = np.abs(R - R_ref)
    assert _report(name, err, residual_tolerance(R_ref)) <= 1.0


@pytest.mark.parametrize("kernel", [1, 0])
@pytest.mark.parametrize("name", CASES)
def test_tangent_parity(built, checker, name, kernel):
    """kernel 1: FP64 tensor path (mma f64), kernel 0: FP64 FMA pipe."""
    c = make_case(name)
    rp_ref, cols_ref, v_ref = _ref_case(checker, c).tangent(c["U"])
    A = _assembly(c)
    A.set_option(1, kernel)
    rp, cols = A.pattern()
    assert np.array_equal(rp, rp_ref)
    assert np.array_equal(cols, cols_ref)
    v = A.tangent(c["U"], "fp64")
    err = np.abs(v - v_ref)
    assert _report(name, err, tangent_tolerance(rp_ref, v_ref)) <= 1.0


def test_tangent_fp32_close(built, checker):
    """FP32-built tangent: an inexact-Newton Jacobian, compared rowwise in norm."""
    c = make_case("perturbed_lame")
    rp_ref, _, v_ref = _ref_case(checker, c).tangent(c["U"])
    A = _assembly(c)
    v = A.tangent(c["U"], "fp32").astype(np.float64)
    rowmax = np.maximum.reduceat(np.abs(v_ref), rp_ref[:-1])
    err = np.maximum.reduceat(np.abs(v - v_ref), rp_ref[:-1])
    assert np.all(err <= 1e-5 * rowmax)


def test_dropin_matches_reference(built, checker):
    """The PETSc drop-in (snesiga_Residual/snesiga_Tangent of libsnesiga_b200) on
    the same PETSc-subset objects the reference callbacks fill."""
    from igap4standard_b200 import gpu_case
    c = make_case("perturbed_lame")
    args = ("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"], c["par_dirichlet"],
            c["par_neumann"])
    ref = checker(*args)
    gpu = gpu_case(*args)
    R_ref = ref.residual(c["U"])
    R = gpu.residual(c["U"])
    assert _report("dropin residual", np.abs(R - R_ref), residual_tolerance(R_ref)) <= 1.0
    # the callback's side effect: U_hist level 0 holds the iterate
    assert np.array_equal(gpu.get_history(0), c["U"])
    rp_ref, cols_ref, v_ref = ref.tangent(c["U"])
    rp, cols, v = gpu.tangent(c["U"])
    assert np.array_equal(rp, rp_ref) and np.array_equal(cols, cols_ref)
    assert _report("dropin tangent", np.abs(v - v_ref), tangent_tolerance(rp_ref, v_ref)) <= 1.0
    # a second call re-uses the installed pattern
    U2 = c["U"] * 0.5
    rp_ref2, _, v_ref2 = ref.tangent(U2)
    _, _, v2 = gpu.tangent(U2)
    assert _report("dropin tangent 2", np.abs(v2 - v_ref2), tangent_tolerance(rp_ref2, v_ref2)) <= 1.0


def test_dropin_traction_update(built, checker):
    """par_neumann changed between calls (a time-dependent traction) is picked up."""
    from igap4standard_b200 import gpu_case
    c = make_case("perturbed_lame")
    args = ("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"], c["par_dirichlet"],
            c["par_neumann"])
    ref = checker(*args)
    gpu = gpu_case(*args)
    gpu.residual(c["U"])
    pn2 = c["par_neumann"] * -3.0
    ref.set_par_neumann(pn2)
    gpu.set_par_neumann(pn2)
    R_ref = ref.residual(c["U"])
    R = gpu.residual(c["U"])
    assert _report("traction update", np.abs(R - R_ref), residual_tolerance(R_ref)) <= 1.0


def test_residual_deterministic(built):
    c = make_case("perturbed_lame")
    A = _assembly(c)
    R1 = A.residual(c["U"])
    R2 = A.residual(c["U"])
    assert np.array_equal(R1, R2)
    v1 = A.tangent(c["U"])
    v2 = A.tangent(c["U"])
    assert np.array_equal(v1, v2)
