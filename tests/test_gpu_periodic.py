"""Periodic directions on one rank: the B200 assembly (local-grid kernels, fold of the
ghost rows and columns into their owners, Dirichlet rows on the owned system) against
the reference's own assembly on the same periodic mesh (oracle/_ref, whose halo
exchange is a message to itself): residual and tangent entries within 1e-12, the AIJ
pattern identical, FP32 tangent rowwise 1e-5; the transient physics with history
levels; the drop-in callbacks; entry points without a periodic form refuse."""
import numpy as np
import pytest

from cases import neumann_values, residual_tolerance, tangent_tolerance
from periodic_cases import PERIODIC, make_periodic_case

pytestmark = pytest.mark.gpu


def _ref(oracle_lib, c):
    return oracle_lib.case(c["phys"], c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                           c["par_dirichlet"], c["par_neumann"], bc_periodic=c["bc_periodic"])


def _assembly(c):
    from igap4standard_b200 import Assembly
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"],
                 phys=c["phys"], bc_periodic=c["bc_periodic"])
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, c["par_neumann"]))
    return A


def _worst(err, tol):
    return float(np.max(err / np.maximum(tol, 1e-300))) if err.size else 0.0


@pytest.mark.parametrize("per", PERIODIC)
def test_periodic_residual_and_tangent_match_reference(built, oracle_lib, per):
    c = make_periodic_case(per, seed=sum(per) + 4 * per[0])
    ref = _ref(oracle_lib, c)
    A = _assembly(c)
    assert A.ndof == ref.ndof
    R_ref = ref.residual(c["U"])
    R = A.residual(c["U"])
    w = _worst(np.abs(R - R_ref), residual_tolerance(R_ref))
    print(per, "residual worst diff/tol %.3f" % w)
    assert w <= 1.0
    rp_ref, cols_ref, v_ref = ref.tangent(c["U"])
    rp, cols = A.pattern()
    assert np.array_equal(rp, rp_ref) and np.array_equal(cols, cols_ref)
    v = A.tangent(c["U"], "fp64")
    w = _worst(np.abs(v - v_ref), tangent_tolerance(rp_ref, v_ref))
    print(per, "tangent worst diff/tol %.3f" % w)
    assert w <= 1.0
    v32 = A.tangent(c["U"], "fp32").astype(np.float64)
    rowmax = np.maximum.reduceat(np.abs(v_ref), rp_ref[:-1])
    assert np.all(np.maximum.reduceat(np.abs(v32 - v_ref), rp_ref[:-1]) <= 1e-5 * rowmax)
    # the Dirichlet rows are owned rows of the non-periodic faces
    rows = A.dirichlet_rows()
    assert np.all(rows < A.ndof)
    A.close()


def test_periodic_device_entry_points_and_offsets(built, oracle_lib):
    import torch
    c = make_periodic_case((1, 0, 1), seed=3)
    A = _assembly(c)
    Ud = torch.as_tensor(c["U"]).cuda()
    Rd = torch.empty(A.ndof, dtype=torch.float64, device="cuda")
    Vd = torch.empty(A.nnz, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    A.residual_device(Ud.data_ptr(), Rd.data_ptr())
    A.tangent_device(Ud.data_ptr(), Vd.data_ptr(), "fp64")
    A.sync()
    assert np.array_equal(Rd.cpu().numpy(), A.residual(c["U"]))
    assert np.array_equal(Vd.cpu().numpy(), A.tangent(c["U"], "fp64"))
    rp, cols = A.pattern()
    for r in np.random.default_rng(0).choice(A.ndof, 20, replace=False):
        k = rp[r] + np.random.default_rng(int(r)).integers(0, rp[r + 1] - rp[r])
        assert A.csr_offset(r, cols[k]) == k
    with pytest.raises(RuntimeError) as e:
        A.newton_solve_device(Ud.data_ptr(), "fp64")
    assert e.value.code == 5   # IGAB_ERR_UNSUPPORTED
    A.close()


def test_periodic_transient_with_history(built, oracle_lib):
    c = make_periodic_case((0, 1, 0), nelem=(3, 4, 3), seed=8, phys="getime")
    ref = _ref(oracle_lib, c)
    A = _assembly(c)
    rng = np.random.default_rng(12)
    U1, U0 = rng.uniform(-2e-3, 2e-3, A.ndof), rng.uniform(-2e-3, 2e-3, A.ndof)
    for level, H in ((1, U1), (2, U0)):
        ref.set_history(level, H)
        A.set_history(level, H)
    R_ref = ref.residual(c["U"])
    assert _worst(np.abs(A.residual(c["U"]) - R_ref), residual_tolerance(R_ref)) <= 1.0
    rp_ref, cols_ref, v_ref = ref.tangent(c["U"])
    v = A.tangent(c["U"], "fp64")
    assert _worst(np.abs(v - v_ref), tangent_tolerance(rp_ref, v_ref)) <= 1.0
    A.close()


def test_periodic_dropin_callbacks(built, oracle_lib):
    """snesiga_Residual / snesiga_Tangent of libsnesiga_b200 on a periodic single-rank mesh
    (the case's Nurbs owns nelem points along x and y and is its own halo neighbour)."""
    from igap4standard_b200 import gpu_case
    c = make_periodic_case((1, 1, 0), seed=6)
    args = (c["phys"], c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"], c["par_dirichlet"],
            c["par_neumann"])
    ref = _ref(oracle_lib, c)
    gpu = gpu_case(*args, bc_periodic=c["bc_periodic"])
    R_ref = ref.residual(c["U"])
    assert _worst(np.abs(gpu.residual(c["U"]) - R_ref), residual_tolerance(R_ref)) <= 1.0
    rp_ref, cols_ref, v_ref = ref.tangent(c["U"])
    rp, cols, v = gpu.tangent(c["U"])
    assert np.array_equal(rp, rp_ref) and np.array_equal(cols, cols_ref)
    assert _worst(np.abs(v - v_ref), tangent_tolerance(rp_ref, v_ref)) <= 1.0
    gpu.close()
