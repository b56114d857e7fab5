"""Autotuner of the assembly schedule: the choices it leaves applied are valid,
the tuned assembly still matches the reference, a cache file short-cuts the
timing, and a tuned batch schedule gives bit-identical batched results."""
import numpy as np
import pytest

from cases import make_case, neumann_values, residual_tolerance, tangent_tolerance

pytestmark = pytest.mark.gpu


def _assembly(c):
    from igap4standard_b200 import Assembly
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"])
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, c["par_neumann"]))
    return A


def test_autotune_mesh_keeps_parity(built, checker, tmp_path):
    import torch
    c = make_case("config0_8")
    ref = checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                  c["par_dirichlet"], c["par_neumann"])
    A = _assembly(c)
    U = torch.as_tensor(c["U"]).cuda()
    cache = str(tmp_path / "tune.json")
    r = A.autotune(U.data_ptr(), what=7, reps=2, cache=cache)
    assert not r["cached"]
    assert r["residual_tile"] in (2, 4) and r["tangent_fp64_kernel"] in (0, 1) and r["tangent_fp32_kernel"] in (0, 1)
    assert r["residual_ms"] > 0 and r["tangent_fp64_ms"] > 0 and r["tangent_fp32_ms"] > 0
    assert A.get_option(1) == r["tangent_fp64_kernel"] and A.get_option(2) == r["tangent_fp32_kernel"]
    R_ref = ref.residual(c["U"])
    rp, _, v_ref = ref.tangent(c["U"])
    assert np.all(np.abs(A.residual(c["U"]) - R_ref) <= residual_tolerance(R_ref))
    assert np.all(np.abs(A.tangent(c["U"]) - v_ref) <= tangent_tolerance(rp, v_ref))
    # a second context picks the stored schedule up without timing
    B = _assembly(c)
    r2 = B.autotune(None, what=7, reps=2, cache=cache)
    assert r2["cached"]
    assert B.get_option(1) == r["tangent_fp64_kernel"] and B.get_option(2) == r["tangent_fp32_kernel"]


@pytest.mark.parametrize("order", [1, 2])
def test_colour_orders_keep_parity(built, checker, order):
    """Every colour order of the element schedule matches the reference, and the x-slab
    tangent of the host entry point equals the whole-mesh device tangent bit for bit."""
    import torch
    c = make_case("config0_8")
    ref = checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                  c["par_dirichlet"], c["par_neumann"])
    A = _assembly(c)
    A.set_option(3, order)
    assert A.get_option(3) == order
    R_ref = ref.residual(c["U"])
    rp, _, v_ref = ref.tangent(c["U"])
    assert np.all(np.abs(A.residual(c["U"]) - R_ref) <= residual_tolerance(R_ref))
    V = A.tangent(c["U"])
    assert np.all(np.abs(V - v_ref) <= tangent_tolerance(rp, v_ref))
    # x-slab host tangent (26 elements along x: 13 tiles, slabs with downloads) = device tangent
    from igap4standard_b200 import Assembly, mesh
    ne = (26, 3, 2)
    S = Assembly(ne, mesh.knots_for(ne, perturb=0.1, seed=4), c["par_mat"], *mesh.bc_config0())
    S.set_option(3, order)
    U = np.random.default_rng(8).uniform(-1e-3, 1e-3, S.ndof)
    Ud = torch.as_tensor(U).cuda()
    for prec, dt in (("fp64", torch.float64), ("fp32", torch.float32)):
        Vd = torch.empty(S.nnz, dtype=dt, device="cuda")
        torch.cuda.synchronize()
        S.tangent_device(Ud.data_ptr(), Vd.data_ptr(), prec)
        S.sync()
        assert np.array_equal(Vd.cpu().numpy(), S.tangent(U, prec)), prec


def test_autotune_colour_order(built, checker, tmp_path):
    import torch
    c = make_case("config0_8")
    ref = checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                  c["par_dirichlet"], c["par_neumann"])
    A = _assembly(c)
    U = torch.as_tensor(c["U"]).cuda()
    cache = str(tmp_path / "tune.json")
    r = A.autotune(U.data_ptr(), what=15, reps=2, cache=cache)
    assert r["colour_order"] in (0, 1, 2) and A.get_option(3) == r["colour_order"]
    R_ref = ref.residual(c["U"])
    assert np.all(np.abs(A.residual(c["U"]) - R_ref) <= residual_tolerance(R_ref))
    B = _assembly(c)
    r2 = B.autotune(None, what=15, reps=2, cache=cache)
    assert r2["cached"] and B.get_option(3) == r["colour_order"]


def test_autotune_batch_colour_order(built):
    from igap4standard_b200 import Batch, mesh
    inst = mesh.batch_config3(n_instances=6, seed=7, nmin=2, nmax=5)
    B = Batch(inst)
    r = B.autotune(None, what=15, reps=2)
    assert r["colour_order"] in (0, 1, 2) and B.get_colour_order() == r["colour_order"]
    U = np.random.default_rng(1).uniform(-1e-3, 1e-3, B.ndof)
    R1 = B.residual(U)
    B.set_colour_order(0)
    R0 = B.residual(U)
    assert np.abs(R1 - R0).max() <= 1e-12 * np.abs(R0).max()


def test_autotune_batch_bit_identical(built, tmp_path):
    from igap4standard_b200 import Batch, mesh
    inst = mesh.batch_config3(n_instances=12, seed=7, nmin=2, nmax=7)
    B = Batch(inst)
    U = np.random.default_rng(1).uniform(-1e-3, 1e-3, B.ndof)
    R0, V0, W0 = B.residual(U), B.tangent(U, "fp64"), B.tangent(U, "fp32")
    r = B.autotune(None, what=7, reps=2, cache=str(tmp_path / "tune.json"))
    assert r["order"] in (0, 1) and min(r["ctas_res"], r["ctas_tan64"], r["ctas_tan32"]) >= 0
    assert B.get_schedule() == (r["ctas_res"], r["ctas_tan64"], r["ctas_tan32"], r["order"])
    assert np.array_equal(B.residual(U), R0)
    assert np.array_equal(B.tangent(U, "fp64"), V0)
    assert np.array_equal(B.tangent(U, "fp32"), W0)
