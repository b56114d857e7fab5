"""Batched assembly (one persistent launch per operator over many meshes): every
instance's slice of the batched residual and tangent equals that instance's
single-mesh assembly bit for bit (same per-entry accumulation order), for every
schedule, and through a captured CUDA graph."""
import numpy as np
import pytest

from igap4standard_b200 import mesh

pytestmark = pytest.mark.gpu


def _instances(seed=11):
    rng = np.random.default_rng(seed)
    sizes = [(1, 1, 1), (2, 3, 5), (4, 4, 4), (3, 1, 2), (6, 5, 7), (2, 2, 2), (5, 3, 3), (7, 6, 4)]
    out = []
    for k, ne in enumerate(sizes):
        lam, mu = np.exp(rng.normal(0.0, 0.25, 2))
        pm = mesh.par_mat_from_lame(lam, mu, rng.uniform(0.05, 0.2)) if k % 3 else mesh.PAR_MAT_DEFAULT.copy()
        if k % 4 == 1:
            bc, pd = mesh.bc_example()
        elif k % 4 == 2:
            bc = rng.integers(0, 2, 36).astype(np.int32)
            pd = rng.uniform(-0.05, 0.05, 9)
        else:
            bc, pd = mesh.bc_config0()
        pp = rng.uniform(-0.01, 0.01, 9) if k == 5 else np.zeros(9)
        out.append(dict(nelem=ne, knots=mesh.knots_for(ne, perturb=0.1, seed=k), par_mat=pm, bc_type=bc,
                        par_dirichlet=pd, par_periodic=pp))
    return out


def _single(c, U, prec, colour_order=0):
    from igap4standard_b200 import Assembly
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"])
    A.set_option(3, colour_order)
    R = A.residual(U)
    V = A.tangent(U, prec)
    A.close()
    return R, V


@pytest.fixture(scope="module")
def batch_case(built):
    from igap4standard_b200 import Batch
    inst = _instances()
    B = Batch(inst)
    U = np.random.default_rng(5).uniform(-2e-3, 2e-3, B.ndof)
    return inst, B, U


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_batch_equals_single_mesh(batch_case, prec):
    inst, B, U = batch_case
    R = B.residual(U)
    V = B.tangent(U, prec)
    assert B.last_launch_count() >= 1
    for i, c in enumerate(inst):
        d0, d1 = B.dof_offsets[i], B.dof_offsets[i + 1]
        z0, z1 = B.nnz_offsets[i], B.nnz_offsets[i + 1]
        R1, V1 = _single(c, U[d0:d1], prec)
        assert np.array_equal(R[d0:d1], R1), "instance %d residual" % i
        assert np.array_equal(V[z0:z1], V1), "instance %d tangent (%s)" % (i, prec)


@pytest.mark.parametrize("colour_order", [1, 2])
def test_batch_colour_orders_equal_single_mesh(batch_case, colour_order):
    """Under each colour order the batch (waits by sweep position) equals the single-mesh
    assembly swept in the same order, bit for bit."""
    inst, B, U = batch_case
    B.set_colour_order(colour_order)
    assert B.get_colour_order() == colour_order
    R, V, W = B.residual(U), B.tangent(U, "fp64"), B.tangent(U, "fp32")
    B.set_colour_order(0)
    for i, c in enumerate(inst):
        d0, d1 = B.dof_offsets[i], B.dof_offsets[i + 1]
        z0, z1 = B.nnz_offsets[i], B.nnz_offsets[i + 1]
        R1, V1 = _single(c, U[d0:d1], "fp64", colour_order)
        _, W1 = _single(c, U[d0:d1], "fp32", colour_order)
        assert np.array_equal(R[d0:d1], R1) and np.array_equal(V[z0:z1], V1) and np.array_equal(W[z0:z1], W1), i


@pytest.mark.parametrize("sched", [(1, 1, 1, 0), (0, 0, 0, 1), (1, 1, 1, 1)])
def test_batch_schedules_agree(batch_case, sched):
    inst, B, U = batch_case
    B.set_schedule(0, 0, 0, 0)
    R0, V0, W0 = B.residual(U), B.tangent(U, "fp64"), B.tangent(U, "fp32")
    B.set_schedule(*sched)
    assert B.get_schedule() == sched
    R1, V1, W1 = B.residual(U), B.tangent(U, "fp64"), B.tangent(U, "fp32")
    B.set_schedule(0, 0, 0, 0)
    assert np.array_equal(R0, R1) and np.array_equal(V0, V1) and np.array_equal(W0, W1)


def test_batch_graph_replay(batch_case):
    import torch
    inst, B, U = batch_case
    R_ref, V_ref = B.residual(U), B.tangent(U, "fp32")
    Ud = torch.as_tensor(U).cuda()
    Rd = torch.zeros(B.ndof, dtype=torch.float64, device="cuda")
    Vd = torch.zeros(B.nnz, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    B.graph_capture(Ud.data_ptr(), Rd.data_ptr(), Vd.data_ptr(), "fp32")
    for _ in range(2):
        B.graph_launch()
    B.sync()
    assert np.array_equal(Rd.cpu().numpy(), R_ref)
    assert np.array_equal(Vd.cpu().numpy(), V_ref)


def test_batch_config3_shapes(built):
    """A slice of the 512-instance workload generator (sizes 6..24 per side)."""
    from igap4standard_b200 import Batch
    inst = mesh.batch_config3(n_instances=6, seed=3)
    assert all(6 <= n <= 24 for c in inst for n in c["nelem"])
    B = Batch(inst)
    assert B.ndof == sum(mesh.n_dof(c["nelem"]) for c in inst)
    assert B.nnz == sum(mesh.nnz_of(c["nelem"]) for c in inst)
    U = np.random.default_rng(0).uniform(-1e-3, 1e-3, B.ndof)
    R = B.residual(U)
    i = 2
    d0, d1 = B.dof_offsets[i], B.dof_offsets[i + 1]
    R1, _ = _single(dict(inst[i], par_periodic=np.zeros(9)), U[d0:d1], "fp64")
    assert np.array_equal(R[d0:d1], R1)


@pytest.mark.parametrize("op", ["residual", "fp64", "fp32"])
def test_batch_wait_gives_up_and_recovers(built, op):
    """A colour-dependency wait that cannot finish (its target count is raised past
    what the tiles publish) gives up after its poll limit: the launch ends,
    igab_batch_sync reports status 2, and the next launch is correct again."""
    import torch
    from igap4standard_b200 import Batch
    inst = _instances()[2:5]              # (4,4,4), (3,1,2), (6,5,7): several tiles per colour
    B = Batch(inst)
    U = np.random.default_rng(9).uniform(-1e-3, 1e-3, B.ndof)
    ref = B.residual(U) if op == "residual" else B.tangent(U, op)
    Ud = torch.as_tensor(U).cuda()
    out = torch.zeros(ref.size, dtype=torch.float32 if op == "fp32" else torch.float64, device="cuda")
    torch.cuda.synchronize()
    B.set_wait_limit(64, unreachable=True)
    if op == "residual":
        B.residual_device(Ud.data_ptr(), out.data_ptr())
    else:
        B.tangent_device(Ud.data_ptr(), out.data_ptr(), op)
    rc = B.lib.igab_batch_sync(B.h)
    assert rc == 2, "the unreachable wait did not report"
    assert b"status 2" in B.lib.igab_last_error()
    B.set_wait_limit(0, unreachable=False)
    again = B.residual(U) if op == "residual" else B.tangent(U, op)
    assert np.array_equal(again, ref)
    B.close()


@pytest.mark.slow
def test_batch_config3_against_reference(built, checker):
    """Batched results at the 512-instance workload's sizes (n^3, n in 6..24, each
    instance with its own lambda, mu, l) against the reference's own CPU assembly:
    the residual of every instance of an 8-instance draw, and the FP64 (entrywise
    1e-12) and FP32 (rowwise 1e-5) tangents of its two 6^3 instances."""
    from cases import residual_tolerance, tangent_tolerance
    from igap4standard_b200 import Batch
    inst = mesh.batch_config3(n_instances=8, seed=3)
    B = Batch(inst)
    U = np.random.default_rng(3).uniform(-1e-3, 1e-3, B.ndof)
    R = B.residual(U)
    V = B.tangent(U, "fp64")
    W = B.tangent(U, "fp32").astype(np.float64)
    small = [i for i, c in enumerate(inst) if c["nelem"][0] == 6]
    assert len(small) == 2
    for i, c in enumerate(inst):
        d0, d1 = B.dof_offsets[i], B.dof_offsets[i + 1]
        ref = checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], np.zeros(9),
                      c["par_dirichlet"], np.zeros(39))
        R_ref = ref.residual(U[d0:d1])
        assert np.all(np.abs(R[d0:d1] - R_ref) <= residual_tolerance(R_ref)), "instance %d residual" % i
        if i not in small:
            continue
        rp, cols, v_ref = ref.tangent(U[d0:d1])
        z0, z1 = B.nnz_offsets[i], B.nnz_offsets[i + 1]
        rp_b, cols_b = B.pattern(i)
        assert np.array_equal(rp_b, rp) and np.array_equal(cols_b, cols)
        assert np.all(np.abs(V[z0:z1] - v_ref) <= tangent_tolerance(rp, v_ref)), "instance %d FP64 tangent" % i
        rowmax = np.maximum.reduceat(np.abs(v_ref), rp[:-1])
        err = np.maximum.reduceat(np.abs(W[z0:z1] - v_ref), rp[:-1])
        assert np.max(err / rowmax) <= 1e-5, "instance %d FP32 tangent" % i
    B.close()
