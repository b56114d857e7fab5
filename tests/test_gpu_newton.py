"""GPU Newton and CUDA-graph tests.

Newton: the reference driver's loop (src/snes_init.c, src/snes_solve.c,
restated in igap4standard_b200/newton.py) run twice from U = 0, once over the
B200 assembly and once over the reference's CPU assembly.  Criterion: same
termination reason, same number of Newton steps, and
||U_gpu - U_ref||_inf <= 1e-10 * max(||U_ref||_inf, 1).

Mixed precision: the same loop with the tangent built in FP32 (residual,
boundary rows and norms stay FP64) reaches ||F|| < 1e-10 in at most one more
step than the FP64 loop.

Graphs: a captured residual + tangent replayed on new inputs equals eager
assembly bit for bit, including parameter updates made between replays."""
import numpy as np
import pytest

from cases import make_case, neumann_values

pytestmark = pytest.mark.gpu


def _assembly(c):
    from igap4standard_b200 import Assembly
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"])
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, c["par_neumann"]))
    return A


def _ref_problem(checker, c):
    from oracle import newton_loop as newton
    case = checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                   c["par_dirichlet"], c["par_neumann"])
    return newton.case_problem(case), case.ndof


@pytest.mark.parametrize("name", ["perturbed_lame", "ragged_config0", "newton_backtrack", "config0_8"])
def test_newton_parity(built, checker, name):
    from oracle import newton_loop as newton
    c = make_case(name)
    (r_ref, j_ref), n = _ref_problem(checker, c)
    ref = newton.solve(r_ref, j_ref, np.zeros(n))
    A = _assembly(c)
    r, j = newton.assembly_problem(A, "fp64")
    got = newton.solve(r, j, np.zeros(n))
    print(name, "ref", ref.reason, ref.iterations, ref.fnorms, ref.line_search_lambdas)
    print(name, "gpu", got.reason, got.iterations, got.fnorms, got.line_search_lambdas)
    assert got.reason == ref.reason
    assert got.iterations == ref.iterations
    scale = max(np.abs(ref.U).max(), 1.0)
    assert np.abs(got.U - ref.U).max() <= 1e-10 * scale


@pytest.mark.parametrize("name", ["perturbed_lame", "config0_8", "newton_backtrack"])
def test_mixed_precision_newton(built, name):
    from oracle import newton_loop as newton
    c = make_case(name)
    A = _assembly(c)
    n = A.ndof
    r64, j64 = newton.assembly_problem(A, "fp64")
    r32, j32 = newton.assembly_problem(A, "fp32")
    a = newton.solve(r64, j64, np.zeros(n))
    b = newton.solve(r32, j32, np.zeros(n))
    print(name, "fp64", a.iterations, a.fnorms)
    print(name, "fp32 tangent", b.iterations, b.fnorms)
    assert a.converged and b.converged
    assert b.fnorms[-1] < 1e-10
    assert b.iterations <= a.iterations + 1
    assert np.abs(b.U - a.U).max() <= 1e-8 * max(np.abs(a.U).max(), 1.0)


def test_graph_replay_matches_eager(built):
    import torch
    c = make_case("perturbed_lame")
    A = _assembly(c)
    n, nnz = A.ndof, A.nnz
    dev = torch.device("cuda:0")
    U = torch.zeros(n, dtype=torch.float64, device=dev)
    R = torch.zeros(n, dtype=torch.float64, device=dev)
    V = torch.zeros(nnz, dtype=torch.float64, device=dev)
    U.copy_(torch.from_numpy(c["U"]))
    torch.cuda.synchronize()
    A.graph_capture(U.data_ptr(), R.data_ptr(), V.data_ptr(), "fp64")
    rng = np.random.default_rng(11)
    xyz, meta = A.neumann_points()
    for it in range(3):
        U1 = c["U"] + rng.uniform(-1e-3, 1e-3, n)
        pd = c["par_dirichlet"] + 0.01 * it
        pn = c["par_neumann"] * (1.0 + it)
        if it == 2:
            pn = np.zeros_like(pn)          # zero traction after nonzero: replays must see it
        A.set_par_dirichlet(pd)
        A.set_neumann_values(neumann_values(xyz, meta, pn))
        U.copy_(torch.from_numpy(U1))
        torch.cuda.synchronize()
        A.graph_launch()
        A.sync()
        R_eager = A.residual(U1)
        V_eager = A.tangent(U1, "fp64")
        assert np.array_equal(R.cpu().numpy(), R_eager)
        assert np.array_equal(V.cpu().numpy(), V_eager)
    A.graph_destroy()
