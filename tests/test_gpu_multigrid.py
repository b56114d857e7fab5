"""Multigrid-preconditioned GMRES and CG on the assembled tangent (igab_solve_mg_device).

  * 8^3 (two levels, dense coarsest): both methods' solutions equal scipy's sparse direct
    solve of the same CSR system to 1e-9 relative;
  * 16^3 and 32^3 of the config-1 workload (perturbed knots), at a nonzero state and with
    element scales exp(g), g ~ N(0, 0.3^2): the true residual ||b - K x|| (scipy's CSR
    product) meets the tolerance and the iteration count stays small where the Jacobi
    BiCGStab of igab_solve_device needs thousands; CG at the zero state likewise;
  * repeated solves are bitwise equal; a changed material rebuilds the hierarchy."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from igap4standard_b200 import mesh

pytestmark = pytest.mark.gpu


def _problem(n, scales=False, seed=0, amp=1e-3):
    import torch
    from igap4standard_b200 import Assembly
    nelem = (n, n, n)
    A = Assembly(nelem, mesh.knots_for(nelem, perturb=0.1, seed=1), mesh.par_mat_from_lame(1.0, 1.0, 0.1),
                 *mesh.bc_config0())
    st = torch.cuda.Stream()
    A.set_stream(st.cuda_stream)
    if scales:
        A.set_element_log_scale(np.random.default_rng(4).normal(0.0, 0.3, A.nelem_total))
    rng = np.random.default_rng(seed)
    U = torch.as_tensor(rng.uniform(-amp, amp, A.ndof)).cuda()
    b = torch.as_tensor(rng.normal(size=A.ndof)).cuda()
    return A, st, U, b


def _solve(A, st, U, b, prec="fp64", rtol=1e-8, method="gmres"):
    import torch
    V = torch.empty(A.nnz, dtype=torch.float64 if prec == "fp64" else torch.float32, device="cuda")
    x = torch.zeros(A.ndof, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    A.tangent_device(U.data_ptr(), V.data_ptr(), prec)
    A.sync()
    its, ok, rn, lev = A.solve_mg_device(V.data_ptr(), b.data_ptr(), x.data_ptr(), prec, rtol, 0.0, 500, method)
    return V.cpu().numpy().astype(np.float64), x.cpu().numpy(), its, ok, rn, lev


@pytest.mark.parametrize("method", ["gmres", "cg"])
def test_mg_matches_direct_solve_8cubed(built, method):
    A, st, U, b = _problem(8)
    v, x, its, ok, rn, lev = _solve(A, st, U, b, rtol=1e-12, method=method)
    rp, cols = A.pattern()
    K = sp.csr_matrix((v, cols, rp), shape=(A.ndof, A.ndof))
    x_ref = spla.spsolve(K.tocsc(), b.cpu().numpy())
    print("8^3: levels %d, iterations %d, residual %.3e" % (lev, its, rn))
    assert ok and lev == 2
    assert np.abs(x - x_ref).max() <= 1e-9 * np.abs(x_ref).max()


@pytest.mark.parametrize("n,scales,prec", [(16, False, "fp64"), (16, True, "fp32"), (32, True, "fp64")])
def test_mg_converges_in_few_iterations(built, n, scales, prec):
    """16^3 at a rough state (control values uniform in +-1e-3); 32^3 at the Newton start of
    the workload (affine field with the Dirichlet rows at their values)."""
    import torch
    A, st, U, b = _problem(n, scales)
    if n == 32:
        U = torch.as_tensor(A.affine_start(mesh.knots_for((n, n, n), perturb=0.1, seed=1),
                                           mesh.bc_config0()[1])).cuda()
    v, x, its, ok, rn, lev = _solve(A, st, U, b, prec, rtol=1e-8)
    rp, cols = A.pattern()
    K = sp.csr_matrix((v, cols, rp), shape=(A.ndof, A.ndof))
    bh = b.cpu().numpy()
    true_res = np.linalg.norm(bh - K @ x) / np.linalg.norm(bh)
    print("%d^3 %s scales=%s: levels %d, iterations %d, true relative residual %.2e" % (n, prec, scales, lev, its,
                                                                                         true_res))
    assert ok and true_res <= 2e-8
    assert its <= 100
    assert lev == {16: 3, 32: 4}[n]


def test_mg_cg_at_zero_state_32cubed(built):
    A, st, U, b = _problem(32, amp=0.0)
    v, x, its, ok, rn, lev = _solve(A, st, U, b, rtol=1e-8, method="cg")
    rp, cols = A.pattern()
    K = sp.csr_matrix((v, cols, rp), shape=(A.ndof, A.ndof))
    bh = b.cpu().numpy()
    true_res = np.linalg.norm(bh - K @ x) / np.linalg.norm(bh)
    print("32^3 CG at U = 0: levels %d, iterations %d, true relative residual %.2e" % (lev, its, true_res))
    assert ok and true_res <= 2e-8 and its <= 60


def test_mg_repeatable_and_rebuilt(built):
    import torch
    A, st, U, b = _problem(16)
    _, x1, its1, _, _, _ = _solve(A, st, U, b)
    _, x2, its2, _, _, _ = _solve(A, st, U, b)
    assert its1 == its2 and np.array_equal(x1, x2)
    A.set_par_mat(mesh.par_mat_from_lame(2.0, 0.5, 0.1))     # new material: new coarse tangents
    v, x3, its3, ok, _, _ = _solve(A, st, U, b)
    rp, cols = A.pattern()
    K = sp.csr_matrix((v, cols, rp), shape=(A.ndof, A.ndof))
    bh = b.cpu().numpy()
    assert ok and np.linalg.norm(bh - K @ x3) <= 2e-8 * np.linalg.norm(bh)
