"""Device linear algebra on the tangent (igab_spmv_device, igab_solve_device).

K x against scipy's CSR product of the same values; the BiCGStab solve against
a restatement of the same iteration in torch (van der Vorst's right-
preconditioned BiCGStab, Jacobi, x0 = 0) -- equal iterates after a fixed number
of iterations, up to the rounding of the different summation orders -- and
against the tolerance it promises (||b - K x|| <= rtol ||b||, checked with
scipy); repeated solves are bitwise equal."""
import numpy as np
import pytest
import scipy.sparse as sp

from cases import make_case, make_transient_case

pytestmark = pytest.mark.gpu


def _torch_bicgstab(matvec, b, dinv, rtol, maxit=2000):
    import torch
    x = torch.zeros_like(b)
    r = b.clone()
    tol = rtol * float(b.norm())
    rhat = r.clone()
    rho = alpha = omega = 1.0
    v = torch.zeros_like(b)
    p = torch.zeros_like(b)
    for it in range(1, maxit + 1):
        rho_new = float(torch.dot(rhat, r))
        beta = (rho_new / rho) * (alpha / omega) if it > 1 else 0.0
        p = r + beta * (p - omega * v) if it > 1 else r.clone()
        phat = dinv * p
        v = matvec(phat)
        alpha = rho_new / float(torch.dot(rhat, v))
        s = r - alpha * v
        if float(s.norm()) <= tol:
            return x + alpha * phat, it
        shat = dinv * s
        t = matvec(shat)
        omega = float(torch.dot(t, s)) / float(torch.dot(t, t))
        x = x + alpha * phat + omega * shat
        r = s - omega * t
        rho = rho_new
        if float(r.norm()) <= tol:
            return x, it
    return x, maxit


def _tangent_on_device(A, U, prec):
    import torch
    Ud = torch.as_tensor(U).cuda()
    V = torch.empty(A.nnz, dtype=torch.float64 if prec == "fp64" else torch.float32, device="cuda")
    torch.cuda.synchronize()
    A.tangent_device(Ud.data_ptr(), V.data_ptr(), prec)
    A.sync()
    return V


def _transient_assembly():
    from igap4standard_b200 import Assembly, mesh
    c = make_transient_case("getime_config2")
    c["bc_type"], c["par_dirichlet"] = mesh.bc_transient()
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"],
                 phys="getime")
    A.set_history(1, c["U1"])
    A.set_history(2, c["U0"])
    return A, c


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_spmv_matches_csr_product(built, prec):
    import torch
    from igap4standard_b200 import Assembly
    c = make_case("mixed_bc")
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"])
    V = _tangent_on_device(A, c["U"], prec)
    x = np.random.default_rng(1).normal(size=A.ndof)
    xd = torch.as_tensor(x).cuda()
    yd = torch.empty_like(xd)
    torch.cuda.synchronize()
    A.spmv_device(V.data_ptr(), xd.data_ptr(), yd.data_ptr(), prec)
    A.sync()
    rp, cols = A.pattern()
    K = sp.csr_matrix((V.cpu().numpy().astype(np.float64), cols, rp), shape=(A.ndof, A.ndof))
    y_ref = K @ x
    scale = abs(K).sum(axis=1).max() * np.abs(x).max()
    assert np.abs(yd.cpu().numpy() - y_ref).max() <= 1e-13 * scale


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_solve_matches_restated_bicgstab(built, prec):
    """Five iterations of both (capped, not converged) agree to rounding -- the same
    iteration; the converged solves meet rtol on the true residual with iteration
    counts within 20% (over ~90 iterations the different summation orders of the
    dot products move BiCGStab's trajectory by a few iterations)."""
    import torch
    A, c = _transient_assembly()
    stream = torch.cuda.Stream()
    A.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        V = _tangent_on_device(A, c["U"], prec)
        b = torch.as_tensor(np.random.default_rng(2).normal(size=A.ndof)).cuda()
        x5, x = torch.empty_like(b), torch.empty_like(b)
        stream.synchronize()
        its5, ok5, _ = A.solve_device(V.data_ptr(), b.data_ptr(), x5.data_ptr(), prec, rtol=1e-10, maxit=5)
        its, ok, rnorm = A.solve_device(V.data_ptr(), b.data_ptr(), x.data_ptr(), prec, rtol=1e-10)
        rp, cols = A.pattern()
        Vh = V.cpu().numpy().astype(np.float64)
        K = sp.csr_matrix((Vh, cols, rp), shape=(A.ndof, A.ndof))
        Kt = torch.sparse_csr_tensor(torch.as_tensor(rp, dtype=torch.int64), torch.as_tensor(cols, dtype=torch.int64),
                                     torch.as_tensor(Vh), size=(A.ndof, A.ndof)).cuda()
        d = torch.as_tensor(K.diagonal()).cuda()
        dinv = torch.where(d != 0, 1.0 / d, torch.ones_like(d))
        x5_ref, _ = _torch_bicgstab(lambda v: Kt @ v, b, dinv, 1e-10, maxit=5)
        x_ref, its_ref = _torch_bicgstab(lambda v: Kt @ v, b, dinv, 1e-10)
    torch.cuda.synchronize()
    bh = b.cpu().numpy()
    d5 = np.abs(x5.cpu().numpy() - x5_ref.cpu().numpy()).max() / np.abs(x5_ref.cpu().numpy()).max()
    res = np.linalg.norm(bh - K @ x.cpu().numpy()) / np.linalg.norm(bh)
    res_ref = np.linalg.norm(bh - K @ x_ref.cpu().numpy()) / np.linalg.norm(bh)
    print("%s: 5 iterations max rel diff %.2e; iterations %d (torch restatement %d), converged %s, "
          "relative residual %.2e (restatement %.2e)" % (prec, d5, its, its_ref, ok, res, res_ref))
    assert its5 == 5 and not ok5
    assert d5 <= 1e-10
    assert ok and abs(its - its_ref) <= 0.2 * its_ref
    assert res <= 2e-10


def test_solve_deterministic_zero_rhs_and_cap(built):
    import torch
    A, c = _transient_assembly()
    stream = torch.cuda.Stream()
    A.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        V = _tangent_on_device(A, c["U"], "fp64")
        b = torch.as_tensor(np.random.default_rng(3).normal(size=A.ndof)).cuda()
        x1, x2 = torch.empty_like(b), torch.empty_like(b)
        z = torch.zeros_like(b)
        xz = torch.full_like(b, 7.0)
        x3 = torch.empty_like(b)
        stream.synchronize()
        r1 = A.solve_device(V.data_ptr(), b.data_ptr(), x1.data_ptr(), "fp64", rtol=1e-8)
        r2 = A.solve_device(V.data_ptr(), b.data_ptr(), x2.data_ptr(), "fp64", rtol=1e-8)
        rz = A.solve_device(V.data_ptr(), z.data_ptr(), xz.data_ptr(), "fp64", rtol=1e-8)
        # an iteration cap that stops the solve early is reported as not converged
        r3 = A.solve_device(V.data_ptr(), b.data_ptr(), x3.data_ptr(), "fp64", rtol=1e-14, maxit=3)
    torch.cuda.synchronize()
    assert r1 == r2 and torch.equal(x1, x2)
    assert rz[0] == 0 and rz[1] and float(xz.abs().max()) == 0.0
    assert r3[0] == 3 and not r3[1]
