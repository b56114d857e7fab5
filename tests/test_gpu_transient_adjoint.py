"""Discrete adjoint of the transient time stepping (phys/getime, element scaling
s_e = exp(g_e)) with checkpoints:
  * the history Jacobians dR/dU_hist[1], dR/dU_hist[2] against central differences
    of the reference's own getime residual (oracle/_ref) in the history levels;
  * dJ/dg of J = 1/2 sum_{face x=1} |U_N - U*|^2 after N steps, with checkpoints
    every 2 steps and segment recomputation, against central differences of the
    GPU time stepping (h = 1e-6), agreement 1e-6 relative."""
import numpy as np
import pytest
import scipy.sparse as sp

from cases import make_transient_case

pytestmark = pytest.mark.gpu

NSTEPS, EVERY = 6, 2
DT = 0.05
AMP = 0.5


def _case():
    from igap4standard_b200 import mesh
    c = make_transient_case("getime_config2")
    c["bc_type"], c["par_dirichlet"] = mesh.bc_transient()
    c["par_mat"] = c["par_mat"].copy()
    c["par_mat"][7] = DT
    return c


def _assembly(c):
    from igap4standard_b200 import Assembly
    return Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"],
                    phys="getime")


def _face_x1_mask(nelem):
    nb = np.asarray(nelem) + 2
    m = np.zeros((nb[0], nb[1], nb[2], 3))
    m[-1] = 1.0
    return m.reshape(-1)


@pytest.mark.parametrize("level", [1, 2])
def test_history_jacobian_matches_reference_differences(built, oracle_lib, level):
    import torch
    c = _case()
    A = _assembly(c)
    n = A.ndof
    rng = np.random.default_rng(3)
    U, U1, U0 = (rng.uniform(-2e-2, 2e-2, n) for _ in range(3))
    A.set_history(1, U1)
    A.set_history(2, U0)
    Ud = torch.as_tensor(U).cuda()
    V = torch.empty(A.nnz, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    A.history_jacobian_device(Ud.data_ptr(), V.data_ptr(), level, "fp64")
    A.sync()
    rp, cols = A.pattern()
    Jm = sp.csr_matrix((V.cpu().numpy(), cols, rp), shape=(n, n))
    free = np.setdiff1d(np.arange(n), A.dirichlet_rows())
    Ji = Jm[free][:, free]
    assert abs(Ji - Ji.T).max() <= 1e-12 * abs(Ji).max()      # interior block symmetric, as the tangent
    assert abs(Jm[A.dirichlet_rows()]).max() == 0.0            # Dirichlet rows do not see the history
    ref = oracle_lib.case("getime", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                          c["par_dirichlet"], np.zeros(39))
    hist = {1: U1, 2: U0}
    eps = 1e-6
    worst = 0.0
    for j in rng.choice(n, 10, replace=False):
        cols_fd = []
        for sgn in (1.0, -1.0):
            h = dict(hist)
            h[level] = hist[level].copy()
            h[level][j] += sgn * eps
            ref.set_history(1, h[1])
            ref.set_history(2, h[2])
            cols_fd.append(ref.residual(U))
        fd = (cols_fd[0] - cols_fd[1]) / (2 * eps)
        col = Jm[:, j].toarray().ravel()
        err = np.abs(fd - col).max() / max(np.abs(col).max(), 1e-30)
        worst = max(worst, err)
    print("level %d: worst column rel err %.2e" % (level, worst))
    assert worst <= 1e-6


def test_transient_adjoint_matches_central_differences(built):
    from igap4standard_b200 import transient
    c = _case()
    A = _assembly(c)
    n, ne = A.ndof, A.nelem_total
    mask = _face_x1_mask(c["nelem"])
    Ustar = np.random.default_rng(21).uniform(-1e-3, 1e-3, n)
    g0 = np.random.default_rng(5).normal(0.0, 0.3, ne)

    def J(U):
        return 0.5 * np.sum(mask * (U - Ustar) ** 2)

    out = transient.adjoint(A, NSTEPS, DT, g0, lambda U: mask * (U - Ustar), every=EVERY, rtol_lin=1e-13,
                            amplitude=AMP, abs_tol=1e-14, objective=J)
    assert out["checkpoints"] == [0, 2, 4] and out["recomputed_steps"] == NSTEPS
    info = out["info"]
    assert info["forward_converged"] == NSTEPS and info["adjoint_solves"] == NSTEPS
    assert info["adjoint_solves_converged"] == NSTEPS
    assert np.abs(out["U_N"]).max() > 1e-4            # the traction moved the body
    grad = out["grad"]

    def J_of(g):
        A.set_element_log_scale(g)
        hist, res, _ = transient.run(A, NSTEPS, DT, prec="fp64", use_graph=False, rtol_lin=1e-13,
                                     amplitude=AMP, abs_tol=1e-14)
        A.set_element_log_scale(None)
        return J(hist[-1])

    rng = np.random.default_rng(9)
    h = 1e-6
    worst = 0.0
    for k in range(4):
        d = rng.normal(size=ne)
        ad = grad @ d
        fd = (J_of(g0 + h * d) - J_of(g0 - h * d)) / (2 * h)
        err = abs(fd - ad) / max(abs(ad), 1e-3 * np.linalg.norm(grad) * np.linalg.norm(d))
        worst = max(worst, err)
        print("direction %d: adjoint %.10e  central difference %.10e  rel %.2e" % (k, ad, fd, err))
    assert worst <= 1e-6
