"""CPU tests of the Newton driver (igap4standard_b200/newton.py): the line
search and the subiteration loop of src/snes_solve.c, on analytic systems and
on the reference's own CPU assembly."""
import numpy as np
import scipy.sparse as sp

from cases import make_case


def _system(a):
    """F_i(x) = x_i^3 + x_i - a_i (unique root, Newton from 0 takes damped steps for large a)."""
    def residual(x):
        return x ** 3 + x - a

    def jacobian(x):
        return sp.diags(3 * x ** 2 + 1).tocsr()
    return residual, jacobian


def test_backtrack_armijo_and_safeguards():
    from oracle import newton_loop as newton
    a = np.array([50.0, -30.0, 1.0])
    residual, jacobian = _system(a)
    X = np.zeros(3)
    F = residual(X)
    fnorm = np.linalg.norm(F)
    J = jacobian(X)
    Y = newton.direct_solve(J, F)
    W, G, gnorm, lam, ok = newton.backtrack(residual, X, F, fnorm, Y, J @ Y)
    assert ok
    assert lam < 1.0                                  # the full step x = a overshoots
    assert 0.5 * gnorm ** 2 <= 0.5 * fnorm ** 2 - 1e-4 * lam * fnorm ** 2
    assert np.allclose(W, X - lam * Y)


def test_solve_converges_to_abs_tol():
    from oracle import newton_loop as newton
    a = np.linspace(-40, 40, 17)
    residual, jacobian = _system(a)
    res = newton.solve(residual, jacobian, np.zeros(a.size))
    assert res.converged and res.reason == newton.CONVERGED_FNORM_ABS
    assert res.fnorms[-1] < newton.ABS_TOL
    assert len(res.fnorms) == res.iterations
    assert res.n_tangent == res.iterations
    assert np.allclose(res.U ** 3 + res.U, a)


def test_already_converged_takes_no_step():
    from oracle import newton_loop as newton
    residual, jacobian = _system(np.zeros(4))
    res = newton.solve(residual, jacobian, np.zeros(4))
    assert res.converged and res.iterations == 0 and res.n_tangent == 0


def test_stagnation_stops_loop():
    """|F_old - F_new| / F_old < 1e-6 ends the loop as a line-search failure
    (src/snes_solve.c:29): a residual whose norm Newton cannot change."""
    from oracle import newton_loop as newton

    def residual(x):
        return np.array([1.0, 0.0]) + 0.0 * x

    def jacobian(x):
        return sp.identity(2, format="csr")
    res = newton.solve(residual, jacobian, np.zeros(2), max_subiter=50)
    assert not res.converged
    assert res.reason == newton.DIVERGED_LINE_SEARCH
    assert res.iterations <= 2


def test_newton_on_reference_assembly(checker):
    """The driver over the reference's CPU callbacks: backtracking first steps, then quadratic convergence."""
    from oracle import newton_loop as newton
    c = make_case("newton_backtrack")
    case = checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                   c["par_dirichlet"], c["par_neumann"])
    r, j = newton.case_problem(case)
    res = newton.solve(r, j, np.zeros(case.ndof))
    assert res.converged
    assert min(res.line_search_lambdas) < 1.0
    assert res.fnorms[-1] < 1e-10
    assert res.fnorms[-2] > res.fnorms[-1]
