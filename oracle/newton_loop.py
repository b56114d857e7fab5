"""Newton driver with the reference application's solver semantics -- test
infrastructure: the parity tests run the reference's CPU assembly and the GPU
assembly through this same host loop; nothing in the product imports it.

IGAP4STANDARD solves R(U) = 0 with PETSc SNES configured in src/snes_init.c:
NEWTONLS (:19), backtracking line search of cubic order (:21-22), absolute
tolerance 1e-10 and relative/step tolerances 1e-20 (:18), one Newton step per
SNESSolve (max_it = 1, :18).  src/snes_solve.c:23-33 repeats SNESSolve until
the reason is not "max iterations", and stops early when ||F|| stagnates
(|F_old - F_new| / F_old < 1e-6, with F_old = 999 before the first pass).

This module restates that loop around any residual/tangent pair (the B200
assembly, or the reference's own CPU assembly in the tests), so both sides of
a parity test run the same driver.  Two deliberate differences from PETSc:
the linear solve is a sparse direct factorisation (the reference's GMRES +
ASM with default rtol 1e-5 is an inexact solve whose arithmetic PETSc owns),
and there is no SNESSetFromOptions.  The line search is the backtracking
algorithm of Dennis & Schnabel, "Numerical Methods for Unconstrained
Optimization and Nonlinear Equations" (1983), Alg. A6.3.1, with the
quadratic first backtrack and the step-length safeguards [0.1, 0.5] that
SNESLINESEARCHBT uses.
"""
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

ABS_TOL = 1e-10        # SNESSetTolerances abstol, src/snes_init.c:18
REL_TOL = 1e-20        # rtol, src/snes_init.c:18
STEP_TOL = 1e-20       # stol, src/snes_init.c:18
STAGNATION = 1e-6      # src/snes_solve.c:29
MAX_SUBITER = 10000    # src/snes_solve.c:24

CONVERGED_FNORM_ABS = 2
CONVERGED_FNORM_RELATIVE = 3
CONVERGED_SNORM_RELATIVE = 4
DIVERGED_FNORM_NAN = -4
DIVERGED_MAX_IT = -5
DIVERGED_LINE_SEARCH = -6


@dataclass
class NewtonResult:
    U: np.ndarray
    converged: bool
    reason: int
    iterations: int                                   # Newton steps taken (= subiterations)
    fnorms: list = field(default_factory=list)        # ||F|| after each subiteration
    n_residual: int = 0
    n_tangent: int = 0
    line_search_lambdas: list = field(default_factory=list)


def _norm(v):
    """2-norm of a numpy array or a torch tensor (device-resident drivers pass tensors)."""
    if hasattr(v, "detach"):
        return float(v.norm())
    return float(np.linalg.norm(v))


class _Counted:
    def __init__(self, fn):
        self.fn, self.n = fn, 0

    def __call__(self, *a):
        self.n += 1
        return self.fn(*a)


def backtrack(residual, X, F, fnorm, Y, JY, alpha=1e-4, minlambda=1e-12, maxstep=1e8, max_its=40):
    """Backtracking along X - lambda*Y.  Returns (X_new, F_new, fnorm_new, lambda, ok).

    JY is J @ Y with the Jacobian the step was solved with; the slope of
    0.5||F||^2 along -Y is -(F, JY), forced negative as PETSc does."""
    ynorm = _norm(Y)
    if ynorm > maxstep:
        Y = Y * (maxstep / ynorm)
        JY = JY * (maxstep / ynorm)
    initslope = float(F @ JY)
    if initslope > 0.0:
        initslope = -initslope
    if initslope == 0.0:
        initslope = -1.0
    lam = 1.0
    W = X - Y
    G = residual(W)
    gnorm = _norm(G)
    if not np.isfinite(gnorm):
        return W, G, gnorm, lam, False
    if 0.5 * gnorm * gnorm <= 0.5 * fnorm * fnorm + lam * alpha * initslope:
        return W, G, gnorm, lam, True
    # quadratic first backtrack
    lamtemp = -initslope / (gnorm * gnorm - fnorm * fnorm - 2.0 * lam * initslope)
    lamtemp = min(lamtemp, 0.5 * lam)
    lam = 0.1 * lam if lamtemp <= 0.1 * lam else lamtemp
    W = X - lam * Y
    G = residual(W)
    gprev, lamprev = gnorm, 1.0
    gnorm = _norm(G)
    if np.isfinite(gnorm) and 0.5 * gnorm * gnorm <= 0.5 * fnorm * fnorm + lam * alpha * initslope:
        return W, G, gnorm, lam, True
    # cubic backtracks
    for _ in range(max_its):
        if lam <= minlambda:
            break
        t1 = 0.5 * (gnorm * gnorm - fnorm * fnorm) - lam * initslope
        t2 = 0.5 * (gprev * gprev - fnorm * fnorm) - lamprev * initslope
        a = (t1 / (lam * lam) - t2 / (lamprev * lamprev)) / (lam - lamprev)
        b = (-lamprev * t1 / (lam * lam) + lam * t2 / (lamprev * lamprev)) / (lam - lamprev)
        d = max(b * b - 3.0 * a * initslope, 0.0)
        lamtemp = -initslope / (2.0 * b) if a == 0.0 else (-b + np.sqrt(d)) / (3.0 * a)
        lamprev, gprev = lam, gnorm
        lamtemp = min(lamtemp, 0.5 * lam)
        lam = 0.1 * lam if lamtemp <= 0.1 * lam else lamtemp
        W = X - lam * Y
        G = residual(W)
        gnorm = _norm(G)
        if np.isfinite(gnorm) and 0.5 * gnorm * gnorm <= 0.5 * fnorm * fnorm + lam * alpha * initslope:
            return W, G, gnorm, lam, True
    return W, G, gnorm, lam, False


def direct_solve(J, F):
    """J Y = F by sparse LU (SuperLU); J is a scipy CSR matrix."""
    return spla.spsolve(sp.csc_matrix(J), F)


def solve(residual, jacobian, U0, linear_solve=direct_solve, max_subiter=MAX_SUBITER, log=None):
    """Run the reference driver's subiteration loop from U0.

    residual(U) -> F (ndarray), jacobian(U) -> scipy sparse matrix (the
    assembled tangent with Dirichlet rows/columns already zeroed, diagonal 1).
    """
    residual = _Counted(residual)
    jacobian = _Counted(jacobian)
    X = np.array(U0, dtype=np.float64, copy=True)
    res = NewtonResult(U=X, converged=False, reason=DIVERGED_MAX_IT, iterations=0)
    f_old = 999.0
    reason = DIVERGED_MAX_IT
    for _ in range(max_subiter):
        # one SNESSolve with max_it = 1
        F = residual(X)
        fnorm = float(np.linalg.norm(F))
        if not np.isfinite(fnorm):
            reason = DIVERGED_FNORM_NAN
        elif fnorm < ABS_TOL:
            reason = CONVERGED_FNORM_ABS
        else:
            ttol = fnorm * REL_TOL
            J = jacobian(X)
            Y = linear_solve(J, F)
            JY = J @ Y
            xnorm = np.linalg.norm(X)
            X, F, fnorm, lam, ok = backtrack(residual, X, F, fnorm, Y, JY)
            res.line_search_lambdas.append(lam)
            res.iterations += 1
            snorm = lam * np.linalg.norm(Y)
            if not ok:
                reason = DIVERGED_LINE_SEARCH
            elif not np.isfinite(fnorm):
                reason = DIVERGED_FNORM_NAN
            elif fnorm < ABS_TOL:
                reason = CONVERGED_FNORM_ABS
            elif fnorm <= ttol:
                reason = CONVERGED_FNORM_RELATIVE
            elif snorm < STEP_TOL * xnorm:
                reason = CONVERGED_SNORM_RELATIVE
            else:
                reason = DIVERGED_MAX_IT
        # src/snes_solve.c:29-32
        f_new = fnorm
        if abs(f_old - f_new) / f_old < STAGNATION:
            reason = DIVERGED_LINE_SEARCH
        f_old = f_new
        res.fnorms.append(f_new)
        if log:
            log("%6d: Fnorm = %e" % (len(res.fnorms), f_new))
        if reason != DIVERGED_MAX_IT:
            break
    res.U = X
    res.reason = reason
    res.converged = reason > 0
    res.n_residual = residual.n
    res.n_tangent = jacobian.n
    return res


def assembly_problem(A, prec="fp64"):
    """(residual, jacobian) of a B200 Assembly; prec "fp32" builds the tangent in FP32."""
    rowptr, cols = A.pattern()
    n = A.ndof

    def residual(U):
        return A.residual(U)

    def jacobian(U):
        v = A.tangent(U, prec)
        return sp.csr_matrix((v.astype(np.float64, copy=False), cols, rowptr), shape=(n, n))

    return residual, jacobian


def case_problem(case):
    """(residual, jacobian) of a Case (drop-in or reference callbacks through PETSc-style objects)."""
    n = case.ndof

    def jacobian(U):
        rp, cols, vals = case.tangent(U)
        return sp.csr_matrix((vals, cols, rp), shape=(n, n))

    return case.residual, jacobian
