"""Device-resident time stepping of the transient physics (phys/getime) with the
reference application's solver semantics.

Per time step the reference example (example/ex1/main.c:48-56) takes the
previous solution as initial guess (initguess, :116-126), runs snes_solve
(src/snes_solve.c:23-33: one Newton step per SNESSolve, absolute ||F||_2 <=
1e-10, stagnation stop) and shifts the history levels, U_hist[k] <- U_hist[k-1]
for k = torder..1 (:55).  This module does the same on the GPU:

  - the residual + tangent assembly of one Newton iteration is captured once in a
    CUDA graph at fixed device buffers (the iterate lives in the captured U
    buffer) and replayed every iteration; history levels and tractions are
    updated in place, which replays pick up;
  - the line search is newton.backtrack (Dennis & Schnabel A6.3.1, as PETSc's
    SNESLINESEARCHBT), on device tensors;
  - the linear solve is the library's device BiCGStab (igab_solve_device:
    Jacobi-preconditioned, van der Vorst, SIAM J. Sci. Stat. Comput. 13 (1992)
    631-644; scalars and the stop test on the device, iterations replayed as a
    CUDA graph).  The reference solves with PETSc GMRES + ASM
    (src/snes_init.c:24-39), which is outside the assembly path; this solver is
    the driver's stand-in for it.

The traction of the transient workload is 0.01 sin(2 pi t) on face x = 1 in
the x direction (face 1, standard order, dof 0), evaluated at t_{n+1}.
"""
import numpy as np

from . import newton


def _torch():
    import torch
    return torch


class DeviceProblem:
    """Residual / tangent / K x of one Assembly on device tensors (FP64 vectors)."""

    def __init__(self, A, prec="fp32", use_graph=True):
        torch = _torch()
        self.A, self.prec = A, prec
        self.dev = torch.device("cuda", A.device)
        # a dedicated stream (graph capture needs one); torch vector work runs on it too
        self.stream = torch.cuda.Stream(device=self.dev)
        A.set_stream(self.stream.cuda_stream)
        n, nnz = A.ndof, A.nnz
        with torch.cuda.stream(self.stream):
            self.X = torch.zeros(n, dtype=torch.float64, device=self.dev)     # captured U buffer (the iterate)
            self.R = torch.zeros(n, dtype=torch.float64, device=self.dev)
            self.V = torch.zeros(nnz, dtype=torch.float64 if prec == "fp64" else torch.float32, device=self.dev)
            self.Rt = torch.zeros(n, dtype=torch.float64, device=self.dev)    # line-search residuals
        self.stream.synchronize()
        rowptr, cols = A.pattern()
        rows = np.repeat(np.arange(n), np.diff(rowptr))
        self.diag_pos = torch.as_tensor(np.nonzero(cols == rows)[0], device=self.dev)
        self.use_graph = use_graph
        self.captured = False
        self.n_assembly = 0
        self.n_residual = 0
        self.krylov_its = []

    def capture(self):
        torch = _torch()
        torch.cuda.synchronize(self.dev)
        self.A.graph_capture(self.X.data_ptr(), self.R.data_ptr(), self.V.data_ptr(), self.prec)
        self.captured = True

    def assemble(self):
        """R and the tangent at the iterate X (graph replay or eager launches)."""
        if self.use_graph:
            if not self.captured:
                self.capture()
            self.A.graph_launch()
        else:
            self.A.residual_device(self.X.data_ptr(), self.R.data_ptr())
            self.A.tangent_device(self.X.data_ptr(), self.V.data_ptr(), self.prec)
        self.n_assembly += 1
        return self.R

    def residual(self, W):
        torch = _torch()
        W = W.contiguous()
        out = torch.empty_like(self.Rt)
        self.A.residual_device(W.data_ptr(), out.data_ptr())
        self.n_residual += 1
        return out

    def matvec(self, x, y=None):
        """K x on the device (igab_spmv_device)."""
        torch = _torch()
        x = x.contiguous()
        y = torch.empty_like(x) if y is None else y
        self.A.spmv_device(self.V.data_ptr(), x.data_ptr(), y.data_ptr(), self.prec)
        return y

    def solve(self, b, rtol, maxit=2000):
        """K^-1 b by the library's device BiCGStab (Jacobi); returns (x, iterations, converged)."""
        torch = _torch()
        b = b.contiguous()
        x = torch.empty_like(b)
        its, ok, _ = self.A.solve_device(self.V.data_ptr(), b.data_ptr(), x.data_ptr(), self.prec, rtol, 0.0, maxit)
        return x, its, ok

    def diagonal(self):
        return self.V[self.diag_pos].to(_torch().float64)


def newton_device(P, rtol_lin=1e-5, max_subiter=newton.MAX_SUBITER, abs_tol=newton.ABS_TOL):
    """snes_solve semantics on device tensors; the iterate is P.X (updated in place).
    abs_tol: the absolute ||F|| test (1e-10 in the reference, src/snes_init.c:18)."""
    torch = _torch()
    res = newton.NewtonResult(U=None, converged=False, reason=newton.DIVERGED_MAX_IT, iterations=0)
    f_old = 999.0
    reason = newton.DIVERGED_MAX_IT
    for _ in range(max_subiter):
        F = P.assemble().clone()
        fnorm = float(F.norm())
        if not np.isfinite(fnorm):
            reason = newton.DIVERGED_FNORM_NAN
        elif fnorm < abs_tol:
            reason = newton.CONVERGED_FNORM_ABS
        else:
            ttol = fnorm * newton.REL_TOL
            Y, its, _ = P.solve(F, rtol_lin)
            P.krylov_its.append(its)
            JY = P.matvec(Y)
            xnorm = float(P.X.norm())
            Xn, F, fnorm, lam, ok = newton.backtrack(P.residual, P.X, F, fnorm, Y, JY)
            P.X.copy_(Xn)
            res.line_search_lambdas.append(lam)
            res.iterations += 1
            snorm = lam * float(Y.norm())
            if not ok:
                reason = newton.DIVERGED_LINE_SEARCH
            elif not np.isfinite(fnorm):
                reason = newton.DIVERGED_FNORM_NAN
            elif fnorm < abs_tol:
                reason = newton.CONVERGED_FNORM_ABS
            elif fnorm <= ttol:
                reason = newton.CONVERGED_FNORM_RELATIVE
            elif snorm < newton.STEP_TOL * xnorm:
                reason = newton.CONVERGED_SNORM_RELATIVE
            else:
                reason = newton.DIVERGED_MAX_IT
        if abs(f_old - fnorm) / f_old < newton.STAGNATION:   # src/snes_solve.c:29
            reason = newton.DIVERGED_LINE_SEARCH
        f_old = fnorm
        res.fnorms.append(fnorm)
        if reason != newton.DIVERGED_MAX_IT:
            break
    res.reason = reason
    res.converged = reason > 0
    return res


def traction_values(A, t, amplitude=0.01, face=1, order=0, dof=0):
    """Surface-point values of the transient traction amplitude sin(2 pi t) on (face, order, dof)."""
    xyz, meta = A.neumann_points()
    val = amplitude * np.sin(2.0 * np.pi * t)
    sel = (meta[:, 0] == face) & (meta[:, 1] == order) & (meta[:, 2] == dof)
    return np.where(sel, val, 0.0)


def run(A, nsteps, dt, prec="fp32", use_graph=True, rtol_lin=1e-5, traction=traction_values, U_init=None,
        U_prev=None, callback=None, abs_tol=newton.ABS_TOL):
    """Time-step A (an Assembly with phys="getime") nsteps times from the history
    (U_init at t_0, U_prev at t_{-1}; zeros by default).  Returns (history of U per
    step as host arrays, per-step NewtonResults, DeviceProblem)."""
    torch = _torch()
    P = DeviceProblem(A, prec, use_graph)
    with torch.cuda.stream(P.stream):
        return _run(P, A, nsteps, dt, rtol_lin, traction, U_init, U_prev, callback, abs_tol)


def _run(P, A, nsteps, dt, rtol_lin, traction, U_init, U_prev, callback, abs_tol=newton.ABS_TOL):
    torch = _torch()
    n = A.ndof
    h1 = torch.zeros(n, dtype=torch.float64, device=P.dev)   # U at t_n     (U_hist level 1)
    h0 = torch.zeros(n, dtype=torch.float64, device=P.dev)   # U at t_{n-1} (U_hist level 2)
    if U_init is not None:
        h1.copy_(torch.as_tensor(np.asarray(U_init, dtype=np.float64)))
    if U_prev is not None:
        h0.copy_(torch.as_tensor(np.asarray(U_prev, dtype=np.float64)))
    hist, results = [], []
    for step in range(nsteps):
        t = (step + 1) * dt
        A.set_neumann_values(traction(A, t))
        A.set_history_device(1, h1.data_ptr())
        A.set_history_device(2, h0.data_ptr())
        P.X.copy_(h1)                                   # initguess: U <- U_hist[1]
        r = newton_device(P, rtol_lin=rtol_lin, abs_tol=abs_tol)
        results.append(r)
        h0.copy_(h1)                                    # history shift (main.c:55)
        h1.copy_(P.X)
        hist.append(P.X.cpu().numpy())
        if callback:
            callback(step, r)
    return hist, results, P


# ---------------------------------------------------------------------------
# Discrete adjoint of the time stepping (element-scaled problem, s_e = exp(g_e))
#
# Steps n = 0..N-1 solve R_n(U_{n+1}; U_n, U_{n-1}, g) = 0 (levels: U_hist[1] = U_n,
# U_hist[2] = U_{n-1}).  For an objective J(U_N), with L = J - sum_n lam_n . R_n,
#   K_n^T lam_n = b_n,  b_n = dJ/dU_{n+1} - J1_{n+1}^T lam_{n+1} - J0_{n+2}^T lam_{n+2},
#   dJ/dg = - sum_n lam_n . dR_n/dg,
# K_n = dR_n/dU_{n+1} (the tangent), J1_n = dR_n/dU_n, J0_n = dR_n/dU_{n-1} (the history
# Jacobians, igab_history_jacobian_device).  The Dirichlet rows of R_n do not depend on
# g or on the history, so lam is zero there (b is zeroed on those rows; K is the
# symmetric-eliminated tangent, identity there).  States are kept at checkpoints every
# `every` steps (U_{s-1}, U_s) and each segment is recomputed forward before its
# backward sweep, so memory is O(N / every + every) states.


def _sym_solve(P, b, rtol):
    """K^T x = b for the symmetric tangent (Dirichlet rows and columns eliminated)."""
    x, its, ok = P.solve(b, rtol)
    return x


def _forward_steps(P, A, n0, n1, dt, states, rtol_lin, traction, abs_tol):
    """Steps n0..n1-1 from states[n0-1], states[n0] (device tensors); fills states[n0+1..n1]."""
    torch = _torch()
    h1 = states[n0].clone()
    h0 = states[n0 - 1].clone()
    results = []
    for n in range(n0, n1):
        A.set_neumann_values(traction(A, (n + 1) * dt))
        A.set_history_device(1, h1.data_ptr())
        A.set_history_device(2, h0.data_ptr())
        P.X.copy_(h1)
        r = newton_device(P, rtol_lin=rtol_lin, abs_tol=abs_tol)
        results.append(r)
        h0, h1 = h1, P.X.clone()
        states[n + 1] = h1
    return results


def adjoint(A, nsteps, dt, g, dJdU_final, every=10, rtol_lin=1e-12, traction=traction_values, abs_tol=1e-13,
            U_init=None, U_prev=None, objective=None):
    """Forward solve of nsteps steps with element log-scales g and checkpoints every
    `every` steps, then the backward sweep.  dJdU_final(U_N) -> dJ/dU_N (host or device
    array); objective(U_N) -> J (optional).  Returns dict(J, grad (dJ/dg, host), U_N,
    checkpoints, forward_results, recomputed_steps)."""
    torch = _torch()
    P = DeviceProblem(A, "fp64", use_graph=False)
    n, ne = A.ndof, A.nelem_total
    with torch.cuda.stream(P.stream):
        A.set_element_log_scale(np.asarray(g, dtype=np.float64))
        zero = torch.zeros(n, dtype=torch.float64, device=P.dev)
        u0 = zero.clone() if U_init is None else torch.as_tensor(np.asarray(U_init, np.float64), device=P.dev)
        um = zero.clone() if U_prev is None else torch.as_tensor(np.asarray(U_prev, np.float64), device=P.dev)
        ckpt = {0: (um.clone(), u0.clone())}
        states = {-1: um, 0: u0}
        fwd = []
        for s in range(0, nsteps, every):
            e = min(s + every, nsteps)
            seg = {s - 1: states[s - 1], s: states[s]}
            fwd += _forward_steps(P, A, s, e, dt, seg, rtol_lin, traction, abs_tol)
            states = {e - 1: seg[e - 1], e: seg[e]}
            if e < nsteps:
                ckpt[e] = (seg[e - 1].clone(), seg[e].clone())
        UN = states[nsteps]
        J = objective(UN.cpu().numpy()) if objective else None
        # ---- backward sweep
        drows = torch.as_tensor(A.dirichlet_rows(), device=P.dev, dtype=torch.long)
        b = {nsteps - 1: torch.as_tensor(np.asarray(dJdU_final(UN.cpu().numpy()), np.float64),
                                         device=P.dev).clone()}
        grad = torch.zeros(ne, dtype=torch.float64, device=P.dev)
        gstep = torch.empty(ne, dtype=torch.float64, device=P.dev)
        Vj = torch.empty(A.nnz, dtype=torch.float64, device=P.dev)
        c = torch.empty(n, dtype=torch.float64, device=P.dev)
        recomputed = 0
        for s in sorted(ckpt.keys(), reverse=True):
            e = min(s + every, nsteps)
            seg = {s - 1: ckpt[s][0], s: ckpt[s][1]}
            _forward_steps(P, A, s, e, dt, seg, rtol_lin, traction, abs_tol)
            recomputed += e - s
            for k in range(e - 1, s - 1, -1):
                bk = b.pop(k, None)
                if bk is None:
                    continue                      # no objective dependence reaches this step
                bk[drows] = 0.0
                A.set_history_device(1, seg[k].data_ptr())
                A.set_history_device(2, seg[k - 1].data_ptr())
                U = seg[k + 1]
                A.tangent_device(U.data_ptr(), P.V.data_ptr(), "fp64")          # K_k
                lam = _sym_solve(P, bk, rtol_lin)
                lam[drows] = 0.0
                A.adjoint_backward_device(U.data_ptr(), None, lam.data_ptr(), None, gstep.data_ptr(), "fp64")
                grad += gstep
                for level, tgt in ((1, k - 1), (2, k - 2)):
                    if tgt < 0:
                        continue
                    A.history_jacobian_device(U.data_ptr(), Vj.data_ptr(), level, "fp64")
                    A.adjoint_backward_device(None, Vj.data_ptr(), lam.data_ptr(), c.data_ptr(), None, "fp64")
                    if tgt in b:
                        b[tgt] -= c
                    else:
                        b[tgt] = -c
        A.set_element_log_scale(None)
        P.stream.synchronize()
        return dict(J=J, grad=(-grad).cpu().numpy(), U_N=UN.cpu().numpy(), checkpoints=sorted(ckpt.keys()),
                    forward_results=fwd, recomputed_steps=recomputed)
