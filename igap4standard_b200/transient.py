"""Time stepping of the transient physics (phys/getime) and its checkpointed discrete
adjoint, as thin host wrappers over the library's device drivers.

Per time step the reference example (example/ex1/main.c:48-56) takes the previous
solution as initial guess (initguess, :116-126), runs snes_solve (src/snes_solve.c:23-33:
one Newton step per SNESSolve, absolute ||F||_2 <= 1e-10, stagnation stop) and shifts the
history levels, U_hist[k] <- U_hist[k-1] for k = torder..1 (:55).  igab_transient_run
(igab_transient.cu) does this on the GPU, each solve being igab_newton_solve: residual and
tangent assemblies replayed from CUDA graphs, cubic backtracking line search, the Jacobi
BiCGStab of igab_solve_device as the stand-in for PETSc's GMRES + ASM
(src/snes_init.c:24-39).  The adjoint (igab_tadj_*) keeps state checkpoints every
`every` steps and recomputes each segment before sweeping it backward.

The traction of the transient workload is amplitude * sin(2 pi t) on face x = 1 in the x
direction (face 1, standard order, dof 0), evaluated at t_{n+1}.
"""
from dataclasses import dataclass, field

import numpy as np

ABS_TOL = 1e-10   # SNESSetTolerances abstol, src/snes_init.c:18


@dataclass
class StepResult:
    """The Newton solve of one time step (igab_newton_info of the step)."""
    U: object
    converged: bool
    reason: int
    iterations: int
    fnorms: list = field(default_factory=list)   # ||F|| at the end of the step's solve
    n_residual: int = 0
    n_tangent: int = 0


def _device_vector(A, x):
    import torch
    dev = torch.device("cuda", A.device)
    if x is None:
        return torch.zeros(A.ndof, dtype=torch.float64, device=dev)
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64)).to(dev)


def run(A, nsteps, dt, prec="fp32", use_graph=True, rtol_lin=1e-5, amplitude=0.01, U_init=None, U_prev=None,
        abs_tol=ABS_TOL, keep_steps=True):
    """Time-step A (an Assembly with phys="getime") nsteps times from the history (U_init
    at t_0, U_prev at t_{-1}; zeros by default) with the time step dt.  Returns (the state
    after every step as host arrays (empty when keep_steps is False), per-step
    StepResults, the run's totals)."""
    import torch
    U = _device_vector(A, U_init)
    Up = _device_vector(A, U_prev) if U_prev is not None else None
    torch.cuda.synchronize(U.device)
    tot, steps, hist = A.transient_run(U.data_ptr(), nsteps, prec, Up.data_ptr() if Up is not None else None,
                                       dt=dt, amplitude=amplitude, ksp_rtol=rtol_lin, abstol=abs_tol,
                                       use_graph=use_graph, keep_steps=keep_steps)
    states = list(hist) if keep_steps else []
    results = [StepResult(U=states[i] if keep_steps else None, converged=bool(s["converged"]), reason=int(s["reason"]),
                          iterations=int(s["iterations"]), fnorms=[s["fnorm"]], n_residual=int(s["n_residual"]),
                          n_tangent=int(s["n_tangent"]))
               for i, s in enumerate(steps)]
    tot["krylov_per_step"] = [int(s["krylov_iterations"]) for s in steps]
    tot["U_final"] = U.cpu().numpy()
    return states, results, tot


def adjoint(A, nsteps, dt, g, dJdU_final, every=10, rtol_lin=1e-12, amplitude=0.01, abs_tol=1e-13, U_init=None,
            U_prev=None, objective=None, use_graph=True):
    """dJ/dg of J(U_N) for the element log-scales g (s_e = exp(g_e)) after nsteps steps:
    the forward solve with checkpoints every `every` steps, then the backward sweep with
    segment recomputation, both on the device.  dJdU_final(U_N) -> dJ/dU_N (host array);
    objective(U_N) -> J (optional).  Returns dict(J, grad (host), U_N, checkpoints,
    recomputed_steps, info)."""
    import torch
    A.set_element_log_scale(np.asarray(g, dtype=np.float64))
    dev = torch.device("cuda", A.device)
    U0 = _device_vector(A, U_init)
    Um = _device_vector(A, U_prev) if U_prev is not None else None
    UN = torch.empty(A.ndof, dtype=torch.float64, device=dev)
    grad = torch.empty(A.nelem_total, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    T = A.transient_adjoint(nsteps, every, U0.data_ptr(), Um.data_ptr() if Um is not None else None, dt=dt,
                            amplitude=amplitude, ksp_rtol=rtol_lin, abstol=abs_tol, use_graph=use_graph)
    try:
        T.forward(UN.data_ptr())
        UN_h = UN.cpu().numpy()
        J = objective(UN_h) if objective else None
        dJ = _device_vector(A, dJdU_final(UN_h))
        torch.cuda.synchronize(dev)
        T.backward(dJ.data_ptr(), grad.data_ptr())
        info = T.info()
    finally:
        T.close()
        A.set_element_log_scale(None)
    return dict(J=J, grad=grad.cpu().numpy(), U_N=UN_h, checkpoints=list(range(0, nsteps, every)),
                recomputed_steps=info["recomputed_steps"], info=info)
