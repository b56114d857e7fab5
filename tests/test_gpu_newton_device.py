"""Device Newton solve (igab_newton_solve): the reference application's solver loop
(src/snes_solve.c:10-36 with the SNES settings of src/snes_init.c:8-47) run on the
GPU, the linear solves by the device BiCGStab, no residual or tangent on the host.

Parity: against the same loop over the reference's own CPU assembly with a direct
linear solve (igap4standard_b200/newton.py), from U = 0.  With the Krylov tolerance
tightened to 1e-10 the two are the same Newton iteration up to the linear-solve
error: same termination reason, same step count, ||U_dev - U_ref||_inf <=
1e-10 * max(||U_ref||_inf, 1).  At PETSc's default KSP tolerance (1e-5) the
device solve still converges to ||F|| < 1e-10, and the FP32-tangent solve needs at
most one more step than the FP64 one."""
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


def _device_solve(A, prec, ksp_rtol):
    import torch
    U = torch.zeros(A.ndof, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    info = A.newton_solve_device(U.data_ptr(), prec, ksp_rtol=ksp_rtol)
    return info, U.cpu().numpy()


@pytest.mark.parametrize("name", ["perturbed_lame", "ragged_config0", "newton_backtrack", "config0_8"])
def test_device_newton_matches_reference_loop(built, checker, name):
    from oracle import newton_loop as newton
    c = make_case(name)
    case = checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                   c["par_dirichlet"], c["par_neumann"])
    r_ref, j_ref = newton.case_problem(case)
    ref = newton.solve(r_ref, j_ref, np.zeros(case.ndof))
    A = _assembly(c)
    info, U = _device_solve(A, "fp64", 1e-10)
    print(name, "ref", ref.reason, ref.iterations, ref.fnorms)
    print(name, "dev", info["reason"], info["iterations"], info["fnorms"], info["krylov"])
    assert info["reason"] == ref.reason
    assert info["iterations"] == ref.iterations
    assert info["n_residual"] == ref.n_residual and info["n_tangent"] == ref.n_tangent
    scale = max(np.abs(ref.U).max(), 1.0)
    assert np.abs(U - ref.U).max() <= 1e-10 * scale
    A.close()


@pytest.mark.parametrize("name", ["perturbed_lame", "config0_8", "newton_backtrack"])
def test_device_newton_default_ksp_and_mixed(built, name):
    c = make_case(name)
    A = _assembly(c)
    a, Ua = _device_solve(A, "fp64", 1e-5)
    b, Ub = _device_solve(A, "fp32", 1e-5)
    print(name, "fp64", a["iterations"], a["fnorms"], a["krylov"])
    print(name, "fp32", b["iterations"], b["fnorms"], b["krylov"])
    assert a["converged"] and b["converged"]
    assert a["fnorm"] < 1e-10 and b["fnorm"] < 1e-10
    assert b["iterations"] <= a["iterations"] + 1
    assert np.abs(Ub - Ua).max() <= 1e-8 * max(np.abs(Ua).max(), 1.0)
    A.close()


def test_device_newton_repeatable(built):
    c = make_case("perturbed_lame")
    A = _assembly(c)
    a, Ua = _device_solve(A, "fp64", 1e-5)
    b, Ub = _device_solve(A, "fp64", 1e-5)
    assert a["fnorms"] == b["fnorms"] and a["krylov"] == b["krylov"]
    assert np.array_equal(Ua, Ub)
    A.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_device_newton_graph_replay_equals_eager(built, prec):
    """Assemblies replayed from the context's graphs give the eager solve bit for bit; a
    second solve on the same buffers replays the cached graphs; a material change
    re-captures them (the graph solve after it equals the eager one)."""
    import torch
    c = make_case("perturbed_lame")
    A = _assembly(c)
    U = torch.zeros(A.ndof, dtype=torch.float64, device="cuda")

    def solve(use_graph):
        U.zero_()
        torch.cuda.synchronize()
        info = A.newton_solve_device(U.data_ptr(), prec, ksp_rtol=1e-5, use_graph=use_graph)
        return info, U.cpu().numpy()

    a, Ua = solve(False)
    b, Ub = solve(True)
    r, Ur = solve(True)
    assert a["converged"] and a["fnorms"] == b["fnorms"] == r["fnorms"] and a["krylov"] == b["krylov"]
    assert np.array_equal(Ua, Ub) and np.array_equal(Ua, Ur)
    pm = np.array(c["par_mat"], dtype=np.float64)
    pm[0] *= 1.25
    A.set_par_mat(pm)
    d, Ud = solve(True)
    e, Ue = solve(False)
    assert d["converged"] and np.array_equal(Ud, Ue) and not np.array_equal(Ud, Ua)
    A.close()


@pytest.mark.parametrize("name", ["config0_8", "perturbed_lame"])
def test_dropin_snes_solve_keeps_tangent_on_device(built, name):
    """snes_solve of the drop-in library (the reference's solver loop, src/snes_solve.c:10)
    against the same loop over the drop-in callbacks with the tangent copied into the
    host AIJ matrix and solved directly: same steps and solution.  The tangent callback
    never runs during the device solve (its timing stays 0) and the host matrix is never
    filled."""
    import ctypes
    from igap4standard_b200 import case as casemod, native
    from oracle import newton_loop as newton
    c = make_case(name)
    args = ("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"], c["par_dirichlet"],
            c["par_neumann"])
    H = casemod.gpu_case(*args)
    host = newton.solve(*newton.case_problem(H), np.zeros(H.ndof))
    H.close()
    D = casemod.gpu_case(*args)
    lib = native.lib_dropin()
    assert lib.snesiga_gpu_set_ksp(D.app, 1e-10, 0) == 0
    ok, U = D.solve(np.zeros(D.ndof))
    info = native.IgabNewtonInfo()
    assert lib.snesiga_gpu_last_solve(D.app, ctypes.byref(info)) == 0
    ms = np.zeros(4)
    assert lib.snesiga_gpu_last_timings(D.app, ms.ctypes.data_as(native.c_double_p)) == 0
    print(name, "host AIJ", host.iterations, host.fnorms, "device", info.iterations, info.fnorm,
          info.krylov_iterations)
    assert ok and info.converged
    assert info.iterations == host.iterations
    assert info.n_tangent == host.n_tangent and info.n_tangent > 0
    assert ms[1] == 0.0                              # no tangent callback: nothing went to the host matrix
    assert np.abs(U - host.U).max() <= 1e-10 * max(np.abs(host.U).max(), 1.0)
    Uh = np.empty(D.ndof)
    D.lib.iga_case_get_history(D.h, 0, Uh.ctypes.data_as(ctypes.c_void_p))
    assert np.array_equal(Uh, U)                     # the U_hist side effect of the callbacks
    assert np.abs(D.residual(U)).max() < 1e-10
    D.close()
