"""Transient driver (igab_transient_run: phys/getime on the device, CUDA-graph replay of
every assembly) against the reference's own transient callbacks driven by the same solver
semantics on the CPU (direct solve): per-step displacements, Newton iteration counts and
the mixed-precision variant."""
import numpy as np
import pytest

from cases import make_transient_case

pytestmark = pytest.mark.gpu

NSTEPS = 4


def _pn(t):
    pn = np.zeros(39)
    pn[6 + 0] = 0.01 * np.sin(2.0 * np.pi * t)   # face 1 (x = 1), standard order, x-dof
    return pn


def _reference_run(oracle_lib, c, dt, nsteps):
    from oracle import newton_loop as newton
    args = ("getime", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"], c["par_dirichlet"],
            _pn(dt))
    ref = oracle_lib.case(*args)
    residual, jacobian = newton.case_problem(ref)
    h1 = np.zeros(ref.ndof)
    h0 = np.zeros(ref.ndof)
    hist, its = [], []
    for step in range(nsteps):
        ref.set_par_neumann(_pn((step + 1) * dt))
        ref.set_history(1, h1)
        ref.set_history(2, h0)
        r = newton.solve(residual, jacobian, h1)
        assert r.converged
        h0, h1 = h1, r.U.copy()
        hist.append(h1)
        its.append(r.iterations)
    return hist, its


def _assembly(c):
    from igap4standard_b200 import Assembly
    return Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"],
                    phys="getime")


@pytest.fixture(scope="module")
def transient_case(built, oracle_lib):
    from igap4standard_b200 import mesh
    c = make_transient_case("getime_config2")
    c["bc_type"], c["par_dirichlet"] = mesh.bc_transient()   # u = 0 on x = 0, traction on x = 1
    dt = c["par_mat"][7]
    ref_hist, ref_its = _reference_run(oracle_lib, c, dt, NSTEPS)
    return c, dt, ref_hist, ref_its


def test_transient_fp64_matches_reference(transient_case):
    from igap4standard_b200 import transient
    c, dt, ref_hist, ref_its = transient_case
    A = _assembly(c)
    hist, res, tot = transient.run(A, NSTEPS, dt, prec="fp64", use_graph=True, rtol_lin=1e-13)
    its = [r.iterations for r in res]
    print("reference iterations", ref_its, "gpu", its, "krylov", tot["krylov_per_step"])
    assert tot["steps"] == NSTEPS and tot["steps_converged"] == NSTEPS
    assert np.array_equal(tot["U_final"], hist[-1])
    assert all(r.converged for r in res)
    assert its == ref_its
    assert np.abs(ref_hist[-1]).max() > 0.0        # the traction moved the body
    for h, hr in zip(hist, ref_hist):              # relative to the step's displacement scale
        assert np.abs(h - hr).max() <= 1e-9 * np.abs(hr).max()


def test_transient_graph_equals_eager(transient_case):
    from igap4standard_b200 import transient
    c, dt, _, _ = transient_case
    h_graph, _, _ = transient.run(_assembly(c), 2, dt, prec="fp32", use_graph=True)
    h_eager, _, _ = transient.run(_assembly(c), 2, dt, prec="fp32", use_graph=False)
    for a, b in zip(h_graph, h_eager):
        assert np.array_equal(a, b)


def test_transient_mixed_precision(transient_case):
    from igap4standard_b200 import transient
    c, dt, ref_hist, ref_its = transient_case
    # FP32 tangent, linear solves to 1e-9: the difference to the FP64 reference is the FP32
    # Jacobian's (an inexact Newton step), not the Krylov tolerance's
    hist, res, _ = transient.run(_assembly(c), NSTEPS, dt, prec="fp32", use_graph=True, rtol_lin=1e-9)
    assert all(r.converged and r.fnorms[-1] < 1e-10 for r in res)
    for r, n in zip(res, ref_its):
        assert r.iterations <= n + 1
    for h, hr in zip(hist, ref_hist):
        assert np.abs(h - hr).max() <= 1e-5 * np.abs(hr).max()
