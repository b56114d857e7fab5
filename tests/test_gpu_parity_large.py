"""GPU parity at the headline workload's sizes, against the reference's own CPU assembly.

  * the full 64^3 residual of the config-1 workload (interior knots perturbed +-0.1h,
    seed 1; lambda = mu = 1, l = 0.1 mapped to par_mat; BCs of config 0; state
    uniform in +-1e-3, seed 0): every entry within 1e-12 relative (cancellation floor
    of tests/cases.py);
  * the full 16^3 tangent of the same workload family (4,096 elements): FP64 entry by
    entry within 1e-12, the FP32 tensor-core tangent rowwise within 1e-5.

The reference side takes minutes on one core (about 40 s for the residual, 100-200 s
for the tangent), so both run at once in spawned processes while the GPU side runs."""
import multiprocessing as mp

import numpy as np
import pytest

from cases import residual_tolerance, tangent_tolerance

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _workload(n):
    from igap4standard_b200 import mesh
    nelem = (n, n, n)
    kn = mesh.knots_for(nelem, perturb=0.1, seed=1)
    pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
    bc, pd = mesh.bc_config0()
    U = np.random.default_rng(0).uniform(-1e-3, 1e-3, mesh.n_dof(nelem))
    return nelem, kn, pm, bc, pd, U


def _reference(job):
    """In a spawned process: the reference's residual or tangent on the n^3 workload."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from oracle import ref
    kind, n = job
    nelem, kn, pm, bc, pd, U = _workload(n)
    C = ref.case("ge", nelem, kn, pm, bc, np.zeros(9), pd, np.zeros(39))
    out = C.residual(U) if kind == "residual" else C.tangent(U)
    C.close()
    return out


@pytest.fixture(scope="module")
def references(built, oracle_lib):
    pool = mp.get_context("spawn").Pool(2)
    jobs = {"residual": pool.apply_async(_reference, (("residual", 64),)),
            "tangent": pool.apply_async(_reference, (("tangent", 16),))}
    yield jobs
    pool.close()
    pool.join()


def test_residual_parity_64cubed(references):
    from igap4standard_b200 import Assembly
    nelem, kn, pm, bc, pd, U = _workload(64)
    A = Assembly(nelem, kn, pm, bc, pd)
    R = A.residual(U)
    A.close()
    R_ref = references["residual"].get(timeout=1800)
    err = np.abs(R - R_ref)
    tol = residual_tolerance(R_ref)
    print("64^3 residual: max |diff| %.3e, worst diff/tol %.3f, ||R_ref||_inf %.3e"
          % (err.max(), np.max(err / tol), np.abs(R_ref).max()))
    assert np.all(err <= tol)


def test_tangent_parity_16cubed(references):
    from igap4standard_b200 import Assembly
    nelem, kn, pm, bc, pd, U = _workload(16)
    A = Assembly(nelem, kn, pm, bc, pd)
    rp, cols = A.pattern()
    v64 = A.tangent(U, "fp64")
    v32 = A.tangent(U, "fp32").astype(np.float64)
    A.close()
    rp_ref, cols_ref, v_ref = references["tangent"].get(timeout=1800)
    assert np.array_equal(rp, rp_ref) and np.array_equal(cols, cols_ref)
    tol = tangent_tolerance(rp_ref, v_ref)
    err = np.abs(v64 - v_ref)
    print("16^3 FP64 tangent: max |diff| %.3e, worst diff/tol %.3f" % (err.max(), np.max(err / tol)))
    assert np.all(err <= tol)
    rowmax = np.maximum.reduceat(np.abs(v_ref), rp_ref[:-1])
    e32 = np.max(np.maximum.reduceat(np.abs(v32 - v_ref), rp_ref[:-1]) / rowmax)
    print("16^3 FP32 tangent: rowwise relative error %.2e" % e32)
    assert e32 <= 1e-5
