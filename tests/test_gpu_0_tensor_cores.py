"""tcgen05 tensor-core path (FP32 tangent of the mixed-precision Newton solve).

This file is collected before the other GPU tests: the operand-layout check
runs first, then the FP32 tensor-core tangent is compared with the reference's
FP64 assembly (rowwise 1e-5, the FP32 tolerance of the parity suite) and with
the FP32 FMA-pipe kernel, and checked for exact symmetry."""
import ctypes

import numpy as np
import pytest

from cases import make_case, neumann_values

pytestmark = pytest.mark.gpu

CASES = ["tiny_default", "ragged_config0", "perturbed_lame", "mixed_bc", "config0_8"]
OPT_FP32_KERNEL = 2


def test_tc_operand_layout_selftest(built):
    """A B^T of fixed small-integer operands through the kernel's descriptors and
    instruction shapes (M 128 / N 96 and M 128 / N 32); exact in FP32."""
    from igap4standard_b200 import native
    lib = native.lib_cuda()
    out = np.zeros((128, 160), dtype=np.float32)
    native.check(lib, "igab_tc_selftest", lib.igab_tc_selftest(0, out.ctypes.data_as(ctypes.c_void_p)))
    m = np.arange(128)[:, None]
    k = np.arange(32)[None, :]
    A = (((m * 5 + k * 3) % 13) - 6) * 0.5
    n = np.arange(96)[:, None]
    B = (((n * 7 + k) % 11) - 5) * 0.25
    D = A @ B.T
    assert np.array_equal(out[:, :96], D.astype(np.float32))
    assert np.array_equal(out[:, 96:128], D[:, :32].astype(np.float32))
    Dn = A[:, :16] @ B[:32, :16].T - A[:, 16:] @ B[:32, 16:].T      # negate-A on the last two k-steps
    assert np.array_equal(out[:, 128:], Dn.astype(np.float32))


def _assembly(c):
    from igap4standard_b200 import Assembly
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"])
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, c["par_neumann"]))
    return A


def _rowwise(rp, v, v_ref):
    rowmax = np.maximum.reduceat(np.abs(v_ref), rp[:-1])
    err = np.maximum.reduceat(np.abs(v - v_ref), rp[:-1])
    return float(np.max(err / np.maximum(rowmax, 1e-300)))


@pytest.mark.parametrize("name", CASES)
def test_fp32_tensor_core_tangent(built, checker, name):
    c = make_case(name)
    ref = checker("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                  c["par_dirichlet"], c["par_neumann"])
    rp_ref, cols_ref, v_ref = ref.tangent(c["U"])
    A = _assembly(c)
    A.set_option(OPT_FP32_KERNEL, 1)
    v_tc = A.tangent(c["U"], "fp32").astype(np.float64)
    A.set_option(OPT_FP32_KERNEL, 0)
    v_fma = A.tangent(c["U"], "fp32").astype(np.float64)
    e_tc, e_fma = _rowwise(rp_ref, v_tc, v_ref), _rowwise(rp_ref, v_fma, v_ref)
    print("%s: rowwise rel err tensor cores %.2e, FMA pipe %.2e" % (name, e_tc, e_fma))
    assert e_tc <= 1e-5
    assert e_fma <= 1e-5


def test_fp32_tensor_core_tangent_symmetric(built):
    import scipy.sparse as sp
    c = make_case("perturbed_lame")
    A = _assembly(c)
    A.set_option(OPT_FP32_KERNEL, 1)
    rp, cols = A.pattern()
    v = A.tangent(c["U"], "fp32")
    K = sp.csr_matrix((v, cols, rp), shape=(A.ndof, A.ndof))
    assert (K - K.T).count_nonzero() == 0 or np.max(np.abs((K - K.T).data)) == 0.0


def test_fp32_tensor_core_tangent_deterministic(built):
    c = make_case("config0_8")
    A = _assembly(c)
    A.set_option(OPT_FP32_KERNEL, 1)
    v1 = A.tangent(c["U"], "fp32")
    v2 = A.tangent(c["U"], "fp32")
    assert np.array_equal(v1, v2)


def test_fp64_tensor_pipe_probe(built):
    """igab_dmma_peak: back-to-back mma.sync m8n8k4 f64 gives a plausible B200 rate (TFLOP/s)."""
    from igap4standard_b200.assembly import dmma_peak_tflops
    t = dmma_peak_tflops(0)
    print("FP64 tensor pipe: %.2f TFLOP/s" % t)
    assert 5.0 < t < 200.0
