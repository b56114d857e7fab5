"""The host-pointer tangent (igab_tangent) is assembled slab by slab along x, each
slab's finished rows downloaded while the next slabs are assembled.  Every CSR
entry receives its element contributions in the same order as the single
whole-mesh pass of the device-pointer entry, so the two agree bit for bit; and the
slabbed result agrees with the reference's own tangent (src/snesiga_Tangent.c)
within the parity tolerance.  Dirichlet conditions on every face put the
MatZeroRowsColumns rows (src/snesiga_Tangent.c:270) and their transposed columns
on both sides of the slab boundaries."""
import numpy as np
import pytest

from cases import neumann_values, tangent_tolerance

pytestmark = pytest.mark.gpu


def _case(nelem, seed):
    from igap4standard_b200 import mesh
    rng = np.random.default_rng(seed)
    kn = mesh.knots_for(nelem, perturb=0.2, seed=seed)
    pm = mesh.par_mat_from_lame(0.7, 1.3, 0.15)
    bc = rng.integers(0, 2, 36).astype(np.int32)
    pd = rng.uniform(-0.05, 0.05, 9)
    pp = np.zeros(9)
    pn = rng.uniform(-0.1, 0.1, 39)
    ndof = 3 * (nelem[0] + 2) * (nelem[1] + 2) * (nelem[2] + 2)
    U = rng.uniform(-5e-2, 5e-2, ndof)
    return nelem, kn, pm, bc, pd, pp, pn, U


def _assembly(nelem, kn, pm, bc, pd, pp, pn):
    from igap4standard_b200 import Assembly
    A = Assembly(nelem, kn, pm, bc, pd, pp)
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, pn))
    return A


@pytest.mark.parametrize("nelem", [(29, 5, 4), (64, 3, 3), (24, 4, 5)])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_slabbed_host_tangent_equals_device(built, nelem, prec):
    import torch
    nelem, kn, pm, bc, pd, pp, pn, U = _case(nelem, 11)
    A = _assembly(nelem, kn, pm, bc, pd, pp, pn)
    assert A.dirichlet_rows().size > 0
    v_host = A.tangent(U, prec)
    dt = torch.float64 if prec == "fp64" else torch.float32
    Ud = torch.from_numpy(U).cuda()
    Vd = torch.full((A.nnz,), float("nan"), dtype=dt, device="cuda")
    torch.cuda.synchronize()
    A.tangent_device(Ud.data_ptr(), Vd.data_ptr(), prec)
    A.sync()
    torch.cuda.synchronize()
    v_dev = Vd.cpu().numpy()
    assert np.array_equal(v_host, v_dev)
    # a second host call into a dirty buffer rewrites every entry
    v2 = np.full_like(v_host, np.nan)
    A.tangent(U, prec, out=v2)
    assert np.array_equal(v2, v_host)


def test_slabbed_host_tangent_matches_reference(built, checker):
    nelem, kn, pm, bc, pd, pp, pn, U = _case((25, 3, 2), 5)
    ref = checker("ge", nelem, kn, pm, bc, pp, pd, pn)
    rp_ref, cols_ref, v_ref = ref.tangent(U)
    A = _assembly(nelem, kn, pm, bc, pd, pp, pn)
    rp, cols = A.pattern()
    assert np.array_equal(rp, rp_ref) and np.array_equal(cols, cols_ref)
    v = A.tangent(U, "fp64")
    tol = tangent_tolerance(rp_ref, v_ref)
    assert np.max(np.abs(v - v_ref) / np.maximum(tol, 1e-300)) <= 1.0
