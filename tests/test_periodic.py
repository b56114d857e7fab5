"""Periodic directions on one rank, without a GPU: the reference's own assembly
(oracle/_ref) on periodic meshes passes its physical known answers (a rigid translation
leaves zero residual; the tangent is symmetric and is the derivative of the residual),
and the drop-in's snesiga_init builds the same rank index maps as the reference's
(src/snesiga_init.c:134-330: owned points, the ghost layers exchanged with itself and
their global indices)."""
import numpy as np
import pytest
import scipy.sparse as sp

from periodic_cases import PERIODIC, make_periodic_case


def _ref(oracle_lib, c):
    return oracle_lib.case(c["phys"], c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                           c["par_dirichlet"], c["par_neumann"], bc_periodic=c["bc_periodic"])


@pytest.mark.parametrize("per", PERIODIC)
def test_reference_periodic_known_answers(oracle_lib, per):
    c = make_periodic_case(per)
    c["bc_type"] = np.ones(36, dtype=np.int32)           # traction-free, no Dirichlet rows
    c["par_neumann"] = np.zeros(39)
    c["par_periodic"] = np.zeros(9)
    ref = _ref(oracle_lib, c)
    nb = [c["nelem"][d] if per[d] else c["nelem"][d] + 2 for d in range(3)]
    assert ref.ndof == 3 * nb[0] * nb[1] * nb[2]
    U = np.tile([1e-3, -2e-3, 3e-3], ref.ndof // 3)       # rigid translation
    assert np.abs(ref.residual(U)).max() < 1e-15
    rp, cols, vals = ref.tangent(c["U"])
    K = sp.csr_matrix((vals, cols, rp), shape=(ref.ndof, ref.ndof))
    assert abs(K - K.T).max() <= 1e-14 * abs(K).max()
    eps = 1e-7
    for j in np.random.default_rng(1).choice(ref.ndof, 3, replace=False):
        d = np.zeros(ref.ndof)
        d[j] = eps
        fd = (ref.residual(c["U"] + d) - ref.residual(c["U"] - d)) / (2 * eps)
        col = K[:, j].toarray().ravel()
        assert np.abs(fd - col).max() <= 1e-6 * np.abs(col).max()


@pytest.mark.parametrize("per", PERIODIC + [(0, 0, 0)])
def test_dropin_index_maps_equal_reference(oracle_lib, per):
    from igap4standard_b200 import case as casemod, native
    c = make_periodic_case(per, nelem=(4, 5, 3))
    ref = _ref(oracle_lib, c)
    ours = casemod.Case(native.lib_dropin(), c["phys"], c["nelem"], c["knots"], c["par_mat"], c["bc_type"],
                        c["par_periodic"], c["par_dirichlet"], c["par_neumann"], bc_periodic=per)
    for a, b, name in zip(ref.index_maps(), ours.index_maps(), ("selfIdx", "sendIdx", "recvIdx", "globalIdx")):
        assert np.array_equal(a, b), name
