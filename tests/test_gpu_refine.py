"""Knot-insertion refinement (mesh/nurbs/nurbs_knotinsert.c) on the GPU against the
reference's own nurbs_knotinsert on the same arrays: one and two refinement
levels, open and periodic directions, through the library entry
(igab_knot_insert) and the drop-in (nurbs_knotinsert of libsnesiga_b200).  The
refined control points agree to the last bit or within 1e-15 relative (the
sums of at most eight dyadic-weighted terms are taken in the reference's
order; contraction into fused multiply-adds may differ by compiler)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [((4, 6, 8), 1, (0, 0, 0)), ((8, 4, 4), 2, (0, 0, 0)), ((4, 6, 8), 1, (1, 0, 1)),
         ((8, 8, 4), 2, (1, 1, 1)), ((2, 2, 2), 1, (0, 1, 0))]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _arrays(nelem, nref, per, ndof, seed):
    nel = np.array(nelem, dtype=np.int32)
    coarse = nel // (1 << nref)
    nbc = [int(coarse[d] + (2 if per[d] == 0 else 0)) for d in range(3)]
    nbf = [int(nel[d] + (2 if per[d] == 0 else 0)) for d in range(3)]
    U = np.zeros(int(np.prod([n + 2 for n in nel])) * ndof)
    nc = int(np.prod(nbc)) * ndof
    U[:nc] = np.random.default_rng(seed).normal(size=nc)
    return nel, np.array(per, dtype=np.int32), U, int(np.prod(nbf)) * ndof


@pytest.mark.parametrize("nelem,nref,per", CASES)
def test_knot_insert_matches_reference(built, oracle_lib, nelem, nref, per):
    from igap4standard_b200 import native
    ndof = 3
    nel, pb, U, nfine = _arrays(nelem, nref, per, ndof, 7)
    U_ref, U_gpu, U_drop = U.copy(), U.copy(), U.copy()
    oracle_lib.lib().nurbs_knotinsert(_p(U_ref), _p(nel), nref, 2, 3, ndof, _p(pb))
    lib = native.lib_cuda()
    assert lib.igab_knot_insert(_p(U_gpu), _p(nel), nref, 2, ndof, _p(pb), 0) == 0
    native.lib_dropin().nurbs_knotinsert(_p(U_drop), _p(nel), nref, 2, 3, ndof, _p(pb))
    a, b, d = U_ref[:nfine], U_gpu[:nfine], U_drop[:nfine]
    err = np.abs(a - b).max() / np.abs(a).max()
    print("%s nref %d periodic %s: %s, max rel diff %.2e" % (nelem, nref, per,
                                                          "bitwise equal" if np.array_equal(a, b) else "differs", err))
    assert err <= 1e-15
    assert np.array_equal(b, d)


def test_knot_insert_rejects_bad_sizes(built):
    from igap4standard_b200 import native
    lib = native.lib_cuda()
    nel = np.array([6, 4, 4], dtype=np.int32)
    pb = np.zeros(3, dtype=np.int32)
    U = np.zeros(8 * 6 * 6 * 3)
    assert lib.igab_knot_insert(_p(U), _p(nel), 2, 2, 3, _p(pb), 0) != 0     # 6 is not a multiple of 4
    assert lib.igab_knot_insert(_p(U), _p(nel), 1, 3, 3, _p(pb), 0) != 0     # porder 3
    assert lib.igab_knot_insert(_p(U), _p(nel), 1, 2, 3, _p(pb), -1) != 0    # no device -1
    assert lib.igab_knot_release(-1) != 0


def test_knot_insert_buffers_kept_and_released(built, oracle_lib):
    """The device buffers kept between calls: a large field, then smaller ones in
    the larger buffers (nothing of the previous call leaks into the result), then
    after igab_knot_release, allocated again."""
    from igap4standard_b200 import native
    lib = native.lib_cuda()
    for k, (nelem, nref, per) in enumerate([((16, 16, 8), 1, (0, 0, 0)), ((4, 6, 8), 1, (1, 0, 1)),
                                            ((8, 4, 4), 2, (0, 0, 0)), (None, 0, 0), ((4, 6, 8), 1, (1, 0, 1))]):
        if nelem is None:
            assert lib.igab_knot_release(0) == 0
            assert lib.igab_knot_release(0) == 0        # nothing held: no-op
            continue
        nel, pb, U, nfine = _arrays(nelem, nref, per, 3, 11 + k)
        U_ref, U_gpu = U.copy(), U.copy()
        oracle_lib.lib().nurbs_knotinsert(_p(U_ref), _p(nel), nref, 2, 3, 3, _p(pb))
        assert lib.igab_knot_insert(_p(U_gpu), _p(nel), nref, 2, 3, _p(pb), 0) == 0
        a, b = U_ref[:nfine], U_gpu[:nfine]
        assert np.abs(a - b).max() <= 1e-15 * np.abs(a).max()
