"""Knot-insertion prolongation of the multigrid solver (igab_mg_prolongation_1d), no GPU:
every coarse B-spline (p = 2, open, perturbed knots) equals the combination of the fine
B-splines that the matrix gives, at random points; rows sum to one (partition of unity)."""
import ctypes

import numpy as np

from igap4standard_b200 import mesh


def _bspline_basis(kv, x):
    """All p = 2 B-splines of knot vector kv at x (Cox-de Boor, right-continuous, last
    point included in the last span)."""
    kv = np.asarray(kv)
    nb = len(kv) - 3
    N = np.zeros(len(kv) - 1)
    span = np.searchsorted(kv, x, side="right") - 1
    span = min(span, len(kv) - 4)
    N[span] = 1.0
    for p in (1, 2):
        M = np.zeros(len(kv) - 1 - p)
        for i in range(len(M)):
            a = (x - kv[i]) / (kv[i + p] - kv[i]) * N[i] if kv[i + p] > kv[i] else 0.0
            b = (kv[i + p + 1] - x) / (kv[i + p + 1] - kv[i + 1]) * N[i + 1] if kv[i + p + 1] > kv[i + 1] else 0.0
            M[i] = a + b
        N = M
    return N[:nb]


def test_prolongation_reproduces_coarse_splines(built):
    from igap4standard_b200 import native
    lib = native.lib_cuda()
    rng = np.random.default_rng(2)
    for n in (2, 4, 6, 16):
        fine = mesh.open_knot_vector(n, perturb=0.2, rng=rng)
        inner = fine[3:-3]
        coarse = np.concatenate([fine[:3], inner[1::2], fine[-3:]])
        ins = np.ascontiguousarray(inner[0::2])
        nc = n // 2
        P = np.zeros((n + 2, nc + 2))
        rc = lib.igab_mg_prolongation_1d(np.ascontiguousarray(coarse).ctypes.data_as(ctypes.c_void_p), nc,
                                         ins.ctypes.data_as(ctypes.c_void_p), len(ins),
                                         P.ctypes.data_as(ctypes.c_void_p))
        assert rc == 0
        assert np.allclose(P.sum(axis=1), 1.0, atol=1e-14)
        assert np.count_nonzero(np.abs(P) > 0, axis=1).max() <= 3
        for x in np.concatenate([rng.uniform(0, 1, 50), [0.0, 1.0]]):
            Nc = _bspline_basis(coarse, x)
            Nf = _bspline_basis(fine, x)
            assert np.allclose(Nc, Nf @ P, atol=1e-13), (n, x)


def test_prolongation_rejects_bad_knots(built):
    from igap4standard_b200 import native
    lib = native.lib_cuda()
    coarse = np.ascontiguousarray(mesh.open_knot_vector(2))
    ins = np.array([0.7, 0.2])                 # not ascending
    P = np.zeros((4 + 2) * 4)
    assert lib.igab_mg_prolongation_1d(coarse.ctypes.data_as(ctypes.c_void_p), 2, ins.ctypes.data_as(ctypes.c_void_p),
                                       2, P.ctypes.data_as(ctypes.c_void_p)) == 1

