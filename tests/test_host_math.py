"""The product's point mathematics (igab_math.cuh, compiled for the host)
against the reference's integrands and basis -- no GPU needed."""
import ctypes

import numpy as np


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_ge_point_matches_reference(golden, host_math):
    for p, par in enumerate(golden["ge_par"]):
        par = np.ascontiguousarray(par)
        for t, u in enumerate(golden["ge_u"]):
            u = np.ascontiguousarray(u)
            r = np.empty(30)
            D27 = np.empty((27, 27))
            host_math.host_ge_point(_p(u), _p(par), _p(r), _p(D27))
            rr = golden["ge_r"][p, t]
            assert np.all(np.abs(r - rr) <= 1e-12 * np.max(np.abs(rr)))
            Dref = golden["ge_D"][p, t]
            idx = [i for i in range(30) if i % 10]
            assert np.all(np.abs(D27 - Dref[np.ix_(idx, idx)]) <= 1e-12 * np.max(np.abs(Dref)))
            # value components carry no energy
            assert np.all(Dref[0::10, :] == 0) and np.all(Dref[:, 0::10] == 0)


def test_bspline_matches_reference(golden, host_math):
    W, X, N = golden["bsp_windows"], golden["bsp_x"], golden["bsp_N"]
    for t in range(W.shape[0]):
        out = [np.empty(9) for _ in range(3)]
        for d in range(3):
            host_math.host_bspline_p2(_p(np.ascontiguousarray(W[t, d])), float(X[t, d]), _p(out[d]))
        tab = [o.reshape(3, 3) for o in out]
        # value and first/second x-derivative of the first basis function products
        assert abs(tab[0][0, 0] * tab[1][0, 0] * tab[2][0, 0] - N[t, 0, 0]) <= 1e-14
        assert abs(tab[0][2, 1] * tab[1][1, 0] * tab[2][2, 0] - N[t, 9 * 2 + 3 + 2, 1]) <= 1e-12 * max(1, abs(N[t, 23, 1]))
        assert abs(tab[0][1, 2] * tab[1][1, 0] * tab[2][0, 0] - N[t, 9 + 3, 4]) <= 1e-12 * max(1, abs(N[t, 12, 4]))


def test_getime_point_matches_reference(golden, host_math):
    """Transient integrand: Taylor-truncated average gradient + inertia/damping."""
    par = np.ascontiguousarray(golden["getime_par"])
    idx = [i for i in range(30) if i % 10]
    for t, u in enumerate(golden["getime_u"]):
        u = np.ascontiguousarray(u)
        r = np.empty(30)
        D27 = np.empty((27, 27))
        host_math.host_getime_point(_p(u), _p(par), _p(r), _p(D27))
        rr = golden["getime_r"][t]
        assert np.all(np.abs(r - rr) <= 1e-12 * np.max(np.abs(rr)))
        Dref = golden["getime_D"][t]
        sub = Dref[np.ix_(idx, idx)]
        assert np.all(np.abs(D27 - sub) <= 1e-12 * np.max(np.abs(sub)))
        mass = par[6] / (2 * par[7]) + par[5] / par[7] ** 2
        assert np.allclose(np.diag(Dref)[0::10], mass, rtol=1e-14)
