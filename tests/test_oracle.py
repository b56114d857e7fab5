"""CPU checks of the oracles against the reference's golden vectors (no GPU)."""
import numpy as np
import pytest

from cases import make_case, residual_tolerance, tangent_tolerance

TOL = 1e-12


def rel_ok(a, b, floor=None):
    s = np.max(np.abs(b)) if floor is None else floor
    return np.all(np.abs(a - b) <= TOL * np.maximum(np.abs(b), s))


def test_port_gauss(golden, port_oracle):
    x, w = port_oracle.gauss()
    assert np.allclose(x, golden["gauss_x"], rtol=0, atol=4e-16)
    assert np.allclose(w, golden["gauss_w"], rtol=0, atol=4e-16)


def test_port_bspline_window(golden, port_oracle):
    W, X, N = golden["bsp_windows"], golden["bsp_x"], golden["bsp_N"]
    KX = [0, 1, 0, 0, 2, 1, 1, 0, 0, 0]
    KY = [0, 0, 1, 0, 0, 1, 0, 2, 1, 0]
    KZ = [0, 0, 0, 1, 0, 0, 1, 0, 1, 2]
    for t in range(W.shape[0]):
        tabs = [port_oracle.bspline_window(W[t, d], X[t, d]) for d in range(3)]
        mine = np.zeros((27, 10))
        for a in range(27):
            for al in range(10):
                mine[a, al] = tabs[0][a // 9, KX[al]] * tabs[1][(a // 3) % 3, KY[al]] * tabs[2][a % 3, KZ[al]]
        assert rel_ok(mine, N[t])


def test_port_evalN(golden, port_oracle):
    kv, xs, ev = golden["evaln_kv"], golden["evaln_x"], golden["evaln_val"]
    for k in range(3):
        for i in range(ev.shape[1]):
            for j, x in enumerate(xs):
                v = port_oracle.bspline_any(kv, k, i, x)
                assert abs(v - ev[k, i, j]) <= 1e-11 * max(1.0, abs(ev[k, i, j])), (k, i, x, v, ev[k, i, j])


def test_port_ge_point(golden, port_oracle):
    for p, par in enumerate(golden["ge_par"]):
        for t, u in enumerate(golden["ge_u"]):
            r, D = port_oracle.ge_point(u, par)
            assert rel_ok(r, golden["ge_r"][p, t])
            assert rel_ok(D, golden["ge_D"][p, t])


@pytest.mark.parametrize("name", ["tiny_default", "ragged_config0", "perturbed_lame", "mixed_bc", "config0_8"])
def test_port_residual_golden(golden, port_oracle, name):
    c = make_case(name)
    P = port_oracle.PortCase(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                             c["par_dirichlet"], c["par_neumann"])
    R = P.residual(c["U"])
    ref = golden["case_%s_R" % name]
    assert np.all(np.abs(R - ref) <= residual_tolerance(ref))


@pytest.mark.parametrize("name", ["tiny_default", "ragged_config0"])
def test_port_tangent_golden(golden, port_oracle, name):
    c = make_case(name)
    P = port_oracle.PortCase(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                             c["par_dirichlet"], c["par_neumann"])
    rp, cols, v = P.tangent(c["U"])
    ref = golden["case_%s_V" % name]
    assert v.shape == ref.shape
    assert np.all(np.abs(v - ref) <= tangent_tolerance(rp, ref))


def test_reference_reproduces_golden(golden, oracle_lib):
    """The in-place reference build still produces the committed vectors."""
    for name in ["ragged_config0", "mixed_bc"]:
        c = make_case(name)
        C = oracle_lib.case("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                            c["par_dirichlet"], c["par_neumann"])
        R = C.residual(c["U"])
        assert np.array_equal(R, golden["case_%s_R" % name])


def test_struct_layouts_match_reference(oracle_lib):
    a, b = oracle_lib.layouts()
    assert len(a) == len(b) and np.array_equal(a, b)


def test_port_matches_reference_random(oracle_lib, port_oracle):
    """Seeded extra cases beyond the golden set: uneven sizes, random BC tables."""
    from igap4standard_b200 import mesh
    rng = np.random.default_rng(99)
    for trial in range(3):
        nelem = tuple(int(x) for x in rng.integers(1, 4, 3))
        kn = mesh.knots_for(nelem, perturb=0.15, seed=trial)
        pm = mesh.par_mat_from_lame(*rng.uniform(0.5, 2.0, 2), rng.uniform(0.05, 0.2))
        bc = rng.integers(0, 2, 36).astype(np.int32)
        pd, pp = rng.uniform(-0.03, 0.03, 9), rng.uniform(-0.01, 0.01, 9)
        pn = rng.uniform(-0.1, 0.1, 39)
        U = rng.uniform(-0.02, 0.02, mesh.n_dof(nelem))
        args = (nelem, kn, pm, bc, pp, pd, pn)
        R_ref = oracle_lib.case("ge", *args).residual(U)
        R = port_oracle.PortCase(*args).residual(U)
        assert np.all(np.abs(R - R_ref) <= residual_tolerance(R_ref))
        rp_r, c_r, v_r = oracle_lib.case("ge", *args).tangent(U)
        rp, cc, v = port_oracle.PortCase(*args).tangent(U)
        assert np.array_equal(rp, rp_r) and np.array_equal(cc, c_r)
        assert np.all(np.abs(v - v_r) <= tangent_tolerance(rp_r, v_r))


def test_reference_intdensity_known_answers(oracle_lib):
    """The reference's iga_intdensity (src/iga_intdensity.c) on states with closed-form
    integrals (unit cube): every phys/ge density vanishes at rest; for phys/getime with
    U_hist[2] = 0 and U_hist[1] = c e_x at every control point (partition of unity:
    a rigid shift) the midpoint energy vanishes and HH[0] = rho c^2 / (2 dt^2), and
    HH[1] is minus the Neumann area (phys/getime/density.c:61), one unit face per
    (face, order, dof) combination marked Neumann."""
    from igap4standard_b200 import mesh
    nelem = (3, 2, 4)
    kn = mesh.knots_for(nelem, perturb=0.1, seed=2)
    bc, pd = mesh.bc_config0()
    pn = np.zeros(39)
    C = oracle_lib.case("ge", nelem, kn, mesh.par_mat_from_lame(1.0, 1.0, 0.1), bc, np.zeros(9), pd, pn)
    C.set_history(0, np.zeros(C.ndof))
    assert np.array_equal(C.intdensity(13), np.zeros(13))
    pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
    rho, dt, c = 1.7, 2e-3, 3e-3
    pm[5], pm[7] = rho, dt
    T = oracle_lib.case("getime", nelem, kn, pm, bc, np.zeros(9), pd, pn)
    U1 = np.zeros(T.ndof)
    U1[0::3] = c
    T.set_history(0, U1)
    T.set_history(1, U1)
    T.set_history(2, np.zeros(T.ndof))
    HH = T.intdensity(2)
    n_neumann = int(np.sum(np.asarray(bc) == 1))
    assert abs(HH[0] - rho * c * c / (2 * dt * dt)) <= 1e-12 * rho * c * c / (2 * dt * dt)
    assert abs(HH[1] + n_neumann) <= 1e-13 * max(n_neumann, 1)
