"""GPU tests of the discrete adjoint of the element-scaled problem.

Every element integrand is scaled by s_e = exp(g_e) (element order of the
reference's loops).  Checked here:
  * forward: scaled residual and tangent against the reference's own CPU
    callbacks with the same scaling (oracle/elem_scale.c), 1e-12 relative;
  * backward dR/dg: grad_e = lam . dR/dg_e against the reference's element
    vectors R(s = s_e * unit_e) - R(s = 0), element by element;
  * backward K^T x: against scipy's CSR transpose product;
  * the gradient dJ/dg of J(U(g)) = 1/2 sum_{face x=1} |U - U*|^2, U(g) the
    solution of R(U, g) = 0, against central differences (h = 1e-6, 16
    seeded directions), both of the B200 solve and of the solve of the
    reference's own residual: agreement 1e-6 relative."""
import numpy as np
import pytest
import scipy.sparse as sp

from cases import make_case, make_transient_case, neumann_values, residual_tolerance, tangent_tolerance

pytestmark = pytest.mark.gpu


def _assembly(c):
    from igap4standard_b200 import Assembly
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"],
                 phys=c["phys"])
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, c["par_neumann"]))
    if c["phys"] == "getime":
        A.set_history(1, c["U1"])
        A.set_history(2, c["U0"])
    return A


def _ref_case(oracle_lib, c):
    C = oracle_lib.case(c["phys"], c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                        c["par_dirichlet"], c["par_neumann"])
    if c["phys"] == "getime":
        C.set_history(1, c["U1"])
        C.set_history(2, c["U0"])
    return C


def _log_scales(c, seed=5):
    n = int(np.prod(c["nelem"]))
    return np.random.default_rng(seed).normal(0.0, 0.3, n)


def _case(name):
    return make_transient_case(name) if name.startswith("getime") else make_case(name)


@pytest.mark.parametrize("name", ["perturbed_lame", "mixed_bc", "getime_config2"])
def test_scaled_forward_parity(built, oracle_lib, name):
    c = _case(name)
    g = _log_scales(c)
    ref = oracle_lib.ScaledCase(_ref_case(oracle_lib, c), g)
    R_ref = ref.residual(c["U"])
    rp, cols, v_ref = ref.tangent(c["U"])
    ref.close()
    A = _assembly(c)
    A.set_element_log_scale(g)
    R = A.residual(c["U"])
    assert np.max(np.abs(R - R_ref) / residual_tolerance(R_ref)) <= 1.0
    v = A.tangent(c["U"], "fp64")
    assert np.max(np.abs(v - v_ref) / tangent_tolerance(rp, v_ref)) <= 1.0
    # clearing the scales restores the unscaled operator exactly
    A.set_element_log_scale(None)
    R_plain = _ref_case(oracle_lib, c).residual(c["U"])
    assert np.max(np.abs(A.residual(c["U"]) - R_plain) / residual_tolerance(R_plain)) <= 1.0


@pytest.mark.parametrize("name", ["perturbed_lame", "getime_small"])
def test_dRdg_against_reference_element_vectors(built, oracle_lib, name):
    c = _case(name)
    g = _log_scales(c)
    n = g.size
    lam = np.random.default_rng(3).normal(size=c["U"].size)
    A = _assembly(c)
    A.set_element_log_scale(g)
    grad = A.dRdg(c["U"], lam)
    base = _ref_case(oracle_lib, c)
    off = np.full(n, -np.inf)                      # s = 0 everywhere
    R0 = oracle_lib.ScaledCase(base, off).residual(c["U"])
    ref = np.empty(n)
    bound = np.empty(n)
    for e in range(n):
        ge = off.copy()
        ge[e] = g[e]
        Re = oracle_lib.ScaledCase(base, ge).residual(c["U"]) - R0
        ref[e] = lam @ Re
        bound[e] = np.abs(lam) @ np.abs(Re)
    tol = 1e-12 * np.maximum(bound, 1e-300) + 1e-13 * np.max(bound)
    print(name, "max |grad - ref| / tol", np.max(np.abs(grad - ref) / tol))
    assert np.all(np.abs(grad - ref) <= tol)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["perturbed_lame", "ragged_config0", "config0_8"])
def test_tangent_transpose_apply(built, name, prec):
    c = make_case(name)
    A = _assembly(c)
    rp, cols = A.pattern()
    v = A.tangent(c["U"], prec)
    x = np.random.default_rng(9).normal(size=A.ndof)
    y = A.tangent_transpose_apply(v, x, prec)
    K = sp.csr_matrix((v.astype(np.float64), cols, rp), shape=(A.ndof, A.ndof))
    y_ref = K.T @ x
    bound = abs(K).T @ np.abs(x)
    assert np.all(np.abs(y - y_ref) <= 1e-14 * bound * 16 + 1e-300)


def _face_x1_mask(nelem):
    nb = [n + 2 for n in nelem]
    m = np.zeros((nb[0], nb[1], nb[2], 3))
    m[-1] = 1.0
    return m.ravel()


def _newton_tight(residual, jacobian, U0):
    """Reference driver, then plain Newton steps until ||F|| stops decreasing (FD needs U to rounding)."""
    from oracle import newton_loop as newton
    res = newton.solve(residual, jacobian, U0)
    assert res.converged
    U = res.U
    F = residual(U)
    f = np.linalg.norm(F)
    for _ in range(4):
        U1 = U - newton.direct_solve(jacobian(U), F)
        F1 = residual(U1)
        f1 = np.linalg.norm(F1)
        if not f1 < f:
            break
        U, F, f = U1, F1, f1
    return U


def test_adjoint_gradient_matches_central_differences(built, oracle_lib):
    from oracle import newton_loop as newton
    c = make_case("perturbed_lame")
    A = _assembly(c)
    n_el = int(np.prod(c["nelem"]))
    g0 = _log_scales(c)
    mask = _face_x1_mask(c["nelem"])
    Ustar = np.random.default_rng(21).uniform(-0.05, 0.05, A.ndof)

    def J(U):
        return 0.5 * np.sum(mask * (U - Ustar) ** 2)

    r_gpu, j_gpu = newton.assembly_problem(A, "fp64")
    base = _ref_case(oracle_lib, c)

    def solve_gpu(g, U0):
        A.set_element_log_scale(g)
        return _newton_tight(r_gpu, j_gpu, U0)

    def solve_ref(g, U0):
        """Zeros of the reference's own scaled residual (the GPU tangent only steers Newton)."""
        ref = oracle_lib.ScaledCase(base, g)
        A.set_element_log_scale(g)
        U = _newton_tight(ref.residual, j_gpu, U0)
        ref.close()
        return U

    U = solve_gpu(g0, np.zeros(A.ndof))
    # adjoint: K^T lam = dJ/dU at the solution, dJ/dg = -lam . dR/dg
    A.set_element_log_scale(g0)
    K = j_gpu(U)
    lam = newton.direct_solve(K.T.tocsr(), mask * (U - Ustar))
    rp, cols = A.pattern()
    vals = A.tangent(U, "fp64")
    assert np.allclose(A.tangent_transpose_apply(vals, lam), mask * (U - Ustar), rtol=0, atol=1e-12)
    grad = -A.dRdg(U, lam)

    rng = np.random.default_rng(5)
    h = 1e-6
    worst = 0.0
    for k in range(16):
        d = rng.normal(size=n_el)
        ad = grad @ d
        solver = solve_gpu if k % 2 == 0 else solve_ref
        fd = (J(solver(g0 + h * d, U)) - J(solver(g0 - h * d, U))) / (2 * h)
        err = abs(fd - ad) / max(abs(ad), 1e-3 * np.linalg.norm(grad) * np.linalg.norm(d))
        worst = max(worst, err)
        print("direction %2d (%s): adjoint %.10e  central difference %.10e  rel %.2e"
              % (k, "gpu" if k % 2 == 0 else "ref", ad, fd, err))
    assert worst <= 1e-6


def test_adjoint_gradient_config4_8cubed(built, oracle_lib):
    """Config-4 objective on an 8^3 mesh: s_e = exp(g_e), g ~ N(0, 0.3^2) (512 parameters),
    J = 1/2 sum over the face x = 1 control points of |U - U*|^2 with U* the solution at a
    second draw g*; dJ/dg by the adjoint against central differences (h = 1e-6, 16
    directions) of the B200 solve and of the reference's own scaled residual, 1e-6."""
    from igap4standard_b200 import mesh
    from oracle import newton_loop as newton
    nelem = (8, 8, 8)
    kn = mesh.knots_for(nelem, perturb=0.1, seed=1)
    pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
    bc, pd = mesh.bc_config0()
    c = dict(phys="ge", nelem=nelem, knots=kn, par_mat=pm, bc_type=bc, par_dirichlet=pd, par_periodic=np.zeros(9),
             par_neumann=np.zeros(39))
    A = _assembly(c)
    n_el = 512
    mask = _face_x1_mask(nelem)
    r_gpu, j_gpu = newton.assembly_problem(A, "fp64")
    base = _ref_case(oracle_lib, c)

    def solve_gpu(g, U0):
        A.set_element_log_scale(g)
        return _newton_tight(r_gpu, j_gpu, U0)

    def solve_ref(g, U0):
        ref = oracle_lib.ScaledCase(base, g)
        A.set_element_log_scale(g)
        U = _newton_tight(ref.residual, j_gpu, U0)
        ref.close()
        return U

    Ustar = solve_gpu(np.random.default_rng(5).normal(0.0, 0.3, n_el), np.zeros(A.ndof))
    g0 = np.random.default_rng(4).normal(0.0, 0.3, n_el)

    def J(U):
        return 0.5 * np.sum(mask * (U - Ustar) ** 2)

    U = solve_gpu(g0, np.zeros(A.ndof))
    A.set_element_log_scale(g0)
    lam = newton.direct_solve(j_gpu(U).T.tocsr(), mask * (U - Ustar))
    grad = -A.dRdg(U, lam)
    rng = np.random.default_rng(6)
    h = 1e-6
    worst = 0.0
    for k in range(16):
        d = rng.normal(size=n_el)
        ad = grad @ d
        solver = solve_gpu if k % 2 == 0 else solve_ref
        fd = (J(solver(g0 + h * d, U)) - J(solver(g0 - h * d, U))) / (2 * h)
        err = abs(fd - ad) / max(abs(ad), 1e-3 * np.linalg.norm(grad) * np.linalg.norm(d))
        worst = max(worst, err)
        print("8^3 direction %2d (%s): adjoint %.10e  central difference %.10e  rel %.2e"
              % (k, "gpu" if k % 2 == 0 else "ref", ad, fd, err))
    assert worst <= 1e-6
