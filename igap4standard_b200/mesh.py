"""Mesh, material and boundary-condition set-up for single-rank IGA cases.

The reference builds open uniform knot vectors (mesh/nurbs/nurbs_genuniform.c:36-38)
with 2^mref elements; here any element count is allowed and interior knots can
be perturbed (the reference's disabled hook at nurbs_genuniform.c:37 perturbs
knots the same way), because physical coordinates are knot coordinates
(mesh/nurbs/eval_Bspline.c:64-74) and there is no separate geometry map.
"""
import numpy as np

P = 2  # quadratic C1 B-splines (eval_Bspline requires p == 2)

# par_mat of phys/ge/init.c:17-18 and phys/getime/init.c:17-18
PAR_MAT_DEFAULT = np.array([0.25, 0.50, 500.0, 250.0, 0.025, 1.0, 1.0, 1.0e-3 * 0.5, 0.0])


def open_knot_vector(n, perturb=0.0, rng=None, length=1.0):
    """Open knot vector on [0, length] with n elements: p+1 repeated end knots.

    perturb: interior knots move by uniform(-perturb*h, +perturb*h), h = length/n
    (must stay below 0.5 so the knots stay increasing)."""
    if n < 1:
        raise ValueError("n must be >= 1")
    if not 0.0 <= perturb < 0.5:
        raise ValueError("perturb must be in [0, 0.5)")
    h = length / n
    inner = np.arange(1, n) * h
    if perturb > 0 and n > 1:
        rng = rng if rng is not None else np.random.default_rng(0)
        inner = inner + rng.uniform(-perturb * h, perturb * h, size=n - 1)
    return np.concatenate([np.zeros(P + 1), inner, np.full(P + 1, length)])


def knots_for(nelem, perturb=0.0, seed=0):
    """Three knot vectors back to back (the igab_mesh_desc.knots layout)."""
    rng = np.random.default_rng(seed)
    return np.concatenate([open_knot_vector(int(n), perturb, rng) for n in nelem])


def par_mat_from_lame(lam, mu, ell, r=10.0, base=PAR_MAT_DEFAULT):
    """Map (lambda, mu, strain-gradient length) onto phys/ge's par_mat.

    The quadratic part of the ge energy (phys/ge/density.c:49) is
    e0*vvol^2 + e345*(E01^2+E02^2+E12^2) + c37*(va^2+vb^2); matching the
    St-Venant-Kirchhoff energy lambda/2 tr(E)^2 + mu E:E gives e0 = 3 lambda/2 + mu,
    e345 = 2 mu, c37 = mu.  c37 = -6 curv / (r^2 (1 + 2 curv)) (phys/ge/residual.c:45-47),
    so curv = -mu r^2 / (6 + 2 mu r^2); le = ell."""
    pm = np.array(base, dtype=np.float64).copy()
    curv = -mu * r * r / (6.0 + 2.0 * mu * r * r)
    pm[0] = r
    pm[1] = curv
    pm[2] = 1.5 * lam + mu
    pm[3] = 2.0 * mu
    pm[4] = ell
    return pm


def ge_coefficients(par):
    """(c36, c37, c38) of the energy for a par_mat (phys/ge/residual.c:36-38)."""
    r, cu = par[0], par[1]
    q = 1.3333333333333333 * r - 1.3333333333333333 * r * cu
    den = r * r - 2 * (r * r) * cu - r * q
    return (-(q / ((r * r) * den)), (2 * cu) / den, -(1 / ((r * r) * den)))


def bc_config0():
    """BCs of the static configs: face 0 (x=0) u = 0 and du/dn = 0; face 1 (x=1)
    u_x Dirichlet, the rest traction-free; faces 2-5 traction-free.
    Returns (bc_type[36], par_dirichlet[9]) with u_x = 0.01 X on the Dirichlet faces."""
    bc = np.ones(36, dtype=np.int32)
    bc[0:6] = 0
    bc[6] = 0
    pd = np.zeros(9)
    pd[0] = 0.01
    return bc, pd


def bc_transient():
    """BCs of the transient workload: face 0 (x=0) u = 0 and du/dn = 0; every other
    face traction-driven (the x = 1 traction is the Neumann value of face 1, order 0,
    dof x).  Returns (bc_type[36], par_dirichlet[9] = 0)."""
    bc = np.ones(36, dtype=np.int32)
    bc[0:6] = 0
    return bc, np.zeros(9)


def bc_example():
    """bc_init of the reference example (example/ex1/main.c:69-95): u = 0 on every
    face, high-order Neumann everywhere."""
    row = [0, 0, 0, 1, 1, 1]
    return np.array(row * 6, dtype=np.int32), np.zeros(9)


def greville(kv):
    """Greville abscissae of a p = 2 knot vector: (k[j+1] + k[j+2]) / 2, one per basis
    function.  Control values a + b x_j at these points reproduce the linear function
    a + b x exactly (B-splines of degree >= 1)."""
    kv = np.asarray(kv, dtype=np.float64)
    return 0.5 * (kv[1:-2] + kv[2:-1])


def affine_field(nelem, knots, F0):
    """Control values (dof = 3 cp + i, cp = (x nb1 + y) nb2 + z) of u_i(X) = sum_j F0[i][j] X_j
    on the mesh: the affine map the Dirichlet values reproduce (src/iga_dirichlet.c:10-12,
    par_dirichlet = F0 row-major), so this field satisfies every Dirichlet row (values and
    normal derivatives) of any bc_type table exactly."""
    nelem = [int(n) for n in nelem]
    kv, off = [], 0
    for n in nelem:
        kv.append(np.asarray(knots[off:off + n + 5], dtype=np.float64))
        off += n + 5
    gx, gy, gz = (greville(k) for k in kv)
    X = np.stack(np.meshgrid(gx, gy, gz, indexing="ij"), axis=-1).reshape(-1, 3)
    F = np.asarray(F0, dtype=np.float64).reshape(3, 3)
    return (X @ F.T).reshape(-1)


def n_dof(nelem):
    return 3 * int(np.prod(np.asarray(nelem) + P))


def nnz_of(nelem):
    nnz = 9
    for n in nelem:
        m = int(n) + P
        nnz *= m + 2 * max(m - 1, 0) + 2 * max(m - 2, 0)
    return nnz


def batch_config3(n_instances=512, seed=3, nmin=6, nmax=24, perturb=0.0):
    """Seeded instances of the batched static workload: n^3 elements with n uniform
    in [nmin, nmax] per instance, lambda and mu lognormal(0, 0.25), strain-gradient
    length uniform in [0.05, 0.2], BCs of bc_config0.  Returns a list of dicts
    (nelem, knots, par_mat, bc_type, par_dirichlet)."""
    rng = np.random.default_rng(seed)
    out = []
    bc, pd = bc_config0()
    for _ in range(n_instances):
        n = int(rng.integers(nmin, nmax + 1))
        nelem = (n, n, n)
        lam, mu = np.exp(rng.normal(0.0, 0.25, 2))
        ell = rng.uniform(0.05, 0.2)
        kseed = int(rng.integers(0, 2 ** 31 - 1))
        out.append(dict(nelem=nelem, knots=knots_for(nelem, perturb, kseed), par_mat=par_mat_from_lame(lam, mu, ell),
                        bc_type=bc.copy(), par_dirichlet=pd.copy()))
    return out
