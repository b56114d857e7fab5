"""Seeded meshes with periodic directions (shared by the CPU and GPU periodic tests)."""
import numpy as np

from igap4standard_b200 import mesh


def periodic_knots(n, perturb=0.0, seed=0):
    """Uniform periodic knot vector of mesh/nurbs/nurbs_genuniform.c:40-43 (n + 5 knots,
    spacing 1/n, starting at -2/n); perturb moves the interior knots 0 < t < 1 by up to
    perturb * h and the two extension knots at each end follow their images (t -/+ 1)."""
    h = 1.0 / n
    t = np.array([(i - 2) * h for i in range(n + 5)])
    if perturb:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-perturb * h, perturb * h, n - 1)   # interior knots i = 3 .. n + 1
        t[3:n + 2] += d
        t[0], t[1] = t[n] - 1.0, t[n + 1] - 1.0             # images of the knots below 1
        t[n + 3], t[n + 4] = t[3] + 1.0, t[4] + 1.0         # images of the knots above 0
    return t


def make_periodic_case(per, nelem=(5, 4, 3), seed=0, phys="ge", perturb=0.1):
    """Knots (periodic directions uniform-extended, others open and perturbed), material,
    a BC table with Dirichlet and Neumann rows on the non-periodic faces, a traction, a
    seeded state.  Returns a dict as tests/cases.py's make_case plus bc_periodic."""
    rng = np.random.default_rng(seed)
    kn = []
    for d in range(3):
        if per[d]:
            kn.append(periodic_knots(nelem[d], perturb, seed + d))
        else:
            kn.append(mesh.knots_for((nelem[d], 1, 1), perturb=perturb, seed=seed + d)[:nelem[d] + 5])
    lam, mu = np.exp(rng.normal(0.0, 0.2, 2))
    pm = mesh.par_mat_from_lame(lam, mu, 0.1)
    if phys == "getime":
        pm[5], pm[6], pm[7] = 1.0, 1.0, 1e-2
    bc = rng.integers(0, 2, 36).astype(np.int32)
    pd = rng.uniform(-0.05, 0.05, 9)
    pn = np.zeros(39)
    pn[:36] = rng.uniform(-0.02, 0.02, 36)
    pn[36:39] = rng.uniform(-0.5, 0.5, 3)
    pp = rng.uniform(-0.01, 0.01, 9)
    nb = [nelem[d] if per[d] else nelem[d] + 2 for d in range(3)]
    ndof = 3 * nb[0] * nb[1] * nb[2]
    U = rng.uniform(-2e-3, 2e-3, ndof)
    return dict(nelem=tuple(nelem), knots=np.concatenate(kn), par_mat=pm, bc_type=bc, par_dirichlet=pd,
                par_neumann=pn, par_periodic=pp, U=U, bc_periodic=tuple(per), phys=phys)


PERIODIC = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1), (1, 1, 1)]
