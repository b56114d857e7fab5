#!/usr/bin/env python3
"""Generate tests/golden/reference_vectors.npz from IGAP4STANDARD's own code.

Runs only where the reference tree is present (it drives oracle/_ref, the
reference sources compiled in place by oracle/build_ref.py).  The vectors
are small, seeded, and pin both CPU oracles and the host-compiled point
mathematics of the product:
  gauss_x/gauss_w        legendre_handle(n=4, [0,1])            src/quadrature.c:381
  bsp_*                  eval_Bspline at random windows/points    mesh/nurbs/eval_Bspline.c:9
  evaln_*                evalN incl. derivatives at end points    mesh/nurbs/evalN.c:7
  ge_*                   ge_residual / ge_tangent at random points phys/ge/residual.c, tangent.c
  getime_*               getime_residual / getime_tangent          phys/getime/residual.c, tangent.c
  case_<name>_R          snesiga_Residual on the seeded test cases  src/snesiga_Residual.c:13
  case_<name>_V          snesiga_Tangent CSR values (small cases)   src/snesiga_Tangent.c:13
Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import ref  # noqa: E402
from cases import make_case  # noqa: E402
from igap4standard_b200 import mesh  # noqa: E402

OUT = os.path.join(HERE, "reference_vectors.npz")
RESIDUAL_CASES = ["tiny_default", "ragged_config0", "perturbed_lame", "mixed_bc", "config0_8"]
TANGENT_CASES = ["tiny_default", "ragged_config0"]


def main():
    if not ref.available():
        print("oracle/_ref is not built; run python oracle/build_ref.py first")
        return 1
    rng = np.random.default_rng(2024)
    g = {}
    g["gauss_x"], g["gauss_w"] = ref.gauss(4)
    # eval_Bspline on random 6-knot windows (open and interior)
    wins, xs, Ns = [], [], []
    for t in range(12):
        w3 = []
        x3 = []
        for d in range(3):
            kv = np.sort(rng.uniform(0, 1, 6))
            if t % 3 == 0:
                kv[:3] = kv[0]   # clamped start
            w3.append(kv)
            x3.append(rng.uniform(kv[2], kv[3]))
        wins.append(np.stack(w3))
        xs.append(np.array(x3))
        Ns.append(ref.eval_bspline(w3, x3))
    g["bsp_windows"], g["bsp_x"], g["bsp_N"] = np.stack(wins), np.stack(xs), np.stack(Ns)
    # evalN on a perturbed open knot vector, interior and end points, k = 0, 1, 2
    kv = mesh.open_knot_vector(6, perturb=0.2, rng=np.random.default_rng(5))
    pts = np.concatenate([rng.uniform(0, 1, 8), [0.0, 1.0, 1.0 - 1e-15]])
    ev = np.zeros((3, 8, pts.size))
    for k in range(3):
        for i in range(8):
            for j, x in enumerate(pts):
                ev[k, i, j] = ref.evalN(kv, k, i, x)
    g["evaln_kv"], g["evaln_x"], g["evaln_val"] = kv, pts, ev
    # point integrands
    pars = np.stack([mesh.PAR_MAT_DEFAULT, mesh.par_mat_from_lame(1.0, 1.0, 0.1)])
    us = rng.uniform(-0.1, 0.1, (8, 30))
    g["ge_par"], g["ge_u"] = pars, us
    g["ge_r"] = np.stack([[ref.ge_residual(u, p) for u in us] for p in pars])
    g["ge_D"] = np.stack([[ref.ge_tangent(u, p) for u in us] for p in pars])
    u90 = rng.uniform(-0.05, 0.05, (4, 90))
    pt = mesh.PAR_MAT_DEFAULT.copy()
    g["getime_par"], g["getime_u"] = pt, u90
    g["getime_r"] = np.stack([ref.getime_residual(u, pt) for u in u90])
    g["getime_D"] = np.stack([ref.getime_tangent(u, pt) for u in u90])
    # assembled operators on the seeded cases
    for name in RESIDUAL_CASES:
        c = make_case(name)
        C = ref.case("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"],
                     c["par_dirichlet"], c["par_neumann"])
        g["case_%s_R" % name] = C.residual(c["U"])
        if name in TANGENT_CASES:
            rp, cols, v = C.tangent(c["U"])
            g["case_%s_V" % name] = v
    np.savez_compressed(OUT, **g)
    print("wrote %s (%.0f KB)" % (OUT, os.path.getsize(OUT) / 1024))
    return 0


if __name__ == "__main__":
    sys.exit(main())
