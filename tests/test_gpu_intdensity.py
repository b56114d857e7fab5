"""Integrated densities (src/iga_intdensity.c) on the GPU against the reference's
own iga_intdensity (oracle/_ref) on the same case, state and tractions.

phys/ge: 13 densities (energy, stresses, volume-fraction indicators) with the
Neumann work on standard and high-order faces and the periodic term;
phys/getime: the energy at the midpoint of history levels 1 and 2 plus the
kinetic energy, and the Neumann area.  Criterion: every density within
1e-12 relative, with a floor of the largest continuous density of the case
for the continuous ones (sums of terms of both signs) and of the volume (1)
for the indicator integrals (sums of Gauss weights)."""
import numpy as np
import pytest

from cases import make_case, make_transient_case, neumann_values

pytestmark = pytest.mark.gpu

CASES = ["tiny_default", "ragged_config0", "perturbed_lame", "mixed_bc", "config0_8"]
GE_CONT = list(range(7))      # energy, stresses
GE_IND = list(range(7, 13))   # volume fractions


def _assembly(c, phys="ge"):
    from igap4standard_b200 import Assembly
    A = Assembly(c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_dirichlet"], c["par_periodic"],
                 phys=phys)
    xyz, meta = A.neumann_points()
    if len(xyz):
        A.set_neumann_values(neumann_values(xyz, meta, c["par_neumann"]))
    return A


def _args(c, phys="ge"):
    return (phys, c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"], c["par_dirichlet"],
            c["par_neumann"])


def _check(name, HH, ref, cont, ind):
    tol = np.zeros_like(ref)
    scale = np.abs(ref[cont]).max()
    tol[cont] = 1e-12 * np.maximum(np.abs(ref[cont]), scale)
    tol[ind] = 1e-12 * np.maximum(np.abs(ref[ind]), 1.0)
    err = np.abs(HH - ref)
    worst = float(np.max(err / np.maximum(tol, 1e-300)))
    print("%s: HH %s\n  max |diff| %.3e, worst diff/tol %.3f" % (name, np.array2string(ref, precision=6),
                                                                 err.max(), worst))
    return worst


@pytest.mark.parametrize("name", CASES)
def test_ge_intdensity_matches_reference(built, oracle_lib, name):
    c = make_case(name)
    ref = oracle_lib.case(*_args(c))
    ref.set_history(0, c["U"])
    HH_ref = ref.intdensity(13)
    A = _assembly(c)
    HH = A.intdensity(c["U"])
    assert HH.shape == (13,)
    assert np.abs(HH_ref[GE_CONT]).max() > 0.0
    assert _check(name, HH, HH_ref, GE_CONT, GE_IND) <= 1.0


@pytest.mark.parametrize("name", ["getime_small", "getime_config2"])
def test_getime_intdensity_matches_reference(built, oracle_lib, name):
    c = make_transient_case(name)
    ref = oracle_lib.case(*_args(c, "getime"))
    ref.set_history(0, c["U"])
    ref.set_history(1, c["U1"])
    ref.set_history(2, c["U0"])
    HH_ref = ref.intdensity(2)
    A = _assembly(c, "getime")
    A.set_history(1, c["U1"])
    A.set_history(2, c["U0"])
    HH = A.intdensity(c["U"])
    assert HH.shape == (2,)
    # HH[1] is minus the Neumann area (phys/getime/density.c:61): exact sums of weights
    assert HH_ref[1] < 0.0
    assert _check(name, HH, HH_ref, [0], [1]) <= 1.0


def test_dropin_intdensity(built, oracle_lib):
    """iga_intdensity of the drop-in library (libsnesiga_b200) after a residual call
    (which leaves the iterate in U_hist level 0, as the reference's callbacks do)."""
    from igap4standard_b200 import gpu_case
    c = make_case("perturbed_lame")
    ref = oracle_lib.case(*_args(c))
    gpu = gpu_case(*_args(c))
    ref.residual(c["U"])
    gpu.residual(c["U"])
    HH_ref = ref.intdensity(13)
    HH = gpu.intdensity(13)
    assert _check("dropin", HH, HH_ref, GE_CONT, GE_IND) <= 1.0


def test_intdensity_deterministic(built):
    c = make_case("config0_8")
    A = _assembly(c)
    assert np.array_equal(A.intdensity(c["U"]), A.intdensity(c["U"] * 1.0))
