"""Seeded cases shared by the parity tests."""
import zlib

import numpy as np

from igap4standard_b200 import mesh


def neumann_values(xyz, meta, pn):
    """The case builder's traction hook (iga_case_neumann) evaluated in numpy."""
    f, o, d = meta[:, 0], meta[:, 1], meta[:, 2]
    s = 1.0 + pn[36] * xyz[:, 0] + pn[37] * xyz[:, 1] + pn[38] * xyz[:, 2]
    return pn[6 * f + 3 * o + d] * s


def make_case(name):
    """Returns dict(phys, nelem, knots, par_mat, bc_type, par_dirichlet, par_periodic, par_neumann, U)."""
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "tiny_default":          # 1 element, reference default material, example BCs
        nelem = (1, 1, 1)
        kn = mesh.knots_for(nelem)
        pm = mesh.PAR_MAT_DEFAULT.copy()
        bc, pd = mesh.bc_example()
        pp = np.zeros(9)
        pn = np.zeros(39)
        amp = 1e-3
    elif name == "ragged_config0":      # ragged tiles, config-0 BCs, default material
        nelem = (2, 3, 5)
        kn = mesh.knots_for(nelem)
        pm = mesh.PAR_MAT_DEFAULT.copy()
        bc, pd = mesh.bc_config0()
        pp = np.zeros(9)
        pn = np.zeros(39)
        amp = 1e-3
    elif name == "perturbed_lame":      # perturbed knots, (lambda, mu, l) mapping, traction + periodic term
        nelem = (4, 4, 4)
        kn = mesh.knots_for(nelem, perturb=0.1, seed=1)
        pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
        bc, pd = mesh.bc_config0()
        pd = rng.uniform(-0.02, 0.02, 9)
        pp = rng.uniform(-0.01, 0.01, 9)
        pn = rng.uniform(-0.05, 0.05, 39)
        pn[36:39] = rng.uniform(-0.5, 0.5, 3)
        amp = 1e-2
    elif name == "mixed_bc":            # every face mixes Dirichlet/Neumann per dof and order
        nelem = (3, 2, 4)
        kn = mesh.knots_for(nelem, perturb=0.2, seed=7)
        pm = mesh.par_mat_from_lame(0.7, 1.3, 0.15)
        bc = rng.integers(0, 2, 36).astype(np.int32)
        pd = rng.uniform(-0.05, 0.05, 9)
        pp = np.zeros(9)
        pn = rng.uniform(-0.1, 0.1, 39)
        amp = 5e-2
    elif name == "config0_8":           # BASELINE config 0 shape (8^3), seeded state in +-1e-3
        nelem = (8, 8, 8)
        kn = mesh.knots_for(nelem)
        pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
        bc, pd = mesh.bc_config0()
        pp = np.zeros(9)
        pn = np.zeros(39)
        amp = 1e-3
    elif name == "newton_backtrack":    # strong Dirichlet pull: the first full Newton step is rejected
        nelem = (3, 3, 3)
        kn = mesh.knots_for(nelem, perturb=0.1, seed=3)
        pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
        bc, pd = mesh.bc_config0()
        pd = np.zeros(9)
        pd[0] = 0.3
        pp = np.zeros(9)
        pn = np.zeros(39)
        amp = 1e-3
    else:
        raise KeyError(name)
    ndof = mesh.n_dof(nelem)
    U = np.random.default_rng(0).uniform(-amp, amp, ndof)
    return dict(phys="ge", nelem=nelem, knots=kn, par_mat=pm, bc_type=bc, par_dirichlet=pd,
                par_periodic=pp, par_neumann=pn, U=U)


def residual_tolerance(ref):
    """Per-entry bound |gpu - ref| <= 1e-12 * max(|ref_i|, scale): the reference sums
    element contributions whose size is ~||R||_inf, so an entry that cancels to ~0
    carries rounding of that size (survey parity criterion with a cancellation floor)."""
    scale = np.max(np.abs(ref)) if ref.size else 0.0
    return 1e-12 * np.maximum(np.abs(ref), scale)


def tangent_tolerance(rowptr, vals_ref):
    """|gpu - ref| <= 1e-12 * max(|ref|, ||ref row||_inf)."""
    rowmax = np.maximum.reduceat(np.abs(vals_ref), rowptr[:-1]) if vals_ref.size else np.zeros(0)
    per = np.repeat(rowmax, np.diff(rowptr))
    return 1e-12 * np.maximum(np.abs(vals_ref), per)


def make_transient_case(name):
    """Seeded phys/getime cases: dict as make_case plus U1 (t_n) and U0 (t_{n-1})."""
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "getime_small":        # reference default material (dt = 5e-4), example BCs
        nelem = (2, 3, 2)
        kn = mesh.knots_for(nelem, perturb=0.1, seed=4)
        pm = mesh.PAR_MAT_DEFAULT.copy()
        bc, pd = mesh.bc_example()
        amp = 1e-3
    elif name == "getime_config2":    # BASELINE config-2 physics: rho = 1, dt = 1e-3, traction on x = 1
        nelem = (3, 2, 3)
        kn = mesh.knots_for(nelem)
        pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
        pm[5], pm[6], pm[7] = 1.0, 1.0, 1e-3
        bc, pd = mesh.bc_config0()
        amp = 2e-2
    else:
        raise KeyError(name)
    pn = np.zeros(39)
    pn[6 + 0] = 0.01                  # face 1, standard order, x-dof traction
    ndof = mesh.n_dof(nelem)
    U0 = rng.uniform(-amp, amp, ndof)
    U1 = U0 + rng.uniform(-amp, amp, ndof) * 0.3
    U = U1 + rng.uniform(-amp, amp, ndof) * 0.3
    return dict(phys="getime", nelem=nelem, knots=kn, par_mat=pm, bc_type=bc, par_dirichlet=pd,
                par_periodic=np.zeros(9), par_neumann=pn, U=U, U1=U1, U0=U0)
