"""Failure paths of the drop-in and the library, made on the host.

The reference's error model is assert / exit (e.g. src/snesiga_Residual.c:227,
:241, mesh/nurbs/eval_Bspline.c:59); the callbacks here return a nonzero
PetscErrorCode instead, so PETSc's SNES sees the failure and the process lives on:
  * a NaN planted in the host U: the residual and the tangent report PETSC_ERR_FP,
    and the next call with a finite U succeeds;
  * a bad boundary table (a bc_type entry other than 0 / 1) or knot count
    (nurbs->nknot != nelem + 5): PETSC_ERR_SUP before any device work;
  * a truncated solution file: an error, and the caller's array stays as it was.
Nothing here faults, traps or hangs a GPU: every failure is made on the host."""
import ctypes

import numpy as np
import pytest

from cases import make_case

PETSC_ERR_SUP = 56
PETSC_ERR_FP = 72


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _args(c, bc=None):
    return ("ge", c["nelem"], c["knots"], c["par_mat"], c["bc_type"] if bc is None else bc, c["par_periodic"],
            c["par_dirichlet"], c["par_neumann"])


def _rc_of(fn, *a):
    try:
        fn(*a)
    except RuntimeError as e:
        return int(str(e).rsplit(" ", 1)[-1])
    return 0


def test_bad_bc_type_is_unsupported(built):
    """Checked in igab_create before the first CUDA call: no GPU needed."""
    from igap4standard_b200 import IgabError, Assembly, gpu_case
    c = make_case("ragged_config0")
    bc = np.array(c["bc_type"]).copy()
    bc[7] = 2
    G = gpu_case(*_args(c, bc))
    assert _rc_of(G.residual, c["U"]) == PETSC_ERR_SUP
    assert _rc_of(G.tangent, c["U"]) == PETSC_ERR_SUP
    G.close()
    with pytest.raises(IgabError) as e:
        Assembly(c["nelem"], c["knots"], c["par_mat"], bc, c["par_dirichlet"])
    assert e.value.code == 1


def test_truncated_solution_file(built, tmp_path):
    from igap4standard_b200 import native, gpu_case
    lib = native.lib_cuda()
    n = 300
    f = str(tmp_path / "short.bin").encode()
    np.arange(2 * n - 1, dtype=np.float64).tofile(f.decode())     # one value short of two levels
    U = np.full((2, n), 7.0)
    assert lib.igab_read_solution(f, _p(U), n, 0, 2) == 1
    assert b"fewer" in lib.igab_last_error()
    assert np.all(U == 7.0)                                        # nothing was read into U
    c = make_case("ragged_config0")                                # 240 dofs: drop-in reader, level 0
    G = gpu_case(*_args(c))
    io = G.lib.iga_case_iocomm(G.h)
    np.arange(G.ndof - 1, dtype=np.float64).tofile(f.decode())
    H = np.full(G.ndof, 3.0)
    G.lib.read_solution(f, _p(H), io, 0, 1)                       # prints the error, returns
    assert np.all(H == 3.0)
    G.close()


@pytest.mark.gpu
def test_nonfinite_state_is_reported_and_recovered(built):
    from igap4standard_b200 import gpu_case
    c = make_case("perturbed_lame")
    G = gpu_case(*_args(c))
    R_good = G.residual(c["U"])
    bad = c["U"].copy()
    bad[17] = np.nan
    assert _rc_of(G.residual, bad) == PETSC_ERR_FP
    assert _rc_of(G.tangent, bad) == PETSC_ERR_FP
    bad[17] = np.inf
    assert _rc_of(G.residual, bad) == PETSC_ERR_FP
    assert np.array_equal(G.residual(c["U"]), R_good)             # the context stays usable
    rp, cols, v = G.tangent(c["U"])
    assert np.all(np.isfinite(v))
    G.close()


class _NurbsHead(ctypes.Structure):
    """The leading members of Nurbs (include/igap4_structs.h, the reference's include/nurbs.h:4-8)."""
    _fields_ = [("porder", ctypes.c_int), ("nelem", ctypes.POINTER(ctypes.c_int)),
                ("nbasis", ctypes.POINTER(ctypes.c_int)), ("nknot", ctypes.POINTER(ctypes.c_int))]


class _IGAHead(ctypes.Structure):
    _fields_ = [("phys", ctypes.c_void_p), ("nurbs", ctypes.POINTER(_NurbsHead)), ("bc", ctypes.c_void_p)]


@pytest.mark.gpu
def test_bad_knot_count_is_unsupported(built):
    """The GPU state is rebuilt from the structs after snesiga_gpu_free; a knot count the
    B200 path cannot take (nknot != nelem + 5) is refused with PETSC_ERR_SUP."""
    from igap4standard_b200 import gpu_case, native
    c = make_case("ragged_config0")
    G = gpu_case(*_args(c))
    lib = native.lib_dropin()
    app = ctypes.cast(G.app, ctypes.POINTER(_IGAHead))
    nk = app.contents.nurbs.contents.nknot
    assert nk[0] == c["nelem"][0] + 5
    assert lib.snesiga_gpu_free(G.app) == 0
    nk[0] += 1
    assert _rc_of(G.residual, c["U"]) == PETSC_ERR_SUP
    nk[0] -= 1
    assert np.all(np.isfinite(G.residual(c["U"])))
    G.close()
