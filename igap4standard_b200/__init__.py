"""igap4standard_b200: element assembly of IGAP4STANDARD on NVIDIA B200.

Residual and tangent of the SNES callbacks (C1 quadratic B-splines, phys/ge
strain-gradient elasticity, Dirichlet and higher-order boundary conditions,
scatter into the AIJ pattern) as hand-written sm_100a kernels behind a C ABI
(include/igab.h) and a PETSc drop-in (include/snesiga_b200.h).
"""
from .native import NativeLibraryMissing, IgabError, lib_cuda, lib_dropin
from .mesh import (open_knot_vector, knots_for, par_mat_from_lame, bc_config0, bc_example,
                   n_dof, nnz_of, affine_field, PAR_MAT_DEFAULT)
from .assembly import Assembly
from .batch import Batch
from .case import Case, gpu_case

__all__ = ["NativeLibraryMissing", "IgabError", "lib_cuda", "lib_dropin", "open_knot_vector", "knots_for",
           "par_mat_from_lame", "bc_config0", "bc_example", "n_dof", "nnz_of", "PAR_MAT_DEFAULT",
           "Assembly", "Batch", "Case", "gpu_case"]
