"""ctypes bindings of the in-tree native libraries (built by igap4standard_b200.build).

There is no CPU fallback: if a library is missing, loading raises
NativeLibraryMissing and the caller must build it.
"""
import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(_PKG, "lib")
LIB_CUDA = os.path.join(LIBDIR, "libigap4_b200.so")
LIB_SUBSET = os.path.join(LIBDIR, "libpetsc_subset.so")
LIB_DROPIN = os.path.join(LIBDIR, "libsnesiga_b200.so")

c_int_p = ctypes.POINTER(ctypes.c_int)
c_long_p = ctypes.POINTER(ctypes.c_long)
c_double_p = ctypes.POINTER(ctypes.c_double)
vp = ctypes.c_void_p


class NativeLibraryMissing(RuntimeError):
    pass


class IgabError(RuntimeError):
    def __init__(self, where, code, msg=""):
        super().__init__("%s failed with status %d%s" % (where, code, (": " + msg) if msg else ""))
        self.code = code


class IgabTuneResult(ctypes.Structure):
    """igab_tune_result of include/igab.h"""
    _fields_ = [("residual_tile", ctypes.c_int), ("tangent_fp64_kernel", ctypes.c_int),
                ("tangent_fp32_kernel", ctypes.c_int), ("residual_ms", ctypes.c_double),
                ("tangent_fp64_ms", ctypes.c_double), ("tangent_fp32_ms", ctypes.c_double),
                ("colour_order", ctypes.c_int)]


class IgabSolveInfo(ctypes.Structure):
    """igab_solve_info of include/igab.h"""
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int), ("residual_norm", ctypes.c_double),
                ("rhs_norm", ctypes.c_double)]


class IgabNewtonOpts(ctypes.Structure):
    """igab_newton_opts of include/igab.h"""
    _fields_ = [("prec", ctypes.c_int), ("abstol", ctypes.c_double), ("rtol", ctypes.c_double),
                ("stol", ctypes.c_double), ("stagnation", ctypes.c_double), ("max_subiter", ctypes.c_int),
                ("ksp_rtol", ctypes.c_double), ("ksp_maxit", ctypes.c_int), ("ksp", ctypes.c_int),
                ("verbose", ctypes.c_int), ("fp64_polish", ctypes.c_int), ("use_graph", ctypes.c_int)]


class IgabNewtonInfo(ctypes.Structure):
    """igab_newton_info of include/igab.h"""
    _fields_ = [("iterations", ctypes.c_int), ("reason", ctypes.c_int), ("converged", ctypes.c_int),
                ("n_residual", ctypes.c_int), ("n_tangent", ctypes.c_int), ("n_tangent_fp64", ctypes.c_int),
                ("krylov_iterations", ctypes.c_long),
                ("fnorm", ctypes.c_double), ("ms_residual", ctypes.c_double), ("ms_tangent", ctypes.c_double),
                ("ms_krylov", ctypes.c_double), ("ms_total", ctypes.c_double), ("launches", ctypes.c_long)]


class IgabTransientOpts(ctypes.Structure):
    """igab_transient_opts of include/igab.h"""
    _fields_ = [("nsteps", ctypes.c_int), ("dt", ctypes.c_double), ("amplitude", ctypes.c_double),
                ("face", ctypes.c_int), ("order", ctypes.c_int), ("dof", ctypes.c_int),
                ("newton", IgabNewtonOpts)]


class IgabTransientInfo(ctypes.Structure):
    """igab_transient_info of include/igab.h"""
    _fields_ = [("steps", ctypes.c_int), ("steps_converged", ctypes.c_int), ("newton_iterations", ctypes.c_long),
                ("krylov_iterations", ctypes.c_long), ("n_residual", ctypes.c_long), ("n_tangent", ctypes.c_long),
                ("ms_total", ctypes.c_double), ("launches", ctypes.c_long)]


class IgabTadjInfo(ctypes.Structure):
    """igab_tadj_info_t of include/igab.h"""
    _fields_ = [("forward_steps", ctypes.c_int), ("recomputed_steps", ctypes.c_int), ("checkpoints", ctypes.c_int),
                ("forward_converged", ctypes.c_int), ("krylov_iterations_backward", ctypes.c_long),
                ("adjoint_solves_converged", ctypes.c_int), ("adjoint_solves", ctypes.c_int),
                ("ms_forward", ctypes.c_double), ("ms_backward", ctypes.c_double)]


class IgabBatchTuneResult(ctypes.Structure):
    """igab_batch_tune_result of include/igab.h"""
    _fields_ = [("ctas_res", ctypes.c_int), ("ctas_tan64", ctypes.c_int), ("ctas_tan32", ctypes.c_int),
                ("order", ctypes.c_int), ("residual_ms", ctypes.c_double), ("tangent_fp64_ms", ctypes.c_double),
                ("tangent_fp32_ms", ctypes.c_double), ("colour_order", ctypes.c_int)]


class IgabMeshDesc(ctypes.Structure):
    """igab_mesh_desc of include/igab.h"""
    _fields_ = [
        ("phys", ctypes.c_int),
        ("nelem", ctypes.c_int * 3),
        ("knots", c_double_p),
        ("par_mat", ctypes.c_double * 9),
        ("bc_type", ctypes.c_int * 36),
        ("par_periodic", ctypes.c_double * 9),
        ("par_dirichlet", ctypes.c_double * 9),
        ("bc_periodic", ctypes.c_int * 3),
    ]


# (name, restype, argtypes) of every entry point declared in include/igab.h
IGAB_API = [
    ("igab_create", ctypes.c_int, [ctypes.POINTER(IgabMeshDesc), ctypes.c_int, ctypes.POINTER(vp)]),
    ("igab_destroy", ctypes.c_int, [vp]),
    ("igab_last_error", ctypes.c_char_p, []),
    ("igab_version", ctypes.c_int, []),
    ("igab_sizes", ctypes.c_int, [vp, c_long_p, c_long_p, c_long_p]),
    ("igab_csr_pattern", ctypes.c_int, [vp, vp, vp]),
    ("igab_csr_offset", ctypes.c_long, [vp, ctypes.c_long, ctypes.c_long]),
    ("igab_set_par_mat", ctypes.c_int, [vp, vp]),
    ("igab_set_par_dirichlet", ctypes.c_int, [vp, vp]),
    ("igab_set_par_periodic", ctypes.c_int, [vp, vp]),
    ("igab_neumann_points", ctypes.c_int, [vp, c_long_p, vp, vp]),
    ("igab_set_neumann_values", ctypes.c_int, [vp, vp]),
    ("igab_set_history", ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int]),
    ("igab_residual", ctypes.c_int, [vp, vp, vp]),
    ("igab_residual_device", ctypes.c_int, [vp, vp, vp]),
    ("igab_tangent", ctypes.c_int, [vp, vp, vp, ctypes.c_int]),
    ("igab_tangent_device", ctypes.c_int, [vp, vp, vp, ctypes.c_int]),
    ("igab_set_stream", ctypes.c_int, [vp, vp]),
    ("igab_sync", ctypes.c_int, [vp]),
    ("igab_device_buffers", ctypes.c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_int]),
    ("igab_check_finite", ctypes.c_int, [vp, vp, ctypes.c_long, ctypes.c_int, c_int_p]),
    ("igab_set_tile", ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
    ("igab_last_launch_count", ctypes.c_int, [vp, c_int_p]),
    ("igab_set_profiling", ctypes.c_int, [vp, ctypes.c_int]),
    ("igab_last_kernel_ms", ctypes.c_int, [vp, c_double_p]),
    ("igab_fma_peak", ctypes.c_int, [ctypes.c_int, ctypes.c_int, c_double_p]),
    ("igab_dmma_peak", ctypes.c_int, [ctypes.c_int, c_double_p]),
    ("igab_residual_noalloc", ctypes.c_int, [vp, vp, vp]),
    ("igab_staging_bytes", ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_size_t)]),
    ("igab_newton_defaults", None, [vp]),
    ("igab_solve_mg_device", ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int, vp, vp, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int, vp]),
    ("igab_solve_mg_levels", ctypes.c_int, [vp, c_int_p]),
    ("igab_mg_prolongation_1d", ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int, vp]),
    ("igab_upload", ctypes.c_int, [vp, vp, vp, ctypes.c_long]),
    ("igab_download", ctypes.c_int, [vp, vp, vp, ctypes.c_long]),
    ("igab_newton_solve", ctypes.c_int, [vp, vp, vp, vp, vp, vp, ctypes.c_int]),
    ("igab_transient_defaults", None, [vp]),
    ("igab_transient_run", ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp]),
    ("igab_tadj_create", ctypes.c_int, [vp, vp, ctypes.c_int, vp]),
    ("igab_tadj_forward", ctypes.c_int, [vp, vp, vp, vp]),
    ("igab_tadj_backward", ctypes.c_int, [vp, vp, vp]),
    ("igab_tadj_info", ctypes.c_int, [vp, vp]),
    ("igab_tadj_destroy", None, [vp]),
    ("igab_set_option", ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
    ("igab_graph_capture", ctypes.c_int, [vp, vp, vp, vp, ctypes.c_int, ctypes.c_int]),
    ("igab_graph_launch", ctypes.c_int, [vp]),
    ("igab_graph_destroy", ctypes.c_int, [vp]),
    ("igab_set_element_log_scale", ctypes.c_int, [vp, vp, ctypes.c_int]),
    ("igab_adjoint_forward", ctypes.c_int, [vp, vp, vp, vp, vp, ctypes.c_int]),
    ("igab_adjoint_backward", ctypes.c_int, [vp, vp, vp, ctypes.c_int, vp, vp, vp]),
    ("igab_get_option", ctypes.c_int, [vp, ctypes.c_int, c_int_p]),
    ("igab_tc_selftest", ctypes.c_int, [ctypes.c_int, vp]),
    ("igab_tc_peak", ctypes.c_int, [ctypes.c_int, ctypes.c_int, c_double_p]),
    ("igab_history_jacobian_device", ctypes.c_int, [vp, vp, vp, ctypes.c_int, ctypes.c_int]),
    ("igab_dirichlet_rows", ctypes.c_int, [vp, c_long_p, vp]),
    ("igab_ndensity", ctypes.c_int, [vp, c_int_p]),
    ("igab_intdensity", ctypes.c_int, [vp, vp, vp]),
    ("igab_intdensity_device", ctypes.c_int, [vp, vp, vp]),
    ("igab_spmv_device", ctypes.c_int, [vp, vp, ctypes.c_int, vp, vp]),
    ("igab_knot_insert", ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]),
    ("igab_knot_release", ctypes.c_int, [ctypes.c_int]),
    ("igab_write_solution", ctypes.c_int, [ctypes.c_char_p, vp, ctypes.c_long, ctypes.c_int, ctypes.c_int]),
    ("igab_read_solution", ctypes.c_int, [ctypes.c_char_p, vp, ctypes.c_long, ctypes.c_int, ctypes.c_int]),
    ("igab_solve_device", ctypes.c_int, [vp, vp, ctypes.c_int, vp, vp, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, ctypes.POINTER(IgabSolveInfo)]),
    ("igab_batch_create", ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]),
    ("igab_batch_destroy", ctypes.c_int, [vp]),
    ("igab_batch_sizes", ctypes.c_int, [vp, c_long_p, c_long_p, c_long_p, vp, vp]),
    ("igab_batch_instance", vp, [vp, ctypes.c_int]),
    ("igab_batch_refresh", ctypes.c_int, [vp]),
    ("igab_batch_set_stream", ctypes.c_int, [vp, vp]),
    ("igab_batch_set_schedule", ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("igab_batch_get_schedule", ctypes.c_int, [vp, c_int_p, c_int_p, c_int_p, c_int_p]),
    ("igab_batch_set_colour_order", ctypes.c_int, [vp, ctypes.c_int]),
    ("igab_batch_get_colour_order", ctypes.c_int, [vp, c_int_p]),
    ("igab_batch_residual_device", ctypes.c_int, [vp, vp, vp]),
    ("igab_batch_tangent_device", ctypes.c_int, [vp, vp, vp, ctypes.c_int]),
    ("igab_batch_sync", ctypes.c_int, [vp]),
    ("igab_batch_set_wait_limit", ctypes.c_int, [vp, ctypes.c_long, ctypes.c_int]),
    ("igab_batch_last_launch_count", ctypes.c_int, [vp, c_int_p]),
    ("igab_batch_graph_capture", ctypes.c_int, [vp, vp, vp, vp, ctypes.c_int]),
    ("igab_batch_graph_launch", ctypes.c_int, [vp]),
    ("igab_autotune", ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(IgabTuneResult)]),
    ("igab_batch_autotune", ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(IgabBatchTuneResult)]),
]

# entry points of include/snesiga_b200.h and include/iga_case.h
DROPIN_API = [
    ("snesiga_Residual", ctypes.c_int, [vp, vp, vp, vp]),
    ("snesiga_Tangent", ctypes.c_int, [vp, vp, vp, vp, vp]),
    ("snesiga_init", None, [vp, vp, vp, vp, vp, vp]),
    ("snesiga_b200_Residual", ctypes.c_int, [vp, vp, vp, vp]),
    ("snesiga_b200_Tangent", ctypes.c_int, [vp, vp, vp, vp, vp]),
    ("snesiga_gpu_init", ctypes.c_int, [vp, ctypes.c_int]),
    ("snesiga_gpu_free", ctypes.c_int, [vp]),
    ("snesiga_gpu_set_neumann", ctypes.c_int, [vp, vp]),
    ("snesiga_gpu_set_neumann_policy", ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
    ("snesiga_gpu_set_tangent_precision", ctypes.c_int, [vp, ctypes.c_int]),
    ("snesiga_gpu_context", vp, [vp]),
    ("snesiga_gpu_last_timings", ctypes.c_int, [vp, c_double_p]),
    ("snesiga_gpu_set_ksp", ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int]),
    ("snesiga_gpu_last_solve", ctypes.c_int, [vp, vp]),
    ("snesiga_b200_solve", None, [vp]),
    ("snes_solve", None, [vp]),
    ("iga_intdensity", None, [vp, vp]),
    ("snesiga_b200_intdensity", None, [vp, vp]),
    ("nurbs_knotinsert", None, [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]),
    ("write_solution", None, [ctypes.c_char_p, vp, vp, ctypes.c_int, ctypes.c_int]),
    ("read_solution", None, [ctypes.c_char_p, vp, vp, ctypes.c_int, ctypes.c_int]),
]

CASE_API = [
    ("iga_case_create", vp, [ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int]),
    ("iga_case_create_periodic", vp, [ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, vp]),
    ("iga_case_index_maps", ctypes.c_int, [vp, vp, vp, vp, vp, vp]),
    ("iga_case_destroy", None, [vp]),
    ("iga_case_ndof", ctypes.c_int, [vp]),
    ("iga_case_set_history", ctypes.c_int, [vp, ctypes.c_int, vp]),
    ("iga_case_get_history", ctypes.c_int, [vp, ctypes.c_int, vp]),
    ("iga_case_set_par_neumann", ctypes.c_int, [vp, vp, ctypes.c_int]),
    ("iga_case_set_par_dirichlet", ctypes.c_int, [vp, vp]),
    ("iga_case_set_par_mat", ctypes.c_int, [vp, vp]),
    ("iga_case_residual", ctypes.c_int, [vp, vp, vp]),
    ("iga_case_tangent", ctypes.c_int, [vp, vp]),
    ("iga_case_tangent_nnz", ctypes.c_long, [vp]),
    ("iga_case_tangent_csr", ctypes.c_int, [vp, vp, vp, vp]),
    ("iga_case_app", vp, [vp]),
    ("iga_case_iocomm", vp, [vp]),
    ("iga_case_snesassmbl", vp, [vp]),
    ("iga_case_solve", ctypes.c_int, [vp, vp]),
    ("iga_case_neumann", None, [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]),
]

_cache = {}


def bind(lib, api):
    for name, res, args in api:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def _load(path, api, mode=ctypes.RTLD_GLOBAL):
    if path in _cache:
        return _cache[path]
    if not os.path.exists(path):
        raise NativeLibraryMissing("%s is not built; run `python -m igap4standard_b200.build`" % path)
    lib = bind(ctypes.CDLL(path, mode=mode), api)
    _cache[path] = lib
    return lib


def lib_cuda():
    return _load(LIB_CUDA, IGAB_API)


def lib_dropin():
    lib_cuda()
    _load(LIB_SUBSET, [])
    return _load(LIB_DROPIN, DROPIN_API + CASE_API, mode=ctypes.RTLD_LOCAL)


def check(lib, where, rc):
    if rc != 0:
        msg = lib.igab_last_error()
        raise IgabError(where, rc, msg.decode() if msg else "")
