"""Python face of the plain C ABI (include/igab.h)."""
import ctypes
import numpy as np

from . import native
from .native import IgabMeshDesc, check, vp

PHYS = {"ge": 0, "getime": 1}
PREC = {"fp64": 0, "fp32": 1}
OPT_TANGENT_FP64_KERNEL = 1
OPT_TANGENT_FP32_KERNEL = 2
OPT_COLOUR_ORDER = 3


def _ptr(a):
    return a.ctypes.data_as(vp)


class TransientAdjoint:
    """The checkpointed adjoint pass of igab_tadj_* on one Assembly (see transient_adjoint)."""

    def __init__(self, A, opts, every, U_init_ptr, U_prev_ptr):
        self.A, self.lib = A, A.lib
        self.U_init_ptr, self.U_prev_ptr = U_init_ptr, U_prev_ptr
        h = ctypes.c_void_p()
        check(self.lib, "igab_tadj_create", self.lib.igab_tadj_create(A.h, ctypes.byref(opts), int(every),
                                                                       ctypes.byref(h)))
        self.h = h

    def forward(self, U_final_ptr, U_init_ptr=None):
        """The forward steps from U_init (device; the zero state when never given), U_N into U_final_ptr."""
        u0 = U_init_ptr or self.U_init_ptr
        if u0 is None:
            import torch
            self._zero = torch.zeros(self.A.ndof, dtype=torch.float64, device=torch.device("cuda", self.A.device))
            u0 = self._zero.data_ptr()
        check(self.lib, "igab_tadj_forward",
              self.lib.igab_tadj_forward(self.h, vp(u0), vp(self.U_prev_ptr) if self.U_prev_ptr else None,
                                         vp(U_final_ptr)))

    def backward(self, dJdU_ptr, grad_ptr):
        """dJ/dg (device, nel doubles) from dJ/dU_N (device)."""
        check(self.lib, "igab_tadj_backward", self.lib.igab_tadj_backward(self.h, vp(dJdU_ptr), vp(grad_ptr)))

    def info(self):
        i = native.IgabTadjInfo()
        check(self.lib, "igab_tadj_info", self.lib.igab_tadj_info(self.h, ctypes.byref(i)))
        return {f: getattr(i, f) for f, _ in native.IgabTadjInfo._fields_}

    def close(self):
        if self.h:
            self.lib.igab_tadj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Assembly:
    """One single-rank mesh on one GPU: residual and tangent assembly.

    Mirrors what snesiga_init + snesiga_Residual/snesiga_Tangent do for one
    rank (IGAP4STANDARD src/snesiga_init.c:12, src/snesiga_Residual.c:13,
    src/snesiga_Tangent.c:13), with plain arrays instead of PETSc objects."""

    def __init__(self, nelem, knots, par_mat, bc_type, par_dirichlet=None, par_periodic=None,
                 phys="ge", device=0, bc_periodic=(0, 0, 0)):
        self.lib = native.lib_cuda()
        d = IgabMeshDesc()
        d.phys = PHYS[phys]
        for i in range(3):
            d.nelem[i] = int(nelem[i])
        self._knots = np.ascontiguousarray(knots, dtype=np.float64)
        if self._knots.size != sum(int(n) + 5 for n in nelem):
            raise ValueError("knots must hold nelem[d]+5 values per direction")
        d.knots = self._knots.ctypes.data_as(native.c_double_p)
        for i in range(9):
            d.par_mat[i] = float(par_mat[i])
            d.par_dirichlet[i] = float(par_dirichlet[i]) if par_dirichlet is not None else 0.0
            d.par_periodic[i] = float(par_periodic[i]) if par_periodic is not None else 0.0
        for i in range(36):
            d.bc_type[i] = int(bc_type[i])
        for i in range(3):
            d.bc_periodic[i] = int(bc_periodic[i])
        h = vp()
        check(self.lib, "igab_create", self.lib.igab_create(ctypes.byref(d), int(device), ctypes.byref(h)))
        self.h = h
        nd, nz, ne = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
        check(self.lib, "igab_sizes", self.lib.igab_sizes(h, ctypes.byref(nd), ctypes.byref(nz), ctypes.byref(ne)))
        self.ndof, self.nnz, self.nelem_total = nd.value, nz.value, ne.value
        self.nelem = tuple(int(n) for n in nelem)
        self.phys = phys
        self.device = int(device)

    def close(self):
        if getattr(self, "h", None):
            self.lib.igab_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- pattern
    def pattern(self, with_cols=True):
        rowptr = np.empty(self.ndof + 1, dtype=np.int32)
        cols = np.empty(self.nnz, dtype=np.int32) if with_cols else None
        check(self.lib, "igab_csr_pattern",
              self.lib.igab_csr_pattern(self.h, _ptr(rowptr), _ptr(cols) if with_cols else None))
        return rowptr, cols

    def csr_offset(self, row, col):
        return self.lib.igab_csr_offset(self.h, int(row), int(col))

    # ---- parameters
    def set_par_mat(self, pm):
        a = np.ascontiguousarray(pm, dtype=np.float64)
        check(self.lib, "igab_set_par_mat", self.lib.igab_set_par_mat(self.h, _ptr(a)))

    def set_par_dirichlet(self, pd):
        a = np.ascontiguousarray(pd, dtype=np.float64)
        check(self.lib, "igab_set_par_dirichlet", self.lib.igab_set_par_dirichlet(self.h, _ptr(a)))

    def set_par_periodic(self, pp):
        a = np.ascontiguousarray(pp, dtype=np.float64)
        check(self.lib, "igab_set_par_periodic", self.lib.igab_set_par_periodic(self.h, _ptr(a)))

    def neumann_points(self):
        n = ctypes.c_long()
        check(self.lib, "igab_neumann_points", self.lib.igab_neumann_points(self.h, ctypes.byref(n), None, None))
        xyz = np.empty((n.value, 3))
        meta = np.empty((n.value, 3), dtype=np.int32)
        if n.value:
            check(self.lib, "igab_neumann_points",
                  self.lib.igab_neumann_points(self.h, ctypes.byref(n), _ptr(xyz), _ptr(meta)))
        return xyz, meta

    def set_neumann_values(self, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        check(self.lib, "igab_set_neumann_values", self.lib.igab_set_neumann_values(self.h, _ptr(a)))

    def set_history(self, level, U):
        a = np.ascontiguousarray(U, dtype=np.float64)
        check(self.lib, "igab_set_history", self.lib.igab_set_history(self.h, int(level), _ptr(a), 0))

    def set_history_device(self, level, U_ptr):
        """History level (1 = t_n, 2 = t_{n-1}) from a device pointer (copied in place)."""
        check(self.lib, "igab_set_history", self.lib.igab_set_history(self.h, int(level), vp(U_ptr), 1))

    def set_option(self, option, value):
        check(self.lib, "igab_set_option", self.lib.igab_set_option(self.h, int(option), int(value)))

    def get_option(self, option):
        v = ctypes.c_int()
        check(self.lib, "igab_get_option", self.lib.igab_get_option(self.h, int(option), ctypes.byref(v)))
        return v.value

    def set_tile(self, residual_tile=0, tangent_tile=0):
        check(self.lib, "igab_set_tile", self.lib.igab_set_tile(self.h, residual_tile, tangent_tile))

    def autotune(self, U_ptr=None, what=7, reps=3, cache=None):
        """Time every candidate schedule (igab_autotune) and keep the fastest; with a
        cache file, a schedule stored for this GPU and mesh is applied without timing.
        what: bit 0 residual tile, bit 1 / 2 FP64 / FP32 tangent kernel, bit 3 colour order.
        Returns dict(residual_tile, tangent_fp64_kernel, tangent_fp32_kernel, *_ms, colour_order, cached)."""
        from . import tuning
        key = tuning.mesh_key(self.device, self.nelem, self.phys, what) if cache else None
        hit = tuning.load(cache).get(key) if cache else None
        if hit:
            self.set_tile(hit["residual_tile"], 0)
            self.set_option(OPT_TANGENT_FP64_KERNEL, hit["tangent_fp64_kernel"])
            self.set_option(OPT_TANGENT_FP32_KERNEL, hit["tangent_fp32_kernel"])
            self.set_option(OPT_COLOUR_ORDER, hit.get("colour_order", 0))
            return dict(hit, cached=True)
        r = native.IgabTuneResult()
        check(self.lib, "igab_autotune",
              self.lib.igab_autotune(self.h, vp(U_ptr or 0), int(what), int(reps), ctypes.byref(r)))
        out = {f: getattr(r, f) for f, _ in native.IgabTuneResult._fields_}
        if cache:
            tuning.store(cache, key, out)
        return dict(out, cached=False)

    # ---- host-pointer assembly
    def residual(self, U, out=None):
        U = np.ascontiguousarray(U, dtype=np.float64)
        R = out if out is not None else np.empty(self.ndof)
        check(self.lib, "igab_residual", self.lib.igab_residual(self.h, _ptr(U), _ptr(R)))
        return R

    def tangent(self, U, prec="fp64", out=None):
        U = np.ascontiguousarray(U, dtype=np.float64)
        dt = np.float64 if prec == "fp64" else np.float32
        v = out if out is not None else np.empty(self.nnz, dtype=dt)
        check(self.lib, "igab_tangent", self.lib.igab_tangent(self.h, _ptr(U), _ptr(v), PREC[prec]))
        return v

    # ---- device-pointer assembly (integers from e.g. torch.Tensor.data_ptr())
    def residual_device(self, U_ptr, R_ptr):
        check(self.lib, "igab_residual_device", self.lib.igab_residual_device(self.h, vp(U_ptr), vp(R_ptr)))

    def tangent_device(self, U_ptr, vals_ptr, prec="fp64"):
        check(self.lib, "igab_tangent_device",
              self.lib.igab_tangent_device(self.h, vp(U_ptr), vp(vals_ptr), PREC[prec]))

    def dirichlet_rows(self):
        """Ascending dofs of the Dirichlet residual rows."""
        n = ctypes.c_long()
        check(self.lib, "igab_dirichlet_rows", self.lib.igab_dirichlet_rows(self.h, ctypes.byref(n), None))
        rows = np.empty(n.value, dtype=np.int32)
        if n.value:
            check(self.lib, "igab_dirichlet_rows", self.lib.igab_dirichlet_rows(self.h, ctypes.byref(n), _ptr(rows)))
        return rows

    def spmv_device(self, vals_ptr, x_ptr, y_ptr, prec="fp64"):
        """y = K x on the tangent's pattern (device pointers, FP64 vectors)."""
        check(self.lib, "igab_spmv_device",
              self.lib.igab_spmv_device(self.h, vp(vals_ptr), PREC[prec], vp(x_ptr), vp(y_ptr)))

    def solve_device(self, vals_ptr, b_ptr, x_ptr, prec="fp64", rtol=1e-5, atol=0.0, maxit=2000):
        """x = K^-1 b on the device: Jacobi-preconditioned BiCGStab, x0 = 0, stop at
        ||b - K x|| <= max(rtol ||b||, atol).  Returns (iterations, converged, residual norm)."""
        info = native.IgabSolveInfo()
        check(self.lib, "igab_solve_device",
              self.lib.igab_solve_device(self.h, vp(vals_ptr), PREC[prec], vp(b_ptr), vp(x_ptr), float(rtol),
                                         float(atol), int(maxit), ctypes.byref(info)))
        return info.iterations, bool(info.converged), info.residual_norm

    def affine_start(self, knots, F0):
        """A Newton start for static problems: the affine field u = F0 X at the control points'
        Greville abscissae (mesh.affine_field), with every Dirichlet row set to its value
        (R = U - g there, so g = U - R).  From U = 0 the reference's first step projects onto
        the Dirichlet values and leaves a one-element boundary layer whose strain grows like
        1/h; this start has none."""
        from .mesh import affine_field
        U = affine_field(self.nelem, knots, F0)
        R = self.residual(U)
        rows = self.dirichlet_rows()
        U[rows] -= R[rows]
        return U

    def solve_mg_device(self, vals_ptr, b_ptr, x_ptr, prec="fp64", rtol=1e-5, atol=0.0, maxit=1000, method="gmres"):
        """x = K^-1 b by multigrid-preconditioned GMRES or CG on the device (igab_solve_mg_device).
        Returns (iterations, converged, residual norm, multigrid levels)."""
        info = native.IgabSolveInfo()
        check(self.lib, "igab_solve_mg_device",
              self.lib.igab_solve_mg_device(self.h, {"cg": 1, "gmres": 2}[method], vp(vals_ptr), PREC[prec],
                                            vp(b_ptr), vp(x_ptr), float(rtol), float(atol), int(maxit),
                                            ctypes.byref(info)))
        lev = ctypes.c_int()
        check(self.lib, "igab_solve_mg_levels", self.lib.igab_solve_mg_levels(self.h, ctypes.byref(lev)))
        return info.iterations, bool(info.converged), info.residual_norm, lev.value

    def newton_solve_device(self, U_ptr, prec="fp64", ksp_rtol=1e-5, ksp_maxit=100000, abstol=1e-10,
                            max_subiter=10000, verbose=False, history_cap=64, ksp="mg", fp64_polish=False,
                            use_graph=True):
        """Device Newton solve (igab_newton_solve) from the state at U_ptr (device, FP64,
        overwritten with the result).  Returns a dict of the solve info plus the ||F|| and
        Krylov-iteration history of each subiteration."""
        o = native.IgabNewtonOpts()
        self.lib.igab_newton_defaults(ctypes.byref(o))
        o.prec = PREC[prec]
        o.ksp_rtol = float(ksp_rtol)
        o.ksp_maxit = int(ksp_maxit)
        o.abstol = float(abstol)
        o.max_subiter = int(max_subiter)
        o.ksp = {"mg": 2, "mg-cg": 1, "bicgstab": 0}[ksp]
        o.verbose = 1 if verbose else 0
        o.fp64_polish = 1 if fp64_polish else 0
        o.use_graph = 1 if use_graph else 0
        info = native.IgabNewtonInfo()
        fh = np.zeros(history_cap)
        kh = np.zeros(history_cap, dtype=np.int32)
        check(self.lib, "igab_newton_solve",
              self.lib.igab_newton_solve(self.h, vp(U_ptr), ctypes.byref(o), ctypes.byref(info), _ptr(fh), _ptr(kh),
                                         int(history_cap)))
        out = {f: getattr(info, f) for f, _ in native.IgabNewtonInfo._fields_}
        m = min(out["iterations"] + 1, history_cap)
        out["fnorms"] = fh[:m].tolist()
        out["krylov"] = kh[:m].tolist()
        return out

    def transient_run(self, U_ptr, nsteps, prec="fp32", U_prev_ptr=None, dt=0.0, amplitude=0.01, face=1, order=0,
                      dof=0, ksp_rtol=1e-5, ksp_maxit=100000, abstol=1e-10, use_graph=True, keep_steps=False):
        """Time stepping of the transient physics on the device (igab_transient_run): nsteps
        steps from U at t_0 (device, FP64, at U_ptr; overwritten with U at t_nsteps) and U at
        t_-1 (U_prev_ptr; None = zero).  Returns (totals, per-step info dicts, the states
        after every step as an (nsteps, ndof) array when keep_steps, else None)."""
        o = self._transient_opts(nsteps, prec, dt, amplitude, face, order, dof, ksp_rtol, ksp_maxit, abstol,
                                 use_graph)
        steps = (native.IgabNewtonInfo * max(nsteps, 1))()
        info = native.IgabTransientInfo()
        hist = np.empty((nsteps, self.ndof)) if keep_steps else None
        check(self.lib, "igab_transient_run",
              self.lib.igab_transient_run(self.h, ctypes.byref(o), vp(U_ptr), vp(U_prev_ptr) if U_prev_ptr else None,
                                          _ptr(hist) if keep_steps else None, steps, ctypes.byref(info)))
        per_step = [{f: getattr(steps[i], f) for f, _ in native.IgabNewtonInfo._fields_} for i in range(nsteps)]
        return {f: getattr(info, f) for f, _ in native.IgabTransientInfo._fields_}, per_step, hist

    def _transient_opts(self, nsteps, prec, dt, amplitude, face, order, dof, ksp_rtol, ksp_maxit, abstol, use_graph):
        o = native.IgabTransientOpts()
        self.lib.igab_transient_defaults(ctypes.byref(o))
        o.nsteps = int(nsteps)
        o.dt = float(dt)
        o.amplitude = float(amplitude)
        o.face, o.order, o.dof = int(face), int(order), int(dof)
        o.newton.prec = PREC[prec]
        o.newton.ksp_rtol = float(ksp_rtol)
        o.newton.ksp_maxit = int(ksp_maxit)
        o.newton.abstol = float(abstol)
        o.newton.use_graph = 1 if use_graph else 0
        return o

    def transient_adjoint(self, nsteps, every=10, U_init_ptr=None, U_prev_ptr=None, dt=0.0, amplitude=0.01, face=1,
                          order=0, dof=0, ksp_rtol=1e-12, ksp_maxit=100000, abstol=1e-13, use_graph=True):
        """A checkpointed discrete adjoint of nsteps time steps (igab_tadj_*), FP64 tangents.
        Returns a TransientAdjoint: forward(U_final_ptr), then backward(dJdU_ptr, grad_ptr)."""
        o = self._transient_opts(nsteps, "fp64", dt, amplitude, face, order, dof, ksp_rtol, ksp_maxit, abstol,
                                 use_graph)
        return TransientAdjoint(self, o, every, U_init_ptr, U_prev_ptr)

    def ndensity(self):
        n = ctypes.c_int()
        check(self.lib, "igab_ndensity", self.lib.igab_ndensity(self.h, ctypes.byref(n)))
        return n.value

    def intdensity(self, U):
        """Integrated densities (src/iga_intdensity.c): volume integral of the point
        density at U (phys/ge) or at the history levels (phys/getime) minus the
        Neumann boundary integrals, as in the reference's HH_ array."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        HH = np.empty(self.ndensity())
        check(self.lib, "igab_intdensity", self.lib.igab_intdensity(self.h, _ptr(U), _ptr(HH)))
        return HH

    def intdensity_device(self, U_ptr, HH_ptr):
        check(self.lib, "igab_intdensity_device", self.lib.igab_intdensity_device(self.h, vp(U_ptr), vp(HH_ptr)))

    def history_jacobian_device(self, U_ptr, vals_ptr, level, prec="fp64"):
        """CSR values of dR/dU_hist[level] (transient physics; Dirichlet rows zero)."""
        check(self.lib, "igab_history_jacobian_device",
              self.lib.igab_history_jacobian_device(self.h, vp(U_ptr), vp(vals_ptr), PREC[prec], int(level)))

    def graph_capture(self, U_ptr, R_ptr=None, vals_ptr=None, prec="fp64"):
        what = (1 if R_ptr is not None else 0) | (2 if vals_ptr is not None else 0)
        check(self.lib, "igab_graph_capture",
              self.lib.igab_graph_capture(self.h, vp(U_ptr), vp(R_ptr or 0), vp(vals_ptr or 0), PREC[prec], what))

    def graph_launch(self):
        check(self.lib, "igab_graph_launch", self.lib.igab_graph_launch(self.h))

    def graph_destroy(self):
        check(self.lib, "igab_graph_destroy", self.lib.igab_graph_destroy(self.h))

    # ---- adjoint of the element-scaled problem (s_e = exp(g_e))
    def set_element_log_scale(self, g):
        """g: [nelem_total] log-scales in the reference's element order, or None for s = 1."""
        if g is None:
            check(self.lib, "igab_set_element_log_scale", self.lib.igab_set_element_log_scale(self.h, None, 0))
            return
        a = np.ascontiguousarray(g, dtype=np.float64)
        if a.size != self.nelem_total:
            raise ValueError("g needs one value per element")
        check(self.lib, "igab_set_element_log_scale", self.lib.igab_set_element_log_scale(self.h, _ptr(a), 0))

    def adjoint_forward_device(self, g_ptr, U_ptr, R_ptr=None, vals_ptr=None, prec="fp64"):
        check(self.lib, "igab_adjoint_forward",
              self.lib.igab_adjoint_forward(self.h, vp(g_ptr or 0), vp(U_ptr), vp(R_ptr or 0), vp(vals_ptr or 0),
                                            PREC[prec]))

    def adjoint_backward_device(self, U_ptr, vals_ptr, lam_ptr, KTlam_ptr=None, grad_ptr=None, prec="fp64"):
        check(self.lib, "igab_adjoint_backward",
              self.lib.igab_adjoint_backward(self.h, vp(U_ptr or 0), vp(vals_ptr or 0), PREC[prec], vp(lam_ptr),
                                             vp(KTlam_ptr or 0), vp(grad_ptr or 0)))

    def dRdg(self, U, lam):
        """Host convenience: grad[e] = lam . dR/dg_e at U (Dirichlet rows of lam ignored)."""
        import torch
        dev = torch.device("cuda", self.device)
        Ud = torch.as_tensor(np.ascontiguousarray(U, dtype=np.float64)).to(dev)
        Ld = torch.as_tensor(np.ascontiguousarray(lam, dtype=np.float64)).to(dev)
        G = torch.empty(self.nelem_total, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        self.adjoint_backward_device(Ud.data_ptr(), None, Ld.data_ptr(), None, G.data_ptr())
        self.sync()
        return G.cpu().numpy()

    def tangent_transpose_apply(self, vals, x, prec="fp64"):
        """Host convenience: K^T x for CSR values vals of this mesh's pattern."""
        import torch
        dev = torch.device("cuda", self.device)
        dt = np.float64 if prec == "fp64" else np.float32
        Vd = torch.as_tensor(np.ascontiguousarray(vals, dtype=dt)).to(dev)
        Xd = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64)).to(dev)
        Y = torch.empty(self.ndof, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        self.adjoint_backward_device(None, Vd.data_ptr(), Xd.data_ptr(), Y.data_ptr(), None, prec)
        self.sync()
        return Y.cpu().numpy()

    def set_stream(self, stream_ptr):
        check(self.lib, "igab_set_stream", self.lib.igab_set_stream(self.h, vp(stream_ptr)))

    def sync(self):
        check(self.lib, "igab_sync", self.lib.igab_sync(self.h))

    def last_launch_count(self):
        n = ctypes.c_int()
        check(self.lib, "igab_last_launch_count", self.lib.igab_last_launch_count(self.h, ctypes.byref(n)))
        return n.value

    # ---- measurement
    def set_profiling(self, on=True):
        check(self.lib, "igab_set_profiling", self.lib.igab_set_profiling(self.h, 1 if on else 0))

    def last_kernel_ms(self):
        """[res volume, res boundary, tan volume, tan Dirichlet] ms and the two volume launch counts."""
        ms = (ctypes.c_double * 6)()
        check(self.lib, "igab_last_kernel_ms", self.lib.igab_last_kernel_ms(self.h, ms))
        return list(ms)


def tc_peak_tflops(n_cols=256, device=0):
    """Measured dense TF32 tcgen05 throughput for M 128 x N n_cols MMAs (igab_tc_peak)."""
    lib = native.lib_cuda()
    t = ctypes.c_double()
    check(lib, "igab_tc_peak", lib.igab_tc_peak(int(device), int(n_cols), ctypes.byref(t)))
    return t.value


def dmma_peak_tflops(device=0):
    """FP64 tensor-pipe (mma.sync m8n8k4 f64) throughput of the device, TFLOP/s."""
    lib = native.lib_cuda()
    t = ctypes.c_double()
    check(lib, "igab_dmma_peak", lib.igab_dmma_peak(int(device), ctypes.byref(t)))
    return t.value


def fma_peak_tflops(prec="fp64", device=0):
    lib = native.lib_cuda()
    t = ctypes.c_double()
    check(lib, "igab_fma_peak", lib.igab_fma_peak(int(device), PREC[prec], ctypes.byref(t)))
    return t.value
