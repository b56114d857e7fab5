#!/usr/bin/env python3
"""Newton-step assembly benchmark: IGAP4STANDARD phys/ge at 64^3 quadratic elements.

One step = one residual assembly (volume + Neumann + Dirichlet rows) followed by
one tangent assembly (volume + Dirichlet row/column elimination) into the CSR
arrays of the reference's AIJ pattern: the work snesiga_Residual +
snesiga_Tangent do per Newton iteration (src/snesiga_Residual.c:13,
src/snesiga_Tangent.c:13).  Synthetic, seeded input: 64^3 elements on the unit
cube with interior knots perturbed by +-0.1h (seed 1), (lambda, mu, l) =
(1, 1, 0.1) mapped onto par_mat, x=0 clamped / x=1 u_x = 0.01 X, state
uniform in +-1e-3 (seed 0).

  value     FP64 path, inputs resident in HBM, ms per assembly (device events)
  mixed     FP32-built tangent + FP64 residual, same timing
  e2e       FP64 path through the host-pointer C ABI (U in, R and CSR values out)
  roofline  tangent volume kernel against the measured FP64 FMA peak
  cpu_baseline  the reference's own assembly (oracle/_ref) on the host cores

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "Newton-step assembly ms & adjoint grads/s at 64^3, mixed vs FP64, 1xB200"

# Algorithmic flops per element (4^3 Gauss points):
#  tangent  64 * 2 * (30*81*10 + 81*81*10) = B^T D B with the dof-block-sparse B
#  residual 64 * (2 * (27*30 + 27*30) + 270 + 758): interpolation, test contraction, basis
#           products and the point integrand, whose 758 operations per call are counted in
#           the reference's phys/ge/residual.c by oracle/count_integrand_flops.py
GE_RESIDUAL_INTEGRAND_FLOPS = 758
TAN_ALG_FLOPS = 64 * 2 * (30 * 81 * 10 + 81 * 81 * 10)
RES_ALG_FLOPS = 64 * (2 * (27 * 30 + 27 * 30) + 270 + GE_RESIDUAL_INTEGRAND_FLOPS)
# flops the tangent kernel executes per element on the tensor path: 66 upper 8x8 tiles
# x 12 variables per point, plus 10 upper 8x8 tiles of the geometric block x 6 U / V rows per point
TAN_EXEC_FLOPS = 64 * 2 * (66 * 64 * 12 + 10 * 64 * 6)
# DRAM bytes per element of the FP64 tangent kernel (ncu, 32^3 colour launch: 243.12 MB / 4,096)
TAN64_DRAM_BYTES_PER_ELEMENT = 243.12e6 / 4096


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64, help="elements per side")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the schedule autotuner")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-density", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-instance batched assembly")
    ap.add_argument("--batch-instances", type=int, default=512)
    ap.add_argument("--transient", type=int, default=200, metavar="STEPS",
                    help="time STEPS steps of the transient workload (phys/getime, 32^3, dt 1e-3); 0 skips")
    ap.add_argument("--transient-adjoint", type=int, default=50, metavar="STEPS",
                    help="time one checkpointed transient adjoint gradient over STEPS steps (32^3, every 10); "
                         "0 skips")
    ap.add_argument("--no-newton", action="store_true", help="skip the FP64 / mixed Newton solves at n^3")
    ap.add_argument("--newton-ksp-rtol", type=float, default=1e-5,
                    help="Krylov tolerance of the Newton solves (PETSc's default KSP rtol)")
    ap.add_argument("--no-adjoint-static", action="store_true",
                    help="skip the end-to-end static adjoint gradient at 32^3")
    return ap.parse_args()


def workload(n):
    from igap4standard_b200 import mesh
    nelem = (n, n, n)
    kn = mesh.knots_for(nelem, perturb=0.1, seed=1)
    pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
    bc, pd = mesh.bc_config0()
    return nelem, kn, pm, bc, pd


def config_dict(n, ndof, nnz):
    return {"workload": "phys/ge Newton-step assembly (residual+BCs, tangent+BCs into AIJ) %d^3 elements" % n,
            "nelem": [n, n, n], "dofs": ndof, "nnz": nnz, "gauss_points": "4x4x4",
            "knots": "open, interior perturbed +-0.1h (seed 1)", "material": "lambda=mu=1, l=0.1 mapped to par_mat",
            "state": "uniform +-1e-3 (seed 0)",
            "l2": "inputs larger than L2: every step writes the %.2f GB CSR value array" % (nnz * 8 / 1e9),
            "parallelism": "replicas (one mesh per GPU)"}


# ------------------------------------------------------------------ CPU side

def _ref_sample_worker(args):
    """One process: the reference's residual (then iga_intdensity) on an x-y slab of the
    n^3 workload, and its tangent on a slab of the 8x8x16 sub-block, each on its own
    single-rank mesh with the workload's knot perturbation, material and BCs."""
    res_shape, tan_shape, seed = args
    sys.path.insert(0, REPO)
    from oracle import ref
    from igap4standard_b200 import mesh
    pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
    bc, pd = mesh.bc_config0()
    out = []
    for shape, what in ((res_shape, "res"), (tan_shape, "tan")):
        C = ref.case("ge", shape, mesh.knots_for(shape, perturb=0.1, seed=1), pm, bc, np.zeros(9), pd, np.zeros(39))
        U = np.random.default_rng(seed).uniform(-1e-3, 1e-3, C.ndof)
        t0 = time.perf_counter()
        if what == "res":
            C.residual(U)
            t1 = time.perf_counter()
            C.intdensity(13)   # iga_intdensity on U_hist level 0 (left there by the residual callback)
            t2 = time.perf_counter()
            out += [t1 - t0, t2 - t1]
        else:
            C.tangent(U)
            out.append(time.perf_counter() - t0)
        C.close()
    return out


class RefPool:
    """Host-core pool running the reference's CPU assembly (spawned processes, one mesh each).

    A sample covers the n^3 workload's element count for the residual: P processes, each on
    an n x n x ceil(n/P) slab, run at once; and 1,024 elements for the tangent: the 8x8x16
    sub-block as P slabs of 8 x 8 x ceil(16/P).  Times are per element, from each process's
    own clock around the reference callback."""

    def __init__(self, procs):
        import multiprocessing as mp
        self.procs = procs
        self.pool = mp.get_context("spawn").Pool(procs)

    def shapes(self, n):
        P = self.procs
        return (n, n, max(1, -(-n // P))), (8, 8, max(1, -(-16 // P)))

    def sample(self, n):
        rs, ts = self.shapes(n)
        t0 = time.perf_counter()
        res = self.pool.map(_ref_sample_worker, [(rs, ts, i) for i in range(self.procs)])
        wall = time.perf_counter() - t0
        ne_r, ne_t = rs[0] * rs[1] * rs[2], ts[0] * ts[1] * ts[2]
        tr = float(np.mean([r[0] for r in res])) / ne_r
        self.td = float(np.mean([r[1] for r in res])) / ne_r   # intdensity per element
        tt = float(np.mean([r[2] for r in res])) / ne_t
        self.res_elements = ne_r * self.procs
        self.tan_elements = ne_t * self.procs
        return tr, tt, wall

    def describe(self, n):
        rs, ts = self.shapes(n)
        return ("%d processes at once (throughput mode, no MPI), reference code: residual on %d x %d x %d slabs "
                "(%d elements per sample, the %d^3 workload's count), tangent on %d x %d x %d slabs of the 8x8x16 "
                "sub-block (%d elements per sample, time per element extrapolated to %d^3)"
                % (self.procs, rs[0], rs[1], rs[2], rs[0] * rs[1] * rs[2] * self.procs, n, ts[0], ts[1], ts[2],
                   ts[0] * ts[1] * ts[2] * self.procs, n))

    def close(self):
        self.pool.close()
        self.pool.join()


def cpu_procs():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args):
    """--impl reference: the reference's own assembly on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    try:
        from oracle import ref
        if not ref.available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_iga.so not built here"}))
            return 0
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": "oracle import failed: %s" % e}))
        return 0
    from igap4standard_b200 import mesh
    n = args.n
    nel = n ** 3
    P = cpu_procs()
    pool = RefPool(P)
    for _ in range(max(args.warmup, 0)):
        pool.sample(n)
    per = []
    walls = []
    for _ in range(args.steps):
        tr, tt, wall = pool.sample(n)
        per.append((tr, tt))
        walls.append(wall)
    pool.close()
    tr = float(np.mean([p[0] for p in per]))
    tt = float(np.mean([p[1] for p in per]))
    ms = (tr + tt) * nel / P * 1e3
    ndof, nnz = mesh.n_dof((n, n, n)), mesh.nnz_of((n, n, n))
    sample = pool.describe(n) + "; value = (residual + tangent per element) x %d^3 / %d processes" % (n, P)
    line = {"impl": "reference", "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(n, ndof, nnz),
            "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": P, "kind": "reference", "sample": sample,
                             "residual_us_per_element": tr * 1e6, "tangent_ms_per_element": tt * 1e3,
                             "residual": "measured on the full element count", "tangent": "extrapolated"},
            "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "sample_wall_s": float(np.mean(walls))}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ GPU side

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx.append(float(p[2]))
                except ValueError:
                    continue
                for k, nm in enumerate(names[1:], start=5):
                    if p[k].lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def bench_batch(args, dev, device, barrier):
    """The 512-instance static workload (n^3 elements, n uniform 6..24, own material per
    instance): one Newton iteration's assembly (FP64 residual + FP32 tangent) through the
    persistent batched launch with the autotuned schedule, and the same work as one
    single-mesh assembly per instance for comparison."""
    import ctypes
    import torch
    from igap4standard_b200 import Batch, mesh
    from igap4standard_b200.native import vp, check
    inst = mesh.batch_config3(args.batch_instances, seed=3)
    t0 = time.perf_counter()
    B = Batch(inst, device=device)
    setup_s = time.perf_counter() - t0
    st = torch.cuda.Stream(device=dev)
    B.set_stream(st.cuda_stream)
    g = torch.Generator(device="cpu").manual_seed(0)
    U = (torch.rand(B.ndof, dtype=torch.float64, generator=g) * 2e-3 - 1e-3).to(dev)
    R = torch.empty(B.ndof, dtype=torch.float64, device=dev)
    V = torch.empty(B.nnz, dtype=torch.float32, device=dev)
    tune = B.autotune(U.data_ptr(), what=1 | 4 | 8, reps=1)
    tune.pop("cached", None)

    def step():
        B.residual_device(U.data_ptr(), R.data_ptr())
        B.tangent_device(U.data_ptr(), V.data_ptr(), "fp32")

    step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    K = 2
    e0.record(st)
    for _ in range(K):
        step()
    e1.record(st)
    barrier()
    B.sync()
    ms = e0.elapsed_time(e1) / K
    # the same assembly as one single-mesh call pair per instance (8 colour launches each)
    lib = B.lib
    hs = [B.instance_handle(i) for i in range(B.n)]
    offs = [(int(B.dof_offsets[i]) * 8, int(B.nnz_offsets[i]) * 4) for i in range(B.n)]

    def loop_step():
        for h, (od, on) in zip(hs, offs):
            check(lib, "igab_residual_device", lib.igab_residual_device(h, vp(U.data_ptr() + od), vp(R.data_ptr() + od)))
            check(lib, "igab_tangent_device",
                  lib.igab_tangent_device(h, vp(U.data_ptr() + od), vp(V.data_ptr() + on), 1))

    loop_step()
    barrier()
    e0.record(st)
    loop_step()
    e1.record(st)
    barrier()
    loop_ms = e0.elapsed_time(e1)
    out = {"instances": B.n, "elements": B.nelem_total, "dofs": B.ndof, "nnz": B.nnz,
           "ms_per_step": round(ms, 3), "elements_per_s": round(B.nelem_total / (ms * 1e-3), 1),
           "per_instance_launches_ms": round(loop_ms, 3), "speedup_vs_per_instance": round(loop_ms / ms, 3),
           "dtype": "f64 residual, f32 tangent", "schedule": tune, "setup_s": round(setup_s, 2),
           "workload": "config 3: n^3 elements, n uniform 6..24 (seed 3), lambda, mu lognormal(0,0.25), "
                       "l uniform [0.05,0.2], BCs of config 0; one residual + one FP32 tangent per step"}
    B.close()
    del V
    torch.cuda.empty_cache()
    return out


def bench_transient(args, device):
    """The transient workload: phys/getime on 32^3 elements, rho = 1, c = 1, dt = 1e-3,
    traction 0.01 sin(2 pi t) on x = 1 (x direction), u = 0 / du/dn = 0 on x = 0; each
    Newton iteration's assembly replayed from one CUDA graph, FP32 tangent, FP64 residual,
    Jacobi-BiCGStab on the library's K x kernel for the linear solves."""
    import torch
    from igap4standard_b200 import Assembly, mesh, transient
    n = 32
    nelem = (n, n, n)
    pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
    pm[5], pm[6], pm[7] = 1.0, 1.0, 1e-3
    bc, pd = mesh.bc_transient()
    A = Assembly(nelem, mesh.knots_for(nelem), pm, bc, pd, phys="getime", device=device)
    t0 = time.perf_counter()
    _, res, tot = transient.run(A, args.transient, pm[7], prec="fp32", use_graph=True, rtol_lin=1e-5,
                                keep_steps=False)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    its = [r.iterations for r in res]
    out = {"steps": args.transient, "wall_s": round(wall, 3), "ms_per_step": round(wall * 1e3 / args.transient, 3),
           "driver_ms": round(tot["ms_total"], 1),
           "newton_iterations_total": int(sum(its)), "newton_iterations_max": int(max(its)),
           "tangent_evaluations": int(tot["n_tangent"]), "residual_evaluations": int(tot["n_residual"]),
           "krylov_iterations_total": int(tot["krylov_iterations"]), "converged_all": all(r.converged for r in res),
           "final_fnorms_max": max(r.fnorms[-1] for r in res), "max_abs_u": float(np.abs(tot["U_final"]).max()),
           "launches": int(tot["launches"]),
           "timing": "host wall clock of the whole time loop in igab_transient_run (assembly graph replays, "
                     "line search residuals, BiCGStab solves, C host control)"}
    A.close()
    return out


def bench_transient_adjoint(args, device):
    """dJ/dg (32,768 element log-scales g ~ N(0, 0.3^2), seed 5) of J = 1/2 sum_{x=1}|U_N - U*|^2
    after STEPS steps of the transient workload, state checkpoints every 10 steps: forward
    solve, then the backward sweep with segment recomputation (FP64 tangent and history
    Jacobians, Jacobi-BiCGStab on the library's K x kernel)."""
    import torch
    from igap4standard_b200 import Assembly, mesh, transient
    n = 32
    nelem = (n, n, n)
    pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
    pm[5], pm[6], pm[7] = 1.0, 1.0, 1e-3
    bc, pd = mesh.bc_transient()
    A = Assembly(nelem, mesh.knots_for(nelem), pm, bc, pd, phys="getime", device=device)
    nb = n + 2
    mask = np.zeros((nb, nb, nb, 3))
    mask[-1] = 1.0
    mask = mask.reshape(-1)
    Ustar = np.random.default_rng(21).uniform(-1e-9, 1e-9, A.ndof)
    g = np.random.default_rng(5).normal(0.0, 0.3, A.nelem_total)
    t0 = time.perf_counter()
    out = transient.adjoint(A, args.transient_adjoint, pm[7], g, lambda U: mask * (U - Ustar), every=10,
                            rtol_lin=1e-10, objective=lambda U: 0.5 * float(np.sum(mask * (U - Ustar) ** 2)))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    res = {"steps": args.transient_adjoint, "checkpoint_every": 10, "parameters": A.nelem_total,
           "wall_s": round(wall, 3), "grads_per_s": round(1.0 / wall, 4),
           "recomputed_steps": out["recomputed_steps"], "checkpoints": len(out["checkpoints"]),
           "grad_norm": float(np.linalg.norm(out["grad"])), "J": out["J"],
           "forward_ms": round(out["info"]["ms_forward"], 1), "backward_ms": round(out["info"]["ms_backward"], 1),
           "adjoint_krylov_iterations": int(out["info"]["krylov_iterations_backward"]),
           "timing": "host wall clock: forward solve + backward sweep with segment recomputation (igab_tadj_*)"}
    A.close()
    return res


def bench_newton_config1(args, device):
    """The config-1 problem solved: FP64 and FP32-tangent Newton from the affine start to
    ||F||_2 < 1e-10 at n^3 with the reference application's solver loop (src/snes_solve.c:10-36,
    SNES settings of src/snes_init.c:8-47) run on the device by igab_newton_solve: every
    residual, tangent and multigrid-preconditioned GMRES solve (PETSc's default KSP rtol 1e-5) on the GPU."""
    import torch
    from igap4standard_b200 import Assembly
    n = args.n
    nelem, kn, pm, bc, pd = workload(n)
    A = Assembly(nelem, kn, pm, bc, pd, device=device)
    out, sol = {}, {}
    U0 = A.affine_start(kn, pd)
    for key, prec, polish in (("fp64", "fp64", False), ("fp32", "fp32", False), ("fp32_polish", "fp32", True)):
        U = torch.as_tensor(U0).to(torch.device("cuda", device))
        torch.cuda.synchronize()
        info = A.newton_solve_device(U.data_ptr(), prec, ksp_rtol=args.newton_ksp_rtol, fp64_polish=polish)
        sol[key] = U
        its = max(info["iterations"], 1)
        out[key] = {"newton_iterations": info["iterations"], "converged": bool(info["converged"]),
                     "reason": info["reason"], "final_fnorm": info["fnorm"], "fnorms": info["fnorms"],
                     "krylov_iterations": info["krylov_iterations"], "krylov_per_newton": info["krylov"],
                     "residual_evaluations": info["n_residual"], "tangent_evaluations": info["n_tangent"],
                     "fp64_tangents": info["n_tangent_fp64"],
                     "wall_s": round(info["ms_total"] / 1e3, 3),
                     "ms_per_newton_step": round(info["ms_total"] / its, 3),
                     "assembly_ms_per_newton_step": round((info["ms_residual"] + info["ms_tangent"]) / its, 3),
                     "krylov_ms_per_newton_step": round(info["ms_krylov"] / its, 3),
                     "launches": info["launches"]}
    u64 = sol["fp64"]
    scale = float(u64.abs().max())
    for key in ("fp32", "fp32_polish"):
        out[key]["u_vs_fp64_rel_inf"] = float((sol[key] - u64).abs().max()) / max(scale, 1e-300)
        out[key]["extra_iterations"] = out[key]["newton_iterations"] - out["fp64"]["newton_iterations"]
    out["u_mixed_vs_fp64_rel_inf"] = out["fp32"]["u_vs_fp64_rel_inf"]
    out["extra_iterations_mixed"] = out["fp32"]["extra_iterations"]
    out["polish"] = ("fp32_polish: FP32 tangents until a step reduces ||F|| by less than 10x, then the FP64 "
                     "tangent for the remaining steps")
    out["workload"] = ("config 1: %d^3, knots perturbed +-0.1h (seed 1), lambda=mu=1, l=0.1, BCs of config 0, "
                       "to ||F||_2 < 1e-10 (absolute, the reference's SNES tolerance)" % n)
    out["start"] = ("affine extension of the Dirichlet data (u = F0 X at the Greville abscissae) with the "
                    "Dirichlet rows at their values; from U = 0 the first step leaves a one-element boundary layer "
                    "of strain 0.01/h that the backtracking line search does not unwind at 32^3 and 64^3")
    out["linear_solver"] = ("GMRES(50) right-preconditioned by a geometric multigrid V-cycle on the device "
                            "(stands in for PETSc's GMRES + ASM), rtol %g" % args.newton_ksp_rtol)
    out["timing"] = "host wall clock of igab_newton_solve (phases synchronised)"
    A.close()
    del u64, sol
    torch.cuda.empty_cache()
    return out


def bench_adjoint_static(args, device, n=32):
    """Config 4 (static) end to end at n^3 (32^3 in the config; 64^3 for the metric's mesh):
    per-element stiffness scales s_e = exp(g_e), g ~ N(0, 0.3^2) (seed 4); J = 1/2 sum over
    the control points of face x = 1 of |U - U*|^2 with U* the solution at g* (seed 5).  One
    gradient = the forward Newton solve at g (device), the tangent at the solution, the
    adjoint solve K^T lam = dJ/dU (device multigrid GMRES; K is symmetric), then
    dJ/dg = -lam . dR/dg (igab_adjoint_backward)."""
    import torch
    from igap4standard_b200 import Assembly, mesh
    nelem = (n, n, n)
    kn = mesh.knots_for(nelem, perturb=0.1, seed=1)
    pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
    bc, pd = mesh.bc_config0()
    A = Assembly(nelem, kn, pm, bc, pd, device=device)
    dev = torch.device("cuda", device)
    st = torch.cuda.Stream(device=dev)
    A.set_stream(st.cuda_stream)
    nb = n + 2
    mask = torch.zeros((nb, nb, nb, 3), dtype=torch.float64)
    mask[-1] = 1.0
    mask = mask.reshape(-1).to(dev)
    ne = A.nelem_total
    gstar = np.random.default_rng(5).normal(0.0, 0.3, ne)
    g = np.random.default_rng(4).normal(0.0, 0.3, ne)
    V = torch.empty(A.nnz, dtype=torch.float64, device=dev)
    with torch.cuda.stream(st):
        U0 = torch.as_tensor(A.affine_start(kn, pd)).to(dev)
        Ustar = U0.clone()
        A.set_element_log_scale(gstar)
        A.newton_solve_device(Ustar.data_ptr(), "fp64", ksp_rtol=1e-10)

        def gradient(g):
            t0 = time.perf_counter()
            A.set_element_log_scale(g)
            U = U0.clone()
            fwd = A.newton_solve_device(U.data_ptr(), "fp64", ksp_rtol=1e-10)
            t1 = time.perf_counter()
            A.tangent_device(U.data_ptr(), V.data_ptr(), "fp64")
            b = mask * (U - Ustar)
            lam = torch.zeros_like(U)
            its, ok, _, _ = A.solve_mg_device(V.data_ptr(), b.data_ptr(), lam.data_ptr(), "fp64", 1e-10, 0.0, 2000)
            grad = torch.empty(ne, dtype=torch.float64, device=dev)
            A.adjoint_backward_device(U.data_ptr(), None, lam.data_ptr(), None, grad.data_ptr())
            grad = -grad
            st.synchronize()
            t2 = time.perf_counter()
            J = 0.5 * float((b * b).sum())
            return grad, J, fwd, its, ok, t1 - t0, t2 - t1

        gradient(g)                       # warm-up (graph captures, workspaces)
        grad, J, fwd, its, ok, tf, tb = gradient(g)
    A.set_element_log_scale(None)
    out = {"mesh": [n, n, n], "parameters": ne, "grads_per_s": round(1.0 / (tf + tb), 4), "forward_s": round(tf, 3),
           "adjoint_s": round(tb, 3), "forward_newton_iterations": fwd["iterations"],
           "forward_krylov_iterations": fwd["krylov_iterations"], "forward_fnorm": fwd["fnorm"],
           "adjoint_krylov_iterations": its, "adjoint_converged": bool(ok), "J": J,
           "grad_norm": float(grad.norm()),
           "definition": "one gradient end to end: device Newton solve at g (FP64, KSP rtol 1e-10), tangent at "
                         "the solution, adjoint solve K^T lam = dJ/dU (device multigrid GMRES, rtol 1e-10), "
                         "dJ/dg = -lam . dR/dg; host wall clock"}
    A.close()
    del V
    torch.cuda.empty_cache()
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from igap4standard_b200 import Assembly
    from igap4standard_b200.assembly import dmma_peak_tflops, fma_peak_tflops, tc_peak_tflops

    n = args.n
    nelem, kn, pm, bc, pd = workload(n)
    A = Assembly(nelem, kn, pm, bc, pd, device=local)
    stream = torch.cuda.Stream(device=dev)
    A.set_stream(stream.cuda_stream)
    ndof, nnz, nel = A.ndof, A.nnz, A.nelem_total
    g = torch.Generator(device="cpu").manual_seed(0)
    U_host = (torch.rand(ndof, dtype=torch.float64, generator=g) * 2e-3 - 1e-3)
    U = U_host.to(dev)
    R = torch.empty(ndof, dtype=torch.float64, device=dev)
    V64 = torch.empty(nnz, dtype=torch.float64, device=dev)
    V32 = torch.empty(nnz, dtype=torch.float32, device=dev)
    A.set_profiling(True)

    def step(prec):
        A.residual_device(U.data_ptr(), R.data_ptr())
        launches = A.last_launch_count()
        A.tangent_device(U.data_ptr(), (V64 if prec == "fp64" else V32).data_ptr(), prec)
        launches += A.last_launch_count()
        return launches

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(prec, K, W):
        for _ in range(W):
            step(prec)
            A.last_kernel_ms()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        kms = np.zeros(6)
        launches = 0
        e0.record(stream)
        for _ in range(K):
            launches += step(prec)
            kms += np.array(A.last_kernel_ms())   # waits for this step's events
        e1.record(stream)
        barrier()
        t = e0.elapsed_time(e1) / K
        if world > 1:
            tt = torch.tensor([t], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t, kms / K, launches

    schedule = None
    if not args.no_tune:
        schedule = A.autotune(U.data_ptr(), what=15, reps=2)
        schedule.pop("cached", None)
    peak64_fma = fma_peak_tflops("fp64", local)
    peak64_dmma = dmma_peak_tflops(local)
    peak64 = max(peak64_fma, peak64_dmma)   # DMMA and FP64 FMA issue to one pipe: its best measured rate
    peak32 = fma_peak_tflops("fp32", local)
    peak_tf32 = tc_peak_tflops(256, local)
    peak_tf32_n96 = tc_peak_tflops(96, local)
    clocks = ClockSampler(local)
    clocks.start()
    t64, k64, launches64 = timed("fp64", args.steps, args.warmup)
    clk = clocks.stop()
    t32, k32, launches32 = timed("fp32", args.steps, max(1, args.warmup // 2))

    # ---- end to end through the host-pointer C ABI (pinned host buffers)
    e2e = None
    if not args.no_e2e:
        Uh = U_host.pin_memory()
        Rh = torch.empty(ndof, dtype=torch.float64).pin_memory()
        Vh = torch.empty(nnz, dtype=torch.float64).pin_memory()
        uptr, rptr, vptr = Uh.data_ptr(), Rh.data_ptr(), Vh.data_ptr()
        lib = A.lib
        from igap4standard_b200.native import vp, check

        def e2e_step():
            check(lib, "igab_residual", lib.igab_residual(A.h, vp(uptr), vp(rptr)))
            check(lib, "igab_tangent", lib.igab_tangent(A.h, vp(uptr), vp(vptr), 0))

        e2e_step()
        barrier()
        # each step is synchronous (the C ABI returns with the values in host memory):
        # per-step wall times; the median is reported, since the host and its PCIe links
        # are shared with other jobs and single steps stall by hundreds of ms at times
        # (at least 11 steps, so that the median holds with up to 5 stalled ones)
        ne2e = max(args.steps, 11)
        steps_ms = []
        t0 = time.perf_counter()
        for _ in range(ne2e):
            t1 = time.perf_counter()
            e2e_step()
            steps_ms.append((time.perf_counter() - t1) * 1e3)
        barrier()
        te_mean = (time.perf_counter() - t0) * 1e3 / ne2e
        te = float(np.median(steps_ms))
        if world > 1:
            tt = torch.tensor([te, te_mean], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            te, te_mean = float(tt[0].item()), float(tt[1].item())
        e2e = {"value": round(te / world, 3), "unit": "ms", "h2d_bytes_per_step": 2 * ndof * 8,
               "d2h_bytes_per_step": ndof * 8 + nnz * 8, "ms_per_step": round(te, 3),
               "mean_ms_per_step": round(te_mean, 3), "steps_ms": [round(x, 2) for x in steps_ms],
               "steps": ne2e, "statistic": "median of the per-step wall times (mean over the steps beside it)",
               "timing": "host wall clock around igab_residual + igab_tangent (FP64), pinned host buffers; "
                         "the tangent's rows are downloaded x-slab by x-slab while later slabs are assembled"}
        # the same through the mixed path (FP32 tangent values, 1.22 GB per step)
        del Vh
        Wh = torch.empty(nnz, dtype=torch.float32).pin_memory()
        wptr = Wh.data_ptr()

        def e2e_mixed_step():
            check(lib, "igab_residual", lib.igab_residual(A.h, vp(uptr), vp(rptr)))
            check(lib, "igab_tangent", lib.igab_tangent(A.h, vp(uptr), vp(wptr), 1))

        e2e_mixed_step()
        barrier()
        steps_ms = []
        for _ in range(ne2e):
            t1 = time.perf_counter()
            e2e_mixed_step()
            steps_ms.append((time.perf_counter() - t1) * 1e3)
        barrier()
        tm = float(np.median(steps_ms))
        if world > 1:
            tt = torch.tensor([tm], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            tm = float(tt[0].item())
        e2e["mixed"] = {"value": round(tm / world, 3), "unit": "ms", "ms_per_step": round(tm, 3),
                        "h2d_bytes_per_step": 2 * ndof * 8,
                        "d2h_bytes_per_step": ndof * 8 + nnz * 4, "steps_ms": [round(x, 2) for x in steps_ms],
                        "timing": "as above with the FP32 tangent (igab_tangent, IGAB_PREC_FP32)"}
        del Wh

    # ---- adjoint gradient dJ/dg (s_e = exp(g_e) on every element) at this mesh: one
    # backward pass = dR/dg vector-Jacobian product + K^T lambda on the FP64 tangent
    adjoint = None
    if not args.no_adjoint:
        gen = torch.Generator(device="cpu").manual_seed(4)
        gl = (torch.randn(nel, dtype=torch.float64, generator=gen) * 0.3).to(dev)
        lam = (torch.rand(ndof, dtype=torch.float64, generator=gen) * 2 - 1).to(dev)
        KTl = torch.empty(ndof, dtype=torch.float64, device=dev)
        grad = torch.empty(nel, dtype=torch.float64, device=dev)
        A.set_profiling(False)
        A.adjoint_forward_device(gl.data_ptr(), U.data_ptr(), R.data_ptr(), V64.data_ptr(), "fp64")
        for _ in range(2):
            A.adjoint_backward_device(U.data_ptr(), V64.data_ptr(), lam.data_ptr(), KTl.data_ptr(), grad.data_ptr())
        barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(args.steps):
            A.adjoint_backward_device(U.data_ptr(), V64.data_ptr(), lam.data_ptr(), KTl.data_ptr(), grad.data_ptr())
        a1.record(stream)
        barrier()
        bms = a0.elapsed_time(a1) / args.steps
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        A.adjoint_forward_device(gl.data_ptr(), U.data_ptr(), R.data_ptr(), V64.data_ptr(), "fp64")
        f1.record(stream)
        barrier()
        fms = f0.elapsed_time(f1)
        A.set_element_log_scale(None)
        adjoint = {"grads_per_s": round(1000.0 / bms, 2), "backward_ms": round(bms, 3),
                   "forward_ms": round(fms, 3), "parameters": nel,
                   "definition": "assembly-side adjoint: one gradient = dR/dg VJP (s_e = exp(g_e) per element) + "
                                 "K^T lambda on the FP64 CSR tangent, lambda given; the adjoint linear solve "
                                 "K^T lambda = dJ/dU is the caller's (PETSc KSP in the reference application)"}

    # ---- integrated densities (src/iga_intdensity.c) of the same state: 13 ge densities
    dens = None
    if not args.no_density:
        HHd = torch.empty(16, dtype=torch.float64, device=dev)
        for _ in range(2):
            A.intdensity_device(U.data_ptr(), HHd.data_ptr())
        dlaunch = A.last_launch_count()
        barrier()
        d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        d0.record(stream)
        for _ in range(args.steps):
            A.intdensity_device(U.data_ptr(), HHd.data_ptr())
        d1.record(stream)
        barrier()
        dms = d0.elapsed_time(d1) / args.steps
        dens = {"ms": round(dms, 3), "densities": 13, "launches": int(dlaunch),
                "gauss_points_per_s": round(nel * 64 / (dms * 1e-3), 1),
                "definition": "iga_intdensity: volume integral of the 13 phys/ge densities (energy, stresses, "
                              "volume fractions) at the 64 Gauss points of every element, minus the Neumann "
                              "boundary work; device-resident U, CUDA events"}

    # ---- knot-insertion refinement (mesh/nurbs/nurbs_knotinsert.c) of a 32^3 field to 64^3,
    # host array in place (the reference's interface), and the reference's own routine
    knot = None
    if not args.no_density and rank == 0:
        import ctypes
        lib = A.lib
        kn_nel = np.array([n, n, n], dtype=np.int32)
        per = np.zeros(3, dtype=np.int32)
        base = np.zeros((n + 2) ** 3 * 3)
        nc = (n // 2 + 2) ** 3 * 3
        base[:nc] = np.random.default_rng(6).uniform(-1e-3, 1e-3, nc)
        vp_ = ctypes.c_void_p
        Ut = base.copy()
        lib.igab_knot_insert(Ut.ctypes.data_as(vp_), kn_nel.ctypes.data_as(vp_), 1, 2, 3, per.ctypes.data_as(vp_), local)
        reps = 5
        kms = 0.0
        for _ in range(reps):
            Ut[:] = base
            t0 = time.perf_counter()
            lib.igab_knot_insert(Ut.ctypes.data_as(vp_), kn_nel.ctypes.data_as(vp_), 1, 2, 3, per.ctypes.data_as(vp_), local)
            kms += (time.perf_counter() - t0) * 1e3 / reps
        lib.igab_knot_release(local)
        knot = {"ms": round(kms, 3), "from": [n // 2] * 3, "to": [n] * 3, "dofs": 3 * (n + 2) ** 3,
                "definition": "igab_knot_insert (one level of mid-span knot insertion, host array in place, "
                              "host<->device copies included), wall clock"}
        if not args.no_cpu:
            try:
                from oracle import ref
                if ref.available():
                    Ur = base.copy()
                    t0 = time.perf_counter()
                    ref.lib().nurbs_knotinsert(Ur.ctypes.data_as(vp_), kn_nel.ctypes.data_as(vp_), 1, 2, 3, 3,
                                               per.ctypes.data_as(vp_))
                    knot["reference_cpu_ms"] = round((time.perf_counter() - t0) * 1e3, 3)
                    knot["reference_cpu_cores"] = 1
            except Exception as e:
                knot["reference_cpu_error"] = str(e)

    batch = None
    if not args.no_batch:
        batch = bench_batch(args, dev, local, barrier)
    trans = bench_transient(args, local) if args.transient > 0 else None
    trans_adj = bench_transient_adjoint(args, local) if args.transient_adjoint > 0 else None
    newton1 = None if args.no_newton else bench_newton_config1(args, local)
    adj_static = None if args.no_adjoint_static else bench_adjoint_static(args, local)
    adj_static64 = None if args.no_adjoint_static else bench_adjoint_static(args, local, n=64)

    # ---- roofline of the dominant kernel (tangent volume, 8 colour launches per step)
    tan_ms = k64[2]
    nlaunch = max(k64[5], 1)
    achieved = nel * TAN_ALG_FLOPS / (tan_ms * 1e-3) / 1e12
    executed = nel * TAN_EXEC_FLOPS / (tan_ms * 1e-3) / 1e12
    # DRAM traffic of the FP64 tangent kernel from one ncu capture of a 32^3 colour launch
    # (dram__bytes_read.sum + dram__bytes_write.sum = 151.08 MB + 92.04 MB for 4,096
    # elements), scaled to a launch of this mesh by its elements (the traffic is the CSR
    # read-modify-write of each element matrix, so it grows with the element count)
    traffic = round(TAN64_DRAM_BYTES_PER_ELEMENT * nel / nlaunch)
    roofline = {"bound": "tensor", "pipe": "FP64 tensor (mma.sync m8n8k4 f64) + FP64 FMA", "achieved": round(achieved, 3),
                "peak": round(peak64, 3),
                "unit": "TFLOP/s", "frac": round(achieved / peak64, 4), "traffic": traffic,
                "traffic_source": "ncu dram bytes of one 32^3 colour launch (4,096 elements), scaled per element",
                "kernel": "k_tan_dmma", "avg_launch_ms": round(tan_ms / nlaunch, 3),
                "flops_per_launch": nel * TAN_ALG_FLOPS / nlaunch,
                "flops_definition": "algorithmic B^T D B per element = 64*2*(30*81*10+81*81*10) (effective: the "
                                    "kernel executes %d flops per element)" % TAN_EXEC_FLOPS,
                "executed_tflops": round(executed, 3),
                "peak_fp64_fma": round(peak64_fma, 3), "peak_fp64_dmma": round(peak64_dmma, 3),
                "executed_frac_of_dmma_peak": round(executed / peak64_dmma, 4),
                "peak_source": "measured, burst: the larger of the FP64 FMA probe (igab_fma_peak) and the FP64 "
                               "tensor-pipe probe (igab_dmma_peak, back-to-back mma.sync m8n8k4 f64); "
                               "MEASURED_PEAKS.json has no FP64 figure"}
    res_tf = nel * RES_ALG_FLOPS / (k64[0] * 1e-3) / 1e12 if k64[0] > 0 else None
    # FP32 (mixed) tangent on tcgen05: per element 768 curvature rows in chunks of 32 (about 25 chunks,
    # 8 MMAs M128 x N96 x K8 each); the geometric block runs on the FP32 FMA pipe
    tc_exec_per_el = 25 * 8 * 2 * 128 * 96 * 8
    tan32_ms = k32[2]
    nl32 = max(k32[5], 1)
    roofline_mixed = {"bound": "tensor", "pipe": "TF32 tcgen05 (hi/lo split, FP32 accumulation)",
                      "kernel": "k_tan_tc32<2>", "avg_launch_ms": round(tan32_ms / nl32, 3),
                      "achieved": round(nel * TAN_ALG_FLOPS / (tan32_ms * 1e-3) / 1e12, 3),
                      "executed_tflops": round(nel * tc_exec_per_el / (tan32_ms * 1e-3) / 1e12, 3),
                      "peak": round(peak_tf32, 1), "peak_at_kernel_shape": round(peak_tf32_n96, 1),
                      "unit": "TFLOP/s",
                      "frac": round(nel * TAN_ALG_FLOPS / (tan32_ms * 1e-3) / 1e12 / peak_tf32, 4),
                      "frac_executed_of_shape_peak": round(nel * tc_exec_per_el / (tan32_ms * 1e-3) / 1e12
                                                           / peak_tf32_n96, 4),
                      "peak_source": "measured: igab_tc_peak (back-to-back tcgen05.mma kind::tf32, M128 x N256 / "
                                     "N96, one CTA per SM)"}

    line = {"metric": METRIC, "value": round(t64 / world, 3), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t64, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_dict(n, ndof, nnz),
            "mixed": {"value": round(t32 / world, 3), "unit": "ms", "ms_per_step": round(t32, 3),
                      "speedup_vs_fp64": round(t64 / t32, 3), "dtype": "f32 tangent, f64 residual",
                      "tangent_volume_ms": round(k32[2], 3)},
            "phases_ms": {"residual_volume": round(k64[0], 3), "residual_bc": round(k64[1], 3),
                          "tangent_volume": round(k64[2], 3), "tangent_dirichlet": round(k64[3], 3)},
            "residual_tflops_alg": round(res_tf, 3) if res_tf else None,
            "adjoint_grads_per_s": adjoint["grads_per_s"] if adjoint else None, "adjoint": adjoint,
            "intdensity": dens, "knot_insert": knot,
            "schedule": schedule, "batch_config3": batch, "transient_config2": trans,
            "transient_adjoint_config4": trans_adj, "newton_config1": newton1, "adjoint_config4_e2e": adj_static,
            "adjoint_64cubed_e2e": adj_static64,
            "clocks": clk, "gpu_launches": int(launches64), "roofline": roofline,
            "roofline_mixed": roofline_mixed,
            "peaks_measured": {"fp64_tflops": round(peak64_fma, 2), "fp64_dmma_tflops": round(peak64_dmma, 2), "fp32_tflops": round(peak32, 2),
                               "tf32_tensor_tflops": round(peak_tf32, 1), "tf32_tensor_n96_tflops": round(peak_tf32_n96, 1)},
            "e2e": e2e}

    if rank == 0 and not args.no_cpu:
        try:
            from oracle import ref
            if ref.available():
                P = min(cpu_procs(), 64)
                pool = RefPool(P)
                tr, tt, wall = pool.sample(n)
                pool.close()
                ms = (tr + tt) * nel / P * 1e3
                line["cpu_baseline"] = {"value": round(ms, 1), "unit": "ms", "cores": P, "kind": "reference",
                                        "sample": pool.describe(n) + " (%.1f s wall)" % wall,
                                        "residual_us_per_element": round(tr * 1e6, 3),
                                        "tangent_ms_per_element": round(tt * 1e3, 4),
                                        "residual": "measured on the full element count", "tangent": "extrapolated"}
                if dens is not None:
                    dens["reference_cpu_ms"] = round(pool.td * nel / P * 1e3, 1)
                    dens["reference_cpu_sample"] = ("reference iga_intdensity on the residual sample's slabs "
                                                    "(%d elements), %d processes" % (pool.res_elements, P))
            else:
                line["cpu_baseline"] = None
        except Exception as e:
            line["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(line))
    A.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
