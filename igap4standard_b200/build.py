"""Build the native libraries of igap4standard_b200 in-tree (igap4standard_b200/lib/).

  libigap4_b200.so    CUDA kernels + C ABI (include/igab.h), sm_100a only
  libpetsc_subset.so  sequential PETSc/MPI subset (where no PETSc is installed)
  libsnesiga_b200.so  PETSc SNES drop-in callbacks + single-rank case builder
                      (include/snesiga_b200.h, include/iga_case.h)

nvcc cross-compiles for sm_100a without a GPU.  Rebuilds only what is older
than its sources.  ``python -m igap4standard_b200.build [--force]``.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
SUBSET = os.path.join(CSRC, "petsc_subset")
INC = os.path.join(REPO, "include")
LIBDIR = os.path.join(PKG, "lib")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INC]

CUDA_SOURCES = ["igab_kernels.cu", "igab_tangent_dmma.cu", "igab_tangent_tc.cu", "igab_getime.cu", "igab_capi.cu",
                "igab_batch.cu", "igab_autotune.cu", "igab_noalloc.cu", "igab_density.cu", "igab_krylov.cu",
                "igab_refine.cu", "igab_newton.cu", "igab_mg.cu", "igab_transient.cu", "igab_periodic.cu"]
CUDA_HEADERS = ["igab_internal.h", "igab_math.cuh", "igab_device.cuh", "igab_warp_tiles8.inc", "igab_tc.cuh",
                "igab_reduce.cuh"]

LIB_CUDA = os.path.join(LIBDIR, "libigap4_b200.so")
LIB_SUBSET = os.path.join(LIBDIR, "libpetsc_subset.so")
LIB_DROPIN = os.path.join(LIBDIR, "libsnesiga_b200.so")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in CUDA_HEADERS] + [os.path.join(INC, "igab.h")]
    # ---- CUDA library
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    if force or _stale(LIB_CUDA, srcs + hdrs + [__file__]):
        objs = [os.path.join(LIBDIR, os.path.basename(s) + ".o") for s in srcs]
        with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 4))) as ex:
            list(ex.map(lambda so: _run([NVCC] + NVCC_FLAGS + ["-c", so[0], "-o", so[1]]), zip(srcs, objs)))
        _run([NVCC] + ARCH + ["-shared", "-o", LIB_CUDA] + objs)
        for o in objs:
            os.remove(o)
        if verbose:
            print("built", LIB_CUDA)
    # ---- PETSc/MPI subset
    sub_src = os.path.join(SUBSET, "petsc_subset.c")
    sub_hdr = [os.path.join(SUBSET, "petscsnes.h"), os.path.join(SUBSET, "mpi.h")]
    if force or _stale(LIB_SUBSET, [sub_src] + sub_hdr + [__file__]):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu99", "-I", SUBSET, sub_src, "-o", LIB_SUBSET, "-lm"])
        if verbose:
            print("built", LIB_SUBSET)
    # ---- drop-in callbacks + case builder
    dsrc = [os.path.join(CSRC, "snesiga_b200.c"), os.path.join(CSRC, "iga_case.c")]
    dhdr = [os.path.join(INC, h) for h in ("snesiga_b200.h", "igap4_structs.h", "iga_case.h", "igab.h")]
    if force or _stale(LIB_DROPIN, dsrc + dhdr + sub_hdr + [LIB_CUDA, LIB_SUBSET, __file__]):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu99", "-Wall", "-Wno-unused-result",
              "-I", SUBSET, "-I", INC] + dsrc +
             ["-L", LIBDIR, "-ligap4_b200", "-lpetsc_subset", "-Wl,-rpath,$ORIGIN", "-o", LIB_DROPIN])
        if verbose:
            print("built", LIB_DROPIN)
    return [LIB_CUDA, LIB_SUBSET, LIB_DROPIN]


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
