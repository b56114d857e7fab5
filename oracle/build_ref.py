#!/usr/bin/env python3
"""Build the reference oracle: IGAP4STANDARD's own assembly code, compiled in place.

Test infrastructure only.  This recipe compiles the reference's C sources
where they lie (never copied into this repository) together with

  * the project's sequential PETSc/MPI subset
    (igap4standard_b200/csrc/petsc_subset/), which stands in for PETSc 3.7
    and MPI, both absent from this image, and
  * the project's single-rank case builder (igap4standard_b200/csrc/iga_case.c),
    which fills the reference's structs and calls the reference's own
    snesiga_init / snesiga_Residual / snesiga_Tangent,

into ``oracle/_ref/libref_iga.so``.  Nothing else is written.  The reference
sources compiled (paths inside the reference project):

  src/snesiga_Residual.c  src/snesiga_Tangent.c  src/snesiga_init.c
  src/iga_dirichlet.c     src/quadrature.c       src/mathutil.c
  src/iga_intdensity.c     src/ioutil.c
  mesh/nurbs/eval_Bspline.c  mesh/nurbs/evalN.c  mesh/nurbs/nurbs_knotinsert.c
  phys/ge/{init,assert_par_mat,residual,tangent,density,field}.c
  phys/getime/{init,assert_par_mat,residual,tangent,density,field}.c

Flags follow the reference's makefiles (src/makefile:2: -O3 -std=c99 -fPIC),
with -std=gnu99 (the non-static ``inline`` of include/mathutil.h needs GNU
semantics here) and -march=x86-64-v3 instead of -march=native so that the
library also runs on the GPU hosts' CPUs.

oracle/elem_scale.c wraps the reference's integrand pointers with a per-element
scale (the adjoint tests' oracle of the element-scaled problem).

The struct-layout probe (oracle/layout_probe.c) is compiled twice, once with
the reference's headers and once with include/igap4_structs.h, so the tests
can check that both declare byte-identical structs.

Usage: python oracle/build_ref.py [--reference DIR] [--force]
Exit status 0 also when the reference tree is absent (prints why, builds nothing).
"""
import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT_DIR = os.path.join(HERE, "_ref")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
SUBSET = os.path.join(REPO, "igap4standard_b200", "csrc", "petsc_subset")
CASE_SRC = os.path.join(REPO, "igap4standard_b200", "csrc", "iga_case.c")
OUR_INC = os.path.join(REPO, "include")
LIB = os.path.join(OUT_DIR, "libref_iga.so")

REF_SOURCES = [
    "src/snesiga_Residual.c", "src/snesiga_Tangent.c", "src/snesiga_init.c",
    "src/iga_dirichlet.c", "src/quadrature.c", "src/mathutil.c", "src/iga_intdensity.c", "src/ioutil.c",
    "mesh/nurbs/eval_Bspline.c", "mesh/nurbs/evalN.c", "mesh/nurbs/nurbs_knotinsert.c",
    "phys/ge/init.c", "phys/ge/assert_par_mat.c", "phys/ge/residual.c", "phys/ge/tangent.c",
    "phys/ge/density.c", "phys/ge/field.c",
    "phys/getime/init.c", "phys/getime/assert_par_mat.c", "phys/getime/residual.c",
    "phys/getime/tangent.c", "phys/getime/density.c", "phys/getime/field.c",
]

CFLAGS = ["-O3", "-std=gnu99", "-fPIC", "-march=x86-64-v3", "-w"]


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))


def obj_name(rel):
    return os.path.join(OBJ_DIR, rel.replace("/", "__").replace(".c", ".o"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("IGAP4_REFERENCE", os.path.join(os.path.dirname(REPO),
                                                                                        "reference")),
                    help="the reference tree (default: $IGAP4_REFERENCE, else a directory named "
                         "'reference' beside this repository)")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    ref = args.reference
    if not os.path.isdir(os.path.join(ref, "src")):
        print("build_ref: reference tree not found at %s; oracle/_ref not built" % ref)
        return 0
    os.makedirs(OBJ_DIR, exist_ok=True)
    newest_src = max(os.path.getmtime(p) for p in
                     [os.path.join(ref, s) for s in REF_SOURCES] +
                     [CASE_SRC, os.path.join(SUBSET, "petsc_subset.c"), __file__,
                      os.path.join(HERE, "elem_scale.c"),
                      os.path.join(HERE, "layout_probe.c"), os.path.join(OUR_INC, "igap4_structs.h")])
    if os.path.exists(LIB) and os.path.getmtime(LIB) > newest_src and not args.force:
        print("build_ref: %s is up to date" % LIB)
        return 0

    ref_inc = ["-I", SUBSET, "-I", os.path.join(ref, "include")]
    our_inc = ["-I", SUBSET, "-I", OUR_INC]
    jobs = []
    for rel in REF_SOURCES:
        jobs.append(["gcc"] + CFLAGS + ref_inc + ["-c", os.path.join(ref, rel), "-o", obj_name(rel)])
    jobs.append(["gcc"] + CFLAGS + our_inc + ["-c", CASE_SRC, "-o", os.path.join(OBJ_DIR, "iga_case.o")])
    jobs.append(["gcc"] + CFLAGS + our_inc + ["-c", os.path.join(SUBSET, "petsc_subset.c"),
                                             "-o", os.path.join(OBJ_DIR, "petsc_subset.o")])
    probe = os.path.join(HERE, "layout_probe.c")
    jobs.append(["gcc"] + CFLAGS + ref_inc + ["-DPROBE_REFERENCE_HEADERS", "-c", probe,
                                             "-o", os.path.join(OBJ_DIR, "layout_ref.o")])
    jobs.append(["gcc"] + CFLAGS + our_inc + ["-c", probe, "-o", os.path.join(OBJ_DIR, "layout_ours.o")])
    jobs.append(["gcc"] + CFLAGS + ref_inc + ["-c", os.path.join(HERE, "elem_scale.c"),
                                             "-o", os.path.join(OBJ_DIR, "elem_scale.o")])
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(run, jobs))
    objs = [obj_name(r) for r in REF_SOURCES] + [os.path.join(OBJ_DIR, n) for n in
                                                 ("iga_case.o", "petsc_subset.o", "layout_ref.o", "layout_ours.o",
                                                  "elem_scale.o")]
    run(["gcc", "-shared", "-o", LIB] + objs + ["-lm"])
    print("build_ref: built %s" % LIB)
    return 0


if __name__ == "__main__":
    sys.exit(main())
