"""The ctypes mirrors of the option / info structs of include/igab.h have the C layout:
a small C program compiled here with the system compiler prints sizeof and offsetof of
every member, which must equal ctypes' figures (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "igab_mesh_desc": "IgabMeshDesc",
    "igab_tune_result": "IgabTuneResult",
    "igab_batch_tune_result": "IgabBatchTuneResult",
    "igab_solve_info": "IgabSolveInfo",
    "igab_newton_opts": "IgabNewtonOpts",
    "igab_newton_info": "IgabNewtonInfo",
    "igab_transient_opts": "IgabTransientOpts",
    "igab_transient_info": "IgabTransientInfo",
    "igab_tadj_info_t": "IgabTadjInfo",
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_c_layout(tmp_path):
    from igap4standard_b200 import native
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "igab.h"', "int main(void) {"]
    for c_name, py_name in STRUCTS.items():
        cls = getattr(native, py_name)
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (c_name, c_name))
        for field, _ in cls._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (c_name, field, c_name, field))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                  text=True).stdout.splitlines())
    for c_name, py_name in STRUCTS.items():
        cls = getattr(native, py_name)
        assert int(got[c_name]) == __import__("ctypes").sizeof(cls), c_name
        for field, _ in cls._fields_:
            assert int(got["%s.%s" % (c_name, field)]) == getattr(cls, field).offset, (c_name, field)
