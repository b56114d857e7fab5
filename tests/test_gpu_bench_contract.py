"""bench.py's own arm on a small mesh: one JSON line with the keys a driver reads
(metric, value, steps, warmup, clocks, gpu_launches, roofline, cpu_baseline, and
e2e with the bytes it copies), values consistent with the mesh."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_small_mesh(built):
    n = 16
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--n", str(n), "--steps", "3",
                          "--warmup", "3", "--no-batch", "--no-adjoint", "--no-density", "--no-tune",
                          "--transient", "0", "--transient-adjoint", "0", "--no-adjoint-static"], cwd=REPO, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "dtype", "data", "config", "clocks", "gpu_launches", "roofline", "cpu_baseline", "e2e", "mixed"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0
    assert d["gpu_launches"] > 0
    ndof = 3 * (n + 2) ** 3
    assert d["config"]["dofs"] == ndof
    nnz = d["config"]["nnz"]
    e = d["e2e"]
    assert e["h2d_bytes_per_step"] == 2 * ndof * 8
    assert e["d2h_bytes_per_step"] == ndof * 8 + nnz * 8
    assert e["steps"] >= 11 and len(e["steps_ms"]) == e["steps"] and e["value"] > 0
    assert e["mixed"]["d2h_bytes_per_step"] == ndof * 8 + nnz * 4
    r = d["roofline"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in r, k
    assert r["achieved"] > 0 and r["peak"] > 0 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-3
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] > 0 and cb["cores"] >= 1
    assert "sm_mhz" in d["clocks"] and "reasons" in d["clocks"]
    nw = d["newton_config1"]
    for prec in ("fp64", "fp32"):
        assert nw[prec]["converged"] and nw[prec]["final_fnorm"] < 1e-10 and nw[prec]["newton_iterations"] >= 1
    assert nw["extra_iterations_mixed"] <= 1 and nw["u_mixed_vs_fp64_rel_inf"] < 1e-6
