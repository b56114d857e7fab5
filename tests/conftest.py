import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than ~30 s")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def built():
    """Native libraries, built in-tree if missing (nvcc cross-compiles without a GPU)."""
    from igap4standard_b200 import build
    build.build()
    return True


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference oracle library oracle/_ref/libref_iga.so not built")
    return ref


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(REPO, "tests", "golden", "reference_vectors.npz")
    return dict(np.load(path))


@pytest.fixture(scope="session")
def port_oracle():
    from oracle import port
    port.lib()
    return port


@pytest.fixture(scope="session")
def host_math():
    """igab_math.cuh compiled for the host (the device kernels' point mathematics)."""
    import ctypes
    import subprocess
    src = os.path.join(REPO, "tests", "host", "igab_math_host.cpp")
    inc = os.path.join(REPO, "igap4standard_b200", "csrc")
    out_dir = os.path.join(REPO, "tests", "_build")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libigab_math_host.so")
    deps = [src, os.path.join(inc, "igab_math.cuh")]
    if not os.path.exists(out) or os.path.getmtime(out) < max(os.path.getmtime(d) for d in deps):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", inc, src, "-o", out], check=True)
    L = ctypes.CDLL(out)
    vp = ctypes.c_void_p
    L.host_ge_point.argtypes = [vp, vp, vp, vp]
    L.host_bspline_p2.argtypes = [vp, ctypes.c_double, vp]
    L.host_getime_point.argtypes = [vp, vp, vp, vp]
    return L


@pytest.fixture(scope="session")
def checker():
    """Factory of reference cases: the reference's own code (oracle/_ref) when it
    is built, else the CPU restatement (oracle/port), pinned to the same
    golden vectors.  Returns f(phys, nelem, knots, par_mat, bc_type, pp, pd, pn)."""
    from oracle import ref, port
    if ref.available():
        return lambda *a: ref.case(*a)
    port.lib()

    def make(phys, *a):
        assert phys == "ge"
        return port.PortCase(*a)
    return make
