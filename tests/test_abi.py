"""C ABI surface, host-side logic and the PETSc subset (no GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    src = open(os.path.join(REPO, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    names = []
    for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M):
        name = m.group(1)
        if name not in ("if", "for", "while", "return", "sizeof", "typedef"):
            names.append(name)
    return [n for n in names if not n.endswith("_ptr")]


@pytest.mark.parametrize("header,lib", [("igab.h", "libigap4_b200.so"),
                                        ("snesiga_b200.h", "libsnesiga_b200.so"),
                                        ("iga_case.h", "libsnesiga_b200.so")])
def test_library_exports_every_declared_symbol(built, header, lib):
    from igap4standard_b200 import native
    native.lib_cuda()
    native.lib_dropin()
    L = ctypes.CDLL(os.path.join(native.LIBDIR, lib))
    names = declared_functions(header)
    assert len(names) > 3
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_bindings_cover_header(built):
    from igap4standard_b200 import native
    bound = {n for n, _, _ in native.IGAB_API}
    assert set(declared_functions("igab.h")) <= bound


def test_create_rejects_bad_arguments(built):
    """Argument checks run before any CUDA call, so they work without a GPU."""
    from igap4standard_b200 import Assembly, IgabError, knots_for, PAR_MAT_DEFAULT, bc_config0
    bc, pd = bc_config0()
    with pytest.raises(IgabError) as e:
        Assembly((0, 2, 2), np.zeros(5 + 7 + 7), PAR_MAT_DEFAULT, bc, pd)
    assert e.value.code == 1
    kn = knots_for((2, 2, 2))
    kn[3], kn[4] = kn[4], kn[3] + 0.1   # decreasing knots
    with pytest.raises(IgabError):
        Assembly((2, 2, 2), kn, PAR_MAT_DEFAULT, bc, pd)
    with pytest.raises(ValueError):
        Assembly((2, 2, 2), np.zeros(5), PAR_MAT_DEFAULT, bc, pd)


def test_mesh_helpers():
    from igap4standard_b200 import mesh
    assert mesh.n_dof((8, 8, 8)) == 3000
    assert mesh.n_dof((64, 64, 64)) == 862488
    assert mesh.nnz_of((8, 8, 8)) == 766656
    assert mesh.nnz_of((64, 64, 64)) == 306110016
    kv = mesh.open_knot_vector(16, perturb=0.1, rng=np.random.default_rng(1))
    assert kv.size == 21 and np.all(np.diff(kv) >= 0) and kv[2] == 0 and kv[-3] == 1
    h = 1 / 16
    assert np.all(np.abs(kv[3:-3] - np.arange(1, 16) * h) <= 0.1 * h + 1e-15)
    pm = mesh.par_mat_from_lame(1.0, 1.0, 0.1)
    c36, c37, c38 = mesh.ge_coefficients(pm)
    assert abs(c37 - 1.0) < 1e-12          # deviatoric quadratic coefficient = mu
    assert pm[2] == 2.5 and pm[3] == 2.0 and pm[4] == 0.1
    # reference default parameters satisfy phys/ge/assert_par_mat.c
    r, cu = mesh.PAR_MAT_DEFAULT[:2]
    assert 2 * r * r - 2 * r * r * cu > 0 and 4 / 3 * r - 4 / 3 * r * cu > 0


def test_bc_presets():
    from igap4standard_b200 import mesh
    bc, pd = mesh.bc_config0()
    assert list(bc[:6]) == [0] * 6 and list(bc[6:12]) == [0, 1, 1, 1, 1, 1] and all(bc[12:] == 1)
    assert pd[0] == 0.01 and np.count_nonzero(pd) == 1


# ---- PETSc subset semantics used by the callbacks
def _subset():
    from igap4standard_b200 import native
    native.lib_dropin()
    L = ctypes.CDLL(native.LIB_SUBSET)
    vp = ctypes.c_void_p
    for f, a in [("MatCreateSeqAIJ", [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp]),
                 ("MatSetValues", [vp, ctypes.c_int, vp, ctypes.c_int, vp, vp, ctypes.c_int]),
                 ("MatAssemblyBegin", [vp, ctypes.c_int]), ("MatAssemblyEnd", [vp, ctypes.c_int]),
                 ("MatZeroRowsColumns", [vp, ctypes.c_int, vp, ctypes.c_double, vp, vp]),
                 ("MatGetRowIJ", [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]),
                 ("MatSeqAIJGetArray", [vp, vp]), ("MatDestroy", [vp]), ("petsc_subset_mat_error", [vp])]:
        getattr(L, f).argtypes = a
        getattr(L, f).restype = ctypes.c_int
    return L


def test_subset_mat_semantics(built):
    L = _subset()
    vp = ctypes.c_void_p
    A = vp()
    nnz = np.array([3, 3, 3], dtype=np.int32)
    assert L.MatCreateSeqAIJ(0, 3, 3, 0, nnz.ctypes.data, ctypes.byref(A)) == 0
    rows = np.array([0, 2], dtype=np.int32)
    cols = np.array([2, 0], dtype=np.int32)
    v = np.array([1.0, 2.0, 3.0, 4.0])
    ADD, INSERT = 2, 1
    L.MatSetValues(A, 2, rows.ctypes.data, 2, cols.ctypes.data, v.ctypes.data, ADD)
    L.MatSetValues(A, 2, rows.ctypes.data, 2, cols.ctypes.data, v.ctypes.data, ADD)
    one = np.array([1], dtype=np.int32)
    z = np.array([0.0])
    L.MatSetValues(A, 1, one.ctypes.data, 1, one.ctypes.data, z.ctypes.data, INSERT)   # explicit zero kept
    L.MatAssemblyBegin(A, 0)
    L.MatAssemblyEnd(A, 0)
    n = ctypes.c_int()
    ia, ja = ctypes.POINTER(ctypes.c_int)(), ctypes.POINTER(ctypes.c_int)()
    done = ctypes.c_int()
    L.MatGetRowIJ(A, 0, 0, 0, ctypes.byref(n), ctypes.byref(ia), ctypes.byref(ja), ctypes.byref(done))
    assert done.value == 1 and [ia[i] for i in range(4)] == [0, 2, 3, 5]
    assert [ja[i] for i in range(5)] == [0, 2, 1, 0, 2]     # ascending within each row
    a = ctypes.POINTER(ctypes.c_double)()
    L.MatSeqAIJGetArray(A, ctypes.byref(a))
    assert [a[i] for i in range(5)] == [4.0, 2.0, 0.0, 8.0, 6.0]
    r = np.array([2], dtype=np.int32)
    L.MatZeroRowsColumns(A, 1, r.ctypes.data, 1.0, None, None)
    assert [a[i] for i in range(5)] == [4.0, 0.0, 0.0, 0.0, 1.0]
    bad = np.array([7], dtype=np.int32)
    assert L.MatSetValues(A, 1, bad.ctypes.data, 1, bad.ctypes.data, v.ctypes.data, ADD) != 0
    assert L.petsc_subset_mat_error(A) != 0
    L.MatDestroy(ctypes.byref(A))


def test_shard_covers_all():
    from igap4standard_b200.replicas import shard
    for n in [0, 1, 7, 512]:
        for w in [1, 2, 3, 8]:
            parts = [shard(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(w - 1))
            assert max(h - l for l, h in parts) - min(h - l for l, h in parts) <= 1


def _gloo_worker(rank, world, port, q):
    import os
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from igap4standard_b200.replicas import max_over_ranks, shard
    lo, hi = shard(512, rank, world)
    m = max_over_ranks(10.0 * (rank + 1))
    q.put((rank, lo, hi, m))
    dist.destroy_process_group()


def test_replicas_gloo_world2():
    """Two CPU ranks: instance shards partition the batch, timing reduces to the max."""
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
    assert out[0][1:3] == (0, 256) and out[1][1:3] == (256, 512)
    assert out[0][3] == 20.0 and out[1][3] == 20.0
