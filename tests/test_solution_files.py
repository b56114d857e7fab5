"""Solution files (src/ioutil.c:89 write_solution, :126 read_solution) on one rank:
files written by the library's igab_write_solution and by the drop-in are read
back bit for bit by the reference's own read_solution, and files the reference
writes are read back by both (no GPU needed)."""
import ctypes
import os

import numpy as np

from cases import make_transient_case


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_solution_files_match_reference(built, oracle_lib, tmp_path):
    from igap4standard_b200 import native, gpu_case
    c = make_transient_case("getime_small")
    args = ("getime", c["nelem"], c["knots"], c["par_mat"], c["bc_type"], c["par_periodic"], c["par_dirichlet"],
            c["par_neumann"])
    ref = oracle_lib.case(*args)
    n = ref.ndof
    hist = np.random.default_rng(4).normal(size=(3, n))
    io_ref = ref.lib.iga_case_iocomm(ref.h)
    lib = native.lib_cuda()
    # library writer -> reference reader (levels 1..2)
    f1 = str(tmp_path / "ours.bin").encode()
    assert lib.igab_write_solution(f1, _p(hist), n, 1, 3) == 0
    assert os.path.getsize(f1) == 2 * n * 8
    back = np.zeros((3, n))
    ref.lib.read_solution(f1, _p(back), io_ref, 1, 3)
    assert np.array_equal(back[1:], hist[1:]) and np.array_equal(back[0], np.zeros(n))
    # reference writer -> library reader and drop-in reader
    f2 = str(tmp_path / "ref.bin").encode()
    ref.lib.write_solution(f2, _p(hist), io_ref, 0, 3)
    mine = np.zeros((3, n))
    assert lib.igab_read_solution(f2, _p(mine), n, 0, 3) == 0
    assert np.array_equal(mine, hist)
    gpu = gpu_case(*args)
    io_gpu = gpu.lib.iga_case_iocomm(gpu.h)
    drop = np.zeros((3, n))
    gpu.lib.read_solution(f2, _p(drop), io_gpu, 0, 3)
    assert np.array_equal(drop, hist)
    # drop-in writer -> reference reader
    f3 = str(tmp_path / "dropin.bin").encode()
    gpu.lib.write_solution(f3, _p(hist), io_gpu, 0, 3)
    back3 = np.zeros((3, n))
    ref.lib.read_solution(f3, _p(back3), io_ref, 0, 3)
    assert np.array_equal(back3, hist)
    # a short file is an error for the library reader
    assert lib.igab_read_solution(f1, _p(mine), n, 0, 3) != 0
