"""Python face of the batched assembly (igab_batch_* of include/igab.h): many
independent phys/ge meshes of uneven size assembled by one persistent launch
per operator."""
import ctypes

import numpy as np

from . import native
from .assembly import PREC, _ptr
from .native import IgabMeshDesc, check, vp


class Batch:
    """instances: iterable of dicts with nelem, knots, par_mat, bc_type, par_dirichlet
    (and optionally par_periodic), e.g. mesh.batch_config3()."""

    def __init__(self, instances, device=0):
        self.lib = native.lib_cuda()
        inst = list(instances)
        descs = (IgabMeshDesc * len(inst))()
        self._knots = []
        for d, c in zip(descs, inst):
            d.phys = 0
            for i in range(3):
                d.nelem[i] = int(c["nelem"][i])
            k = np.ascontiguousarray(c["knots"], dtype=np.float64)
            self._knots.append(k)
            d.knots = k.ctypes.data_as(native.c_double_p)
            pp = c.get("par_periodic")
            for i in range(9):
                d.par_mat[i] = float(c["par_mat"][i])
                d.par_dirichlet[i] = float(c["par_dirichlet"][i])
                d.par_periodic[i] = float(pp[i]) if pp is not None else 0.0
            for i in range(36):
                d.bc_type[i] = int(c["bc_type"][i])
        h = vp()
        check(self.lib, "igab_batch_create", self.lib.igab_batch_create(descs, len(inst), int(device), ctypes.byref(h)))
        self.h = h
        self.n = len(inst)
        self.sizes = [tuple(int(x) for x in c["nelem"]) for c in inst]
        self.device = int(device)
        nd, nz, ne = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
        self.dof_offsets = np.zeros(self.n + 1, dtype=np.int64)
        self.nnz_offsets = np.zeros(self.n + 1, dtype=np.int64)
        check(self.lib, "igab_batch_sizes",
              self.lib.igab_batch_sizes(h, ctypes.byref(nd), ctypes.byref(nz), ctypes.byref(ne),
                                        _ptr(self.dof_offsets), _ptr(self.nnz_offsets)))
        self.ndof, self.nnz, self.nelem_total = nd.value, nz.value, ne.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.igab_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def instance_handle(self, i):
        return self.lib.igab_batch_instance(self.h, int(i))

    def pattern(self, i):
        """(rowptr, cols) of instance i's AIJ pattern."""
        h = self.instance_handle(i)
        n = self.dof_offsets[i + 1] - self.dof_offsets[i]
        z = self.nnz_offsets[i + 1] - self.nnz_offsets[i]
        rowptr = np.empty(n + 1, dtype=np.int32)
        cols = np.empty(z, dtype=np.int32)
        check(self.lib, "igab_csr_pattern", self.lib.igab_csr_pattern(h, _ptr(rowptr), _ptr(cols)))
        return rowptr, cols

    def set_schedule(self, ctas_res=0, ctas_tan64=0, ctas_tan32=0, order=0):
        check(self.lib, "igab_batch_set_schedule",
              self.lib.igab_batch_set_schedule(self.h, int(ctas_res), int(ctas_tan64), int(ctas_tan32), int(order)))

    def get_schedule(self):
        v = [ctypes.c_int() for _ in range(4)]
        check(self.lib, "igab_batch_get_schedule", self.lib.igab_batch_get_schedule(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def set_colour_order(self, order):
        check(self.lib, "igab_batch_set_colour_order", self.lib.igab_batch_set_colour_order(self.h, int(order)))

    def get_colour_order(self):
        v = ctypes.c_int()
        check(self.lib, "igab_batch_get_colour_order", self.lib.igab_batch_get_colour_order(self.h, ctypes.byref(v)))
        return v.value

    def autotune(self, U_ptr=None, what=7, reps=2, cache=None):
        """Time the candidate batch schedules (igab_batch_autotune) and keep the fastest;
        with a cache file, a schedule stored for this GPU and batch shape is applied."""
        from . import tuning
        key = tuning.batch_key(self.device, self.sizes, what) if cache else None
        hit = tuning.load(cache).get(key) if cache else None
        if hit:
            self.set_schedule(hit["ctas_res"], hit["ctas_tan64"], hit["ctas_tan32"], hit["order"])
            self.set_colour_order(hit.get("colour_order", 0))
            return dict(hit, cached=True)
        r = native.IgabBatchTuneResult()
        check(self.lib, "igab_batch_autotune",
              self.lib.igab_batch_autotune(self.h, vp(U_ptr or 0), int(what), int(reps), ctypes.byref(r)))
        out = {f: getattr(r, f) for f, _ in native.IgabBatchTuneResult._fields_}
        if cache:
            tuning.store(cache, key, out)
        return dict(out, cached=False)

    def set_stream(self, stream_ptr):
        check(self.lib, "igab_batch_set_stream", self.lib.igab_batch_set_stream(self.h, vp(stream_ptr)))

    def residual_device(self, U_ptr, R_ptr):
        check(self.lib, "igab_batch_residual_device", self.lib.igab_batch_residual_device(self.h, vp(U_ptr), vp(R_ptr)))

    def tangent_device(self, U_ptr, vals_ptr, prec="fp64"):
        check(self.lib, "igab_batch_tangent_device",
              self.lib.igab_batch_tangent_device(self.h, vp(U_ptr), vp(vals_ptr), PREC[prec]))

    def graph_capture(self, U_ptr, R_ptr, vals_ptr, prec="fp64"):
        check(self.lib, "igab_batch_graph_capture",
              self.lib.igab_batch_graph_capture(self.h, vp(U_ptr), vp(R_ptr), vp(vals_ptr), PREC[prec]))

    def graph_launch(self):
        check(self.lib, "igab_batch_graph_launch", self.lib.igab_batch_graph_launch(self.h))

    def sync(self):
        check(self.lib, "igab_batch_sync", self.lib.igab_batch_sync(self.h))

    def set_wait_limit(self, polls=0, unreachable=False):
        """Poll limit of the colour-dependency wait (0 = default); unreachable=True makes
        the waits on colour 0 of instance 0 run out (test switch of the give-up path)."""
        check(self.lib, "igab_batch_set_wait_limit",
              self.lib.igab_batch_set_wait_limit(self.h, int(polls), 1 if unreachable else 0))

    def last_launch_count(self):
        n = ctypes.c_int()
        check(self.lib, "igab_batch_last_launch_count", self.lib.igab_batch_last_launch_count(self.h, ctypes.byref(n)))
        return n.value

    # ---- host convenience (torch for device memory)
    def residual(self, U):
        import torch
        dev = torch.device("cuda", self.device)
        Ud = torch.as_tensor(np.ascontiguousarray(U, dtype=np.float64)).to(dev)
        R = torch.empty(self.ndof, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        self.residual_device(Ud.data_ptr(), R.data_ptr())
        self.sync()
        return R.cpu().numpy()

    def tangent(self, U, prec="fp64"):
        import torch
        dev = torch.device("cuda", self.device)
        Ud = torch.as_tensor(np.ascontiguousarray(U, dtype=np.float64)).to(dev)
        V = torch.empty(self.nnz, dtype=torch.float64 if prec == "fp64" else torch.float32, device=dev)
        torch.cuda.synchronize(dev)
        self.tangent_device(Ud.data_ptr(), V.data_ptr(), prec)
        self.sync()
        return V.cpu().numpy()
