"""Batched PIV: many image pairs (2D and 3D, mixed sizes, algorithms, masks
and multi-pass refinement) in one pre-allocated schedule captured as a CUDA
graph (include/mqp.h, mqp_batch_plan_*).  Each pair's (VF, SN) equals
PIV(img1, img2, [mask,] pivparams) for that pair alone.

    plan = BatchPlan([(img1, img2, params), (v1, v2, params3d, mask), ...])
    plan.run(); torch.cuda.synchronize()
    VF0, SN0 = plan.results()[0]

Images may be NumPy arrays (copied to the device once, at plan creation) or
torch CUDA tensors (used in place when already column-major).  Results are
torch CUDA tensors shaped like PIV's outputs.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .piv import PIVParameters, get_vectorfield_size


def _colmajor(t):
    nd = t.dim()
    perm = tuple(range(nd - 1, -1, -1))
    return t.permute(perm).contiguous().permute(perm)


def _device_image(x, dtype, dev):
    import torch
    t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.asarray(x))
    return _colmajor(t.to(device=dev, dtype=dtype))


class BatchPlan:
    """A batched PIV schedule over fixed device buffers (see module doc)."""

    def __init__(self, pairs: Sequence[tuple], options: Optional[dict] = None,
                 context: Optional[_lib.Context] = None, device: int = 0):
        import torch
        self.ctx = context or _lib.default_context(device)
        dev = torch.device("cuda", self.ctx.device)
        self._keep = []
        self.outputs = []
        items = (_lib.MqpBatchItem * max(len(pairs), 1))()
        for k, pr in enumerate(pairs):
            img1, img2, params = pr[0], pr[1], pr[2]
            mask = pr[3] if len(pr) > 3 else None
            mask_skip = pr[4] if len(pr) > 4 else None
            if not isinstance(params, PIVParameters):
                raise TypeError("each pair is (img1, img2, PIVParameters[, mask[, mask_skip]])")
            if tuple(img1.shape) != tuple(img2.shape):
                raise AssertionError("PIV inputs need to have the same size.")
            nd = len(img1.shape)
            params.ndims = nd
            f64 = any(str(getattr(x, "dtype", "")).endswith("float64") for x in (img1, img2))
            dt = torch.float64 if f64 else torch.float32
            t1, t2 = _device_image(img1, dt, dev), _device_image(img2, dt, dev)
            tm = _device_image(mask, dt, dev) if mask is not None else None
            ts = _device_image(mask_skip, dt, dev) if mask_skip is not None else None
            vf = get_vectorfield_size(tuple(img1.shape), params)
            VF = torch.zeros(tuple(reversed((nd,) + tuple(vf))), dtype=torch.float64, device=dev)
            SN = torch.zeros(tuple(reversed(tuple(vf))), dtype=torch.float64, device=dev) if params.computeSN else None
            self._keep += [t1, t2, tm, ts, VF, SN]
            self.outputs.append((VF.permute(tuple(range(nd, -1, -1))),
                                 SN.permute(tuple(range(nd - 1, -1, -1))) if SN is not None else None))
            it = items[k]
            it.img1, it.img2 = t1.data_ptr(), t2.data_ptr()
            it.mask = tm.data_ptr() if tm is not None else None
            it.mask_skip = ts.data_ptr() if ts is not None else None
            it.dtype = _lib.MQP_F64 if f64 else _lib.MQP_F32
            it.ndims = nd
            for d in range(3):
                it.dims[d] = int(img1.shape[d]) if d < nd else 1
            it.params = params.to_c()
            it.VF = VF.data_ptr()
            it.SN = SN.data_ptr() if SN is not None else None
        opt = _lib.MqpBatchOptions()
        opt.use_graph = 1
        opt.grab = 2
        for k, v in (options or {}).items():
            setattr(opt, k, int(v))
        self.options = {"use_graph": opt.use_graph, "grab": opt.grab, "chunk3d": opt.chunk3d,
                        "chunk3d_budget": opt.chunk3d_budget}
        torch.cuda.synchronize(dev)  # the inputs are on the device before the plan reads their addresses
        h = C.c_void_p()
        _lib.check(self.ctx.lib.mqp_batch_plan_create(self.ctx.handle, items, len(pairs), C.byref(opt), C.byref(h)),
                   self.ctx.handle)
        self.handle = h
        self.device = dev

    def run(self, stream=None):
        """Enqueue one run on `stream` (a torch.cuda.Stream; default: current)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        _lib.check(self.ctx.lib.mqp_batch_plan_run(self.handle, C.c_void_p(s.cuda_stream)), self.ctx.handle)

    def results(self) -> List[tuple]:
        """[(VF, SN)] per pair: torch CUDA tensors shaped like PIV's outputs."""
        return self.outputs

    def info(self) -> dict:
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        _lib.check(self.ctx.lib.mqp_batch_plan_info(self.handle, C.byref(a), C.byref(b), C.byref(c)), self.ctx.handle)
        return {"total_ia": a.value, "launches": b.value, "scratch_bytes": c.value}

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.mqp_batch_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def PIV_batch(pairs: Sequence[tuple], options: Optional[dict] = None, context=None):
    """One run of a batch plan; returns [(VF, SN)] as NumPy arrays."""
    import torch
    plan = BatchPlan(pairs, options, context)
    plan.run()
    torch.cuda.synchronize(plan.device)
    out = [(VF.cpu().numpy(), SN.cpu().numpy() if SN is not None else None) for VF, SN in plan.results()]
    plan.close()
    return out
