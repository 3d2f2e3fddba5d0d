"""Host mirror of the reference's GpuBroadPhase (src/backend/webgpu/gpu-broadphase.ts:147-386)
over the device LBVH (include/closim_broadphase.h).

    bp = GpuBroadPhase(indices=idx, triCount=m, pad=0.002, pairCapacity=16384)
    res = bp.build(x0, x1)          # x0, x1: torch CUDA float64 tensors [3n]
    res["pairs"]                    # int32 [k, 2], sorted, a < b
    res["diagnostics"]              # scannedCount, writtenCount, candidateOverflow, capacity, detail
    bp.lastMirror                   # GpuBroadPhaseMirrorState as numpy arrays

mode "mirror" returns the FP32 mirror's set (the reference GpuBroadPhase);
mode "exact" returns the CPU TriBvh set (src/collision/bvh.ts:79-124), the
set the FP64 contact path uses.
"""
import ctypes as C

import numpy as np

from . import _lib

MODES = {"mirror": _lib.CS_BROADPHASE_MIRROR, "exact": _lib.CS_BROADPHASE_EXACT}


class GpuBroadPhase:
    name = "GpuBroadPhase"

    def __init__(self, indices, triCount, pad, pairCapacity=16384, mode="mirror", n=None):
        if triCount >= 1000003:
            # gpu-broadphase.ts:160-166
            raise ValueError(f"exclusion key decode needs triCount < 1000003, got {triCount}")
        self.indices = np.ascontiguousarray(indices, np.uint32)
        self.triCount = int(triCount)
        self.pad = float(pad)
        self.pairCapacity = int(pairCapacity)
        self.mode = mode
        nv = int(n) if n is not None else (int(self.indices.max()) + 1 if len(self.indices) else 0)
        self.n = nv
        L = _lib.load()
        self._h = L.cs_broadphase_create(nv, self.triCount, _lib.ptr(self.indices), self.pad, self.pairCapacity,
                                         MODES[mode])
        if not self._h:
            raise ValueError("cs_broadphase_create rejected the mesh or ran out of device memory")
        self.lastMirror = None

    def _check(self, rc):
        if rc != _lib.CS_OK:
            msg = _lib.load().cs_broadphase_last_error(self._h).decode()
            raise RuntimeError(f"broadphase error {rc}: {msg}")

    def build(self, x0, x1):
        """Candidate triangle pairs of the swept segment x0 -> x1 (device f64 tensors)."""
        import torch
        for x in (x0, x1):
            if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float64 and x.is_contiguous()):
                raise TypeError("positions must be contiguous CUDA float64 tensors (already resident on the device)")
            if x.numel() != 3 * self.n:
                raise ValueError("positions must hold 3n values")
        torch.cuda.synchronize(x0.device)
        L = _lib.load()
        self._check(L.cs_broadphase_build(self._h, C.c_void_p(x0.data_ptr()), C.c_void_p(x1.data_ptr())))
        d = _lib.cs_broadphase_diag()
        self._check(L.cs_broadphase_diagnostics(self._h, C.byref(d)))
        pairs = np.zeros((max(d.written_count, 1), 2), np.int32)
        self._check(L.cs_broadphase_pairs(self._h, _lib.ptr(pairs)))
        pairs = pairs[: d.written_count]
        m = self.triCount
        nc = max(1, 2 * m - 1)
        st = dict(aabb=np.zeros(m * 6, np.float32), centroid=np.zeros(m * 3, np.float32),
                  morton=np.zeros(m, np.uint32), payload=np.zeros(m, np.uint32),
                  nodeMin=np.zeros(nc * 3, np.float32), nodeMax=np.zeros(nc * 3, np.float32),
                  nodeLeft=np.zeros(nc, np.int32), nodeRight=np.zeros(nc, np.int32),
                  nodeLeafTri=np.zeros(nc, np.int32))
        self._check(L.cs_broadphase_state(self._h, *[_lib.ptr(st[k]) for k in [
            "aabb", "centroid", "morton", "payload", "nodeMin", "nodeMax", "nodeLeft", "nodeRight", "nodeLeafTri"]]))
        st.update(root=d.root, depth=d.tree_depth)
        self.lastMirror = st
        return {"pairs": pairs,
                "diagnostics": {"scannedCount": d.scanned_count, "writtenCount": d.written_count,
                                "candidateOverflow": d.candidate_overflow, "capacity": d.capacity,
                                "detail": {"treeDepth": d.tree_depth, "mortonSorted": True}}}

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().cs_broadphase_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
