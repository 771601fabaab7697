"""BVH: the triangle LBVH build of seeVR's raytrace mode (src/bvh.zig) over
libseevr_cuda.

    bvh = BVH(vertices, indices)        # BVH.init: device tensors, 18 buffers
    bvh.build(num_tris)                 # BVH.build
    bvh["node_min"], bvh["left"], ...   # the buffers bvh.comp writes
    bvh.deinit()                        # BVH.deinit
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L

_NAMES = ("vertices", "indices", "centroids", "morton", "morton_temp", "sort_indices",
          "sort_temp", "scene_bounds", "node_min", "node_max", "left", "right", "count",
          "parent", "prim_indices", "flags", "temp", "temp_u")


class BVH:
    def __init__(self, vertices, indices, max_tris: int | None = None):
        import torch

        dev = vertices.device
        t = max_tris if max_tris is not None else indices.numel() // 3
        nodes = max(2 * t - 1, 1)
        f32, i32 = torch.float32, torch.int32
        z = lambda n, dt: torch.zeros(max(n, 1), dtype=dt, device=dev)
        self.t = {
            "vertices": vertices.contiguous().view(-1).to(f32),
            "indices": indices.contiguous().view(-1).to(i32),
            "centroids": z(3 * t, f32), "morton": z(t, i32), "morton_temp": z(t, i32),
            "sort_indices": z(t, i32), "sort_temp": z(t, i32), "scene_bounds": z(6, f32),
            "node_min": z(3 * nodes, f32), "node_max": z(3 * nodes, f32), "left": z(nodes, i32),
            "right": z(nodes, i32), "count": z(nodes, i32), "parent": z(nodes, i32),
            "prim_indices": z(t, i32), "flags": z(t, i32), "temp": z(1, f32),
            "temp_u": z(8 + 1024 + 1 + ((t + 2047) // 2048) * 256, i32),
        }
        self._b = L.BvhBindings()
        for i, name in enumerate(_NAMES):
            ten = self.t[name]
            self._b.ptr[i] = ten.data_ptr()
            self._b.bytes[i] = ten.numel() * ten.element_size()
        h = C.c_void_p()
        with torch.cuda.device(dev):
            L.check(L.lib.seevr_bvh_create(C.byref(self._b), t, C.byref(h)))
        self._h = h

    def build(self, num_tris: int) -> None:
        """BVH.build (bvh.zig:63): synchronous."""
        L.check(L.lib.seevr_bvh_build(self._h, num_tris))

    def __getitem__(self, name):
        return self.t[name]

    def deinit(self) -> None:
        if getattr(self, "_h", None):
            L.lib.seevr_bvh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.deinit()
        except Exception:
            pass
