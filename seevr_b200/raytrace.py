"""Raytracer: the path tracer of seeVR's raytrace mode (src/raytracer.zig,
src/shaders/raytrace.comp) over libseevr_cuda, writing a headless RGBA32F
image (a torch tensor of shape (height, width, 4)) instead of a Vulkan
storage image.

    d = Data.pile(seed=0)
    bvh = BVH(vertices, indices); bvh.build(num_tris)     # BVH.init / build
    rt = Raytracer(d, bvh, width=640, height=480)          # Raytracer.init
    img = rt.render(cam_pos, cam_dir, cam_right, cam_up, num_tris)   # render
    rt.reset_accumulation()                                # resetAccumulation
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class Raytracer:
    """Material and triangle-geom tables of a Data on the device, the BVH's
    node buffers, and the output image (Raytracer.init, raytracer.zig:29)."""

    def __init__(self, data, bvh, width: int, height: int):
        import torch

        dev = bvh["vertices"].device
        a = data.arrays()
        u32 = lambda k: torch.from_numpy(np.ascontiguousarray(a[k]).view(np.int32).reshape(-1)).to(dev)
        f32 = lambda k: torch.from_numpy(np.ascontiguousarray(a[k], dtype=np.float32).reshape(-1)).to(dev)
        self.width, self.height, self.frame = width, height, 0
        self.image = torch.zeros((height, width, 4), dtype=torch.float32, device=dev)
        self.t = {"tri_geom": u32("tri_geom"), "geom_material": u32("geom_material"),
                  "mat_albedo": f32("mat_albedo"), "mat_roughness": f32("mat_roughness"),
                  "mat_metallic": f32("mat_metallic"), "mat_emission": f32("mat_emission"),
                  "mat_ior": f32("mat_ior")}
        self.bvh = bvh
        b = L.RtBindings()
        order = [self.image, bvh["vertices"], bvh["indices"], bvh["node_min"], bvh["node_max"],
                 bvh["left"], bvh["right"], bvh["count"], bvh["prim_indices"],
                 self.t["tri_geom"], self.t["geom_material"], self.t["mat_albedo"],
                 self.t["mat_roughness"], self.t["mat_metallic"], self.t["mat_emission"],
                 self.t["mat_ior"]]
        for i, ten in enumerate(order):
            b.ptr[i] = ten.data_ptr()
        self._b = b

    def render(self, cam_pos, cam_dir, cam_right, cam_up, num_tris: int, stream=None):
        """Raytracer.render (raytracer.zig:159): one frame written to
        self.image; the frame number (the RNG seed) advances."""
        p = L.RtParams()
        p.cam_pos[:], p.cam_dir[:] = list(map(float, cam_pos)), list(map(float, cam_dir))
        p.cam_right[:], p.cam_up[:] = list(map(float, cam_right)), list(map(float, cam_up))
        p.width, p.height, p.frame_num, p.num_triangles = self.width, self.height, self.frame, num_tris
        s = getattr(stream, "cuda_stream", stream)
        L.check(L.lib.seevr_raytrace(C.byref(self._b), C.byref(p), C.c_void_p(s) if s else None))
        self.frame += 1
        return self.image

    def reset_accumulation(self) -> None:
        """Raytracer.resetAccumulation (raytracer.zig:202)."""
        self.frame = 0
