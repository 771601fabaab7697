"""Scene data: the CPU staging arrays of seeVR's Data (src/data.zig) and their
upload into device buffers laid out as the physics.comp bindings.

    d = Data()
    m = d.add_material((.8, .2, .2), .4, 0, (0, 0, 0), 0, 1000)   # Data.addMaterial
    d.add_box((0, 1, 0), (.5, .5, .5), (1, 0, 0), .5, 0, m)       # Data.addBox
    d.add_sphere((1, 3, 0), .4, (1, 1, 1), 16, .2, .37, m)         # Data.addSphere
    buf = d.upload("cuda:0")                                       # Data.upload

Seeded workloads: Data.pile, Data.large, Data.batch, Data.rollout,
Data.towers (one splitmix64 stream per scene; see include/seevr_scene.h).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

# seevr_scene_array ids -> (dtype, components, count id)
_S_BODY, _S_GEOM, _S_HULL, _S_VERT, _S_TRI, _S_SUP, _S_SCN, _S_MAT = 0, 1, 2, 3, 4, 5, 6, 7
_ARRAYS = {
    "body_pos": (0, np.float32, 3, _S_BODY),
    "body_quat": (1, np.float32, 4, _S_BODY),
    "body_vel": (2, np.float32, 3, _S_BODY),
    "body_omega": (3, np.float32, 3, _S_BODY),
    "body_inv_mass": (4, np.float32, 1, _S_BODY),
    "body_inv_inertia": (5, np.float32, 3, _S_BODY),
    "body_vert_start": (6, np.uint32, 1, _S_BODY),
    "body_vert_count": (7, np.uint32, 1, _S_BODY),
    "geom_body_idx": (8, np.uint32, 1, _S_GEOM),
    "geom_data": (9, np.float32, 8, _S_GEOM),
    "geom_friction": (10, np.float32, 1, _S_GEOM),
    "geom_restitution": (11, np.float32, 1, _S_GEOM),
    "hull_verts": (12, np.float32, 3, _S_HULL),
    "vertices": (13, np.float32, 3, _S_VERT),
    "orig_vertices": (14, np.float32, 3, _S_VERT),
    "support_offset": (15, np.uint32, 1, _S_GEOM),
    "support_lookup": (16, np.uint32, 1, _S_SUP),
    "indices": (17, np.uint32, 3, _S_TRI),
    "body_inertia": (18, np.float32, 3, _S_BODY),
    "geom_type": (19, np.int32, 1, _S_GEOM),
    "scene_body_offset": (20, np.uint32, 1, None),
    "colors": (21, np.float32, 3, _S_VERT),
    "hull_range": (22, np.uint32, 2, _S_GEOM),
    "geom_material": (23, np.uint32, 1, _S_GEOM),
    "tri_geom": (24, np.uint32, 1, _S_TRI),
    "mat_albedo": (25, np.float32, 3, _S_MAT),
    "mat_roughness": (26, np.float32, 1, _S_MAT),
    "mat_metallic": (27, np.float32, 1, _S_MAT),
    "mat_emission": (28, np.float32, 3, _S_MAT),
    "mat_ior": (29, np.float32, 1, _S_MAT),
}

# host array name -> binding index
_BINDING_OF = {
    "body_pos": L.B_BODY_POS, "body_quat": L.B_BODY_QUAT, "body_vel": L.B_BODY_VEL,
    "body_omega": L.B_BODY_OMEGA, "body_inv_mass": L.B_BODY_INV_MASS,
    "body_inv_inertia": L.B_BODY_INV_INERTIA, "body_vert_start": L.B_BODY_VERT_START,
    "body_vert_count": L.B_BODY_VERT_COUNT, "geom_body_idx": L.B_GEOM_BODY_IDX,
    "geom_data": L.B_GEOM_DATA, "geom_friction": L.B_GEOM_FRICTION,
    "geom_restitution": L.B_GEOM_RESTITUTION, "hull_verts": L.B_HULL_VERTS,
    "vertices": L.B_VERTICES, "orig_vertices": L.B_ORIG_VERTICES,
    "support_offset": L.B_SUPPORT_OFFSET, "support_lookup": L.B_SUPPORT_LOOKUP,
    "hull_range": L.B_HULL_RANGE,
}


def _f3(v):
    return L.fptr(v, 3)


class Data:
    """CPU staging arrays of one or more independent scenes (data.zig:31-177)."""

    def __init__(self, _handle=None):
        self._h = _handle if _handle is not None else L.lib.seevr_scene_create()
        if not self._h:
            raise MemoryError("seevr_scene_create failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(L, "lib", None)  # None while the interpreter shuts down
        if h and lib is not None:
            lib.seevr_scene_destroy(h)
            self._h = None

    # ---- builders (data.zig) ----
    def begin_scene(self) -> None:
        L.lib.seevr_scene_begin(self._h)

    def add_material(self, albedo, roughness, metallic, emission, ior, density) -> int:
        return L.lib.seevr_scene_add_material(self._h, _f3(albedo), roughness, metallic,
                                              _f3(emission), ior, density)

    def add_box(self, center, half, color, friction, restitution, material) -> int:
        return L.lib.seevr_scene_add_box(self._h, _f3(center), _f3(half), _f3(color), friction,
                                         restitution, material)

    def add_sphere(self, center, radius, color, segments, friction, restitution, material) -> int:
        return L.lib.seevr_scene_add_sphere(self._h, _f3(center), radius, _f3(color), segments,
                                            friction, restitution, material)

    def add_hull(self, center, points, color, friction, restitution, material) -> int:
        pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        return L.lib.seevr_scene_add_hull(self._h, _f3(center),
                                          pts.ctypes.data_as(C.POINTER(C.c_float)), len(pts),
                                          _f3(color), friction, restitution, material)

    def set_body_quat(self, body: int, q) -> None:
        L.lib.seevr_scene_set_body_quat(self._h, body, L.fptr(q, 4))

    def set_body_vel(self, body: int, v=None, w=None) -> None:
        L.lib.seevr_scene_set_body_vel(self._h, body, _f3(v) if v is not None else None,
                                       _f3(w) if w is not None else None)

    # ---- seeded workloads ----
    @classmethod
    def pile(cls, seed=0, n_boxes=256, n_spheres=256, segments=16, lo=None, hi=None) -> "Data":
        """Ground box + bodies alternating box/sphere, spawned in x,z [-5,5],
        y [1,21] (or the box [lo, hi]) without initial overlaps."""
        d = cls()
        if lo is None and hi is None:
            L.lib.seevr_scene_gen_pile(d._h, seed, n_boxes, n_spheres, segments)
        else:
            L.lib.seevr_scene_gen_pile_in(d._h, seed, n_boxes, n_spheres, segments,
                                          _f3(lo), _f3(hi))
        return d

    @classmethod
    def large(cls, seed=0, n_bodies=32768, segments=16) -> "Data":
        d = cls()
        L.lib.seevr_scene_gen_large(d._h, seed, n_bodies, segments)
        return d

    @classmethod
    def batch(cls, num_scenes=4096, min_bodies=8, max_bodies=512, segments=16,
              seed_base=0) -> "Data":
        d = cls()
        L.lib.seevr_scene_gen_batch(d._h, num_scenes, min_bodies, max_bodies, segments, seed_base)
        return d

    @classmethod
    def batch_seeds(cls, seeds, min_bodies=8, max_bodies=512, segments=16) -> "Data":
        """The scenes of Data.batch(seed_base=0) whose numbers are listed, in
        the listed order (scene k is generated from seed k)."""
        d = cls()
        arr = np.ascontiguousarray(seeds, dtype=np.uint64)
        L.lib.seevr_scene_gen_batch_seeds(d._h, arr.ctypes.data_as(C.POINTER(C.c_uint64)),
                                          len(arr), min_bodies, max_bodies, segments)
        return d

    @classmethod
    def rollout(cls, num_scenes=1024, bodies=64, segments=16, seed_base=0) -> "Data":
        d = cls()
        L.lib.seevr_scene_gen_rollout(d._h, num_scenes, bodies, segments, seed_base)
        return d

    @classmethod
    def towers(cls, seed=0, towers=1024, height=256, spacing=2.0, overlap=0.0) -> "Data":
        """Stacks of unit boxes; each box sinks `overlap` m into the one below
        (0: boxes that just touch)."""
        d = cls()
        L.lib.seevr_scene_gen_towers_stacked(d._h, seed, towers, height, spacing, overlap)
        return d

    # ---- views ----
    def count(self, which: int) -> int:
        return int(L.lib.seevr_scene_count(self._h, which))

    num_bodies = property(lambda self: self.count(0))
    num_geoms = property(lambda self: self.count(1))
    num_hull_verts = property(lambda self: self.count(2))
    num_vertices = property(lambda self: self.count(3))
    num_triangles = property(lambda self: self.count(4))
    num_support_entries = property(lambda self: self.count(5))
    num_scenes = property(lambda self: self.count(6))
    num_materials = property(lambda self: self.count(7))
    num_dynamic = property(lambda self: self.count(8))
    placement_failures = property(lambda self: self.count(9))

    def array(self, name: str) -> np.ndarray:
        """A copy of one staging array, shaped (count, components)."""
        aid, dt, comp, cnt = _ARRAYS[name]
        n = self.num_scenes + 1 if cnt is None else self.count(cnt)
        ptr = L.lib.seevr_scene_array(self._h, aid)
        total = n * comp
        if total == 0 or not ptr:
            return np.zeros((0, comp) if comp > 1 else (0,), dtype=dt)
        ctype = {np.float32: C.c_float, np.uint32: C.c_uint32, np.int32: C.c_int32}[dt]
        a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(total,)).copy()
        return a.reshape(n, comp) if comp > 1 else a

    def arrays(self) -> dict:
        return {k: self.array(k) for k in _ARRAYS}

    def scene_body_offset(self) -> np.ndarray:
        return self.array("scene_body_offset")

    def save(self, path: str) -> None:
        if L.lib.seevr_scene_save(self._h, str(path).encode()) != 0:
            raise OSError(f"could not write {path}")

    @classmethod
    def load(cls, path: str) -> "Data":
        h = L.lib.seevr_scene_load(str(path).encode())
        if not h:
            raise OSError(f"could not read scene file {path}")
        return cls(h)

    # ---- upload (data.zig:599-655) ----
    def upload(self, device="cuda", caps: "Caps | None" = None) -> "DeviceBuffers":
        return DeviceBuffers.from_data(self, device, caps)


@dataclass
class Caps:
    """Capacities of one handle (data.zig:11-18 hard-codes the reference's)."""
    max_bodies: int
    max_hull_verts: int
    max_vertices: int
    max_pairs: int
    max_contacts: int
    max_scenes: int = 1

    @classmethod
    def for_data(cls, d: Data, pairs_per_body: float = 8.0, contacts_per_body: float = 4.0,
                 min_pairs: int = 10000, min_contacts: int = 4000) -> "Caps":
        nb = max(d.num_bodies, 1)
        return cls(max_bodies=nb, max_hull_verts=max(d.num_hull_verts, 1),
                   max_vertices=max(d.num_vertices, 1),
                   max_pairs=max(int(nb * pairs_per_body), min_pairs),
                   max_contacts=max(int(nb * contacts_per_body), min_contacts),
                   max_scenes=max(d.num_scenes, 1))

    def to_c(self) -> L.Caps:
        return L.Caps(self.max_bodies, self.max_hull_verts, self.max_vertices, self.max_pairs,
                      self.max_contacts, self.max_scenes)


@dataclass
class DeviceBuffers:
    """Device tensors for the 30 physics.comp bindings (+ hull-range extension)."""
    tensors: dict
    caps: Caps
    num_bodies: int
    num_vertices: int
    num_hull_verts: int
    num_scenes: int
    scene_body_offset: np.ndarray
    device: object = None
    extra: dict = field(default_factory=dict)

    @classmethod
    def from_data(cls, d: Data, device="cuda", caps: Caps | None = None) -> "DeviceBuffers":
        import torch

        caps = caps or Caps.for_data(d)
        dev = torch.device(device)
        host = d.arrays()
        t = {}

        def put(name, arr, n_elems, dtype):
            buf = torch.zeros(max(n_elems, 1), dtype=dtype, device=dev)
            flat = np.ascontiguousarray(arr).reshape(-1)
            if flat.size:
                buf[: flat.size].copy_(torch.from_numpy(flat.view(np.int32) if dtype == torch.int32
                                                        else flat))
            t[name] = buf

        f32, i32 = torch.float32, torch.int32
        nb, nhv, nv = caps.max_bodies, caps.max_hull_verts, caps.max_vertices
        for name, mult in (("body_pos", 3), ("body_quat", 4), ("body_vel", 3), ("body_omega", 3),
                           ("body_inv_mass", 1), ("body_inv_inertia", 3), ("geom_data", 8),
                           ("geom_friction", 1), ("geom_restitution", 1)):
            put(name, host[name], nb * mult, f32)
        for name, mult in (("body_vert_start", 1), ("body_vert_count", 1), ("geom_body_idx", 1),
                           ("support_offset", 1), ("hull_range", 2)):
            put(name, host[name], nb * mult, i32)
        put("hull_verts", host["hull_verts"], nhv * 3, f32)
        put("orig_vertices", host["orig_vertices"], nv * 3, f32)
        put("vertices", host["vertices"], nv * 3, f32)
        put("support_lookup", host["support_lookup"], max(len(host["support_lookup"]), 1), i32)
        mc, mp = caps.max_contacts, caps.max_pairs
        for name, n, dt in (("contact_pos", mc * 3, f32), ("contact_normal", mc * 3, f32),
                            ("contact_pen", mc, f32), ("contact_geom_a", mc, i32),
                            ("contact_geom_b", mc, i32), ("lambda_n", mc, f32),
                            ("counters", 4, i32), ("body_aabb_min", nb * 3, f32),
                            ("body_aabb_max", nb * 3, f32), ("collision_pairs", mp * 2, i32)):
            t[name] = torch.zeros(max(n, 1), dtype=dt, device=dev)
        return cls(tensors=t, caps=caps, num_bodies=d.num_bodies, num_vertices=d.num_vertices,
                   num_hull_verts=d.num_hull_verts, num_scenes=d.num_scenes,
                   scene_body_offset=d.scene_body_offset(), device=dev)

    _NAMES = {  # binding index -> tensor name
        L.B_BODY_POS: "body_pos", L.B_BODY_QUAT: "body_quat", L.B_BODY_VEL: "body_vel",
        L.B_BODY_OMEGA: "body_omega", L.B_BODY_INV_MASS: "body_inv_mass",
        L.B_BODY_INV_INERTIA: "body_inv_inertia", L.B_BODY_VERT_START: "body_vert_start",
        L.B_BODY_VERT_COUNT: "body_vert_count", L.B_GEOM_BODY_IDX: "geom_body_idx",
        L.B_GEOM_DATA: "geom_data", L.B_GEOM_FRICTION: "geom_friction",
        L.B_GEOM_RESTITUTION: "geom_restitution", L.B_HULL_VERTS: "hull_verts",
        L.B_VERTICES: "vertices", L.B_ORIG_VERTICES: "orig_vertices",
        L.B_CONTACT_POS: "contact_pos", L.B_CONTACT_NORMAL: "contact_normal",
        L.B_CONTACT_PEN: "contact_pen", L.B_CONTACT_GEOM_A: "contact_geom_a",
        L.B_CONTACT_GEOM_B: "contact_geom_b", L.B_LAMBDA_N: "lambda_n",
        L.B_COUNTERS: "counters", L.B_BODY_AABB_MIN: "body_aabb_min",
        L.B_BODY_AABB_MAX: "body_aabb_max", L.B_COLLISION_PAIRS: "collision_pairs",
        L.B_SUPPORT_OFFSET: "support_offset", L.B_SUPPORT_LOOKUP: "support_lookup",
        L.B_HULL_RANGE: "hull_range",
    }

    def bindings(self, use_hull_range: bool = True) -> L.Bindings:
        b = L.Bindings()
        for idx, name in self._NAMES.items():
            if idx == L.B_HULL_RANGE and not use_hull_range:
                continue
            ten = self.tensors[name]
            b.ptr[idx] = ten.data_ptr()
            b.bytes[idx] = ten.numel() * ten.element_size()
        return b

    def __getitem__(self, name):
        return self.tensors[name]
