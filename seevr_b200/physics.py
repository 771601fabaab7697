"""Physics: the host interface of seeVR's physics step (src/physics.zig) over
libseevr_cuda.

    buf = Data.pile(seed=0).upload("cuda:0")
    ph = Physics(buf)                                    # Physics.init
    ph.step(buf.num_bodies, buf.num_vertices, buf.num_hull_verts,
            10, 1/60, (0, -9.81, 0))                     # Physics.step
    pairs, contacts = ph.read_counters()                 # Physics.readCounters
    ph.deinit()                                          # Physics.deinit

Errors raise SeevrError (the C ABI's status and message).  A capacity
overflow raises SeevrError with status ERR_CAPACITY after the step has run
(the first max_pairs / max_contacts in canonical order were kept).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .data import DeviceBuffers


def make_params(pgs_iterations: int = 4, solver: int = L.SOLVER_WAVEFRONT,
                broadphase: int = L.BROADPHASE_N2, flags: int = 0, **kw) -> L.Params:
    p = L.default_params()
    p.pgs_iterations = pgs_iterations
    p.solver = solver
    p.broadphase = broadphase
    p.flags = flags
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Physics:
    """One libseevr_cuda handle bound to a DeviceBuffers (Physics.init)."""

    def __init__(self, buffers: DeviceBuffers, params: L.Params | None = None,
                 use_hull_range: bool = True, scenes: bool = True):
        import torch

        self.buffers = buffers
        self.params = params or make_params()
        self._bind = buffers.bindings(use_hull_range=use_hull_range)
        self._caps = buffers.caps.to_c()
        h = C.c_void_p()
        with torch.cuda.device(buffers.device):
            L.check(L.lib.seevr_physics_create(C.byref(self._bind), C.byref(self._caps),
                                               C.byref(self.params), C.byref(h)))
        self._h = h
        if scenes and buffers.num_scenes > 1:
            off = np.ascontiguousarray(buffers.scene_body_offset, dtype=np.uint32)
            L.check(L.lib.seevr_physics_set_scenes(
                self._h, off.ctypes.data_as(C.POINTER(C.c_uint32)), buffers.num_scenes))

    def step(self, num_bodies: int, num_vertices: int, num_hull_verts: int, substeps: int,
             dt: float, gravity=(0.0, -9.81, 0.0), prof: L.Profile | None = None) -> None:
        """Physics.step (physics.zig:80): synchronous unless FLAG_NO_SYNC."""
        L.check(L.lib.seevr_physics_step(self._h, num_bodies, num_vertices, num_hull_verts,
                                         substeps, dt, L.fptr(gravity, 3),
                                         C.byref(prof) if prof is not None else None))

    def step_async(self, num_bodies: int, num_vertices: int, num_hull_verts: int, substeps: int,
                   dt: float, gravity=(0.0, -9.81, 0.0), frames: int = 1, stream=None) -> None:
        """`frames` steps ordered on `stream` (torch.cuda.Stream or raw handle;
        None: the handle's own stream)."""
        s = getattr(stream, "cuda_stream", stream)
        if stream is not None and not s:
            s = 1  # torch's default stream is CUDA's legacy default stream (cudaStreamLegacy)
        L.check(L.lib.seevr_physics_step_async(self._h, num_bodies, num_vertices, num_hull_verts,
                                               substeps, dt, L.fptr(gravity, 3), frames,
                                               C.c_void_p(s) if s else None))

    def read_counters(self) -> tuple[int, int]:
        """Physics.readCounters (physics.zig:213): (pairs, contacts) of the last substep."""
        out = (C.c_uint32 * 2)()
        L.check(L.lib.seevr_physics_read_counters(self._h, out))
        return int(out[0]), int(out[1])

    def read_flags(self) -> int:
        f = C.c_uint32()
        L.check(L.lib.seevr_physics_read_flags(self._h, C.byref(f)))
        return int(f.value)

    def get_tuning(self) -> dict:
        """The launch shapes in use (seevr_physics_get_tuning)."""
        t = L.Tuning()
        L.check(L.lib.seevr_physics_get_tuning(self._h, C.byref(t)))
        return {"bundle_bodies": t.bundle_bodies, "narrow_blocks_per_sm": t.narrow_blocks_per_sm,
                "broad_tile_rows": t.broad_tile_rows, "scene_groups": t.scene_groups,
                "giant_island_contacts": t.giant_island_contacts}

    def set_tuning(self, bundle_bodies: int = 0, narrow_blocks_per_sm: int = 0,
                   broad_tile_rows: int = 0, scene_groups: int = 0,
                   giant_island_contacts: int = 0) -> None:
        """seevr_physics_set_tuning (0 = default): launch shapes that change
        speed only, and the coloured mode's grid-wide island threshold."""
        t = L.Tuning(bundle_bodies, narrow_blocks_per_sm, broad_tile_rows, scene_groups,
                     giant_island_contacts)
        L.check(L.lib.seevr_physics_set_tuning(self._h, C.byref(t)))

    def set_wait_limit(self, polls: int) -> None:
        """seevr_physics_set_wait_limit: polls of an unpublished tile before a
        device-side look-back gives up (the step then reports ERR_TIMEOUT)."""
        L.check(L.lib.seevr_physics_set_wait_limit(self._h, polls))

    def upload_state(self, num_bodies: int, pos=None, quat=None, vel=None, omega=None) -> None:
        ptr = lambda a: None if a is None else C.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())
        L.check(L.lib.seevr_physics_upload_state(self._h, num_bodies, ptr(pos), ptr(quat),
                                                 ptr(vel), ptr(omega)))

    def download_state(self, num_bodies: int, pos=None, quat=None, vel=None, omega=None) -> None:
        ptr = lambda a: None if a is None else C.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())
        L.check(L.lib.seevr_physics_download_state(self._h, num_bodies, ptr(pos), ptr(quat),
                                                   ptr(vel), ptr(omega)))

    def step_io(self, num_bodies: int, num_vertices: int, num_hull_verts: int, substeps: int,
                dt: float, gravity=(0.0, -9.81, 0.0), inputs=None, outputs=None, stream=None,
                sync: bool = True) -> None:
        """seevr_physics_step_io: one frame with the state copied in from the
        host arrays `inputs` and out to `outputs` (dicts of pos, quat, vel,
        omega: numpy arrays or CPU tensors; a missing key skips that copy).
        Page-locked arrays (torch's pin_memory) are copied per scene group
        beside the other groups' kernels.  Ordered on `stream` (None: torch's
        current stream); sync=True waits for it before returning, so the
        outputs are ready."""
        import torch

        if stream is None:
            stream = torch.cuda.current_stream()
        ptr = lambda a: None if a is None else (a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())
        i, o = inputs or {}, outputs or {}
        io = L.HostState(*[ptr(i.get(k)) for k in ("pos", "quat", "vel", "omega")],
                         *[ptr(o.get(k)) for k in ("pos", "quat", "vel", "omega")])
        s = getattr(stream, "cuda_stream", stream)
        if stream is not None and not s:
            s = 1  # torch's default stream is CUDA's legacy default stream (cudaStreamLegacy)
        L.check(L.lib.seevr_physics_step_io(self._h, num_bodies, num_vertices, num_hull_verts,
                                            substeps, dt, L.fptr(gravity, 3), C.byref(io),
                                            C.c_void_p(s) if s else None))
        if sync:
            if not hasattr(stream, "synchronize"):
                stream = torch.cuda.ExternalStream(s)
            stream.synchronize()

    def read_lbvh(self, n: int):
        """Sorted Morton codes, body order and centroid bounds of the last
        LBVH build (broadphase=BROADPHASE_LBVH handles)."""
        codes = np.zeros(n, np.uint32)
        order = np.zeros(n, np.uint32)
        bounds = np.zeros(6, np.float32)
        U = C.POINTER(C.c_uint32)
        L.check(L.lib.seevr_physics_read_lbvh(self._h, n, codes.ctypes.data_as(U),
                                              order.ctypes.data_as(U),
                                              bounds.ctypes.data_as(C.POINTER(C.c_float))))
        return codes, order, bounds

    @property
    def kernel_launches(self) -> int:
        return int(L.lib.seevr_physics_kernel_launches(self._h))

    def deinit(self) -> None:
        """Physics.deinit (physics.zig:219)."""
        if getattr(self, "_h", None):
            L.lib.seevr_physics_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.deinit()
        except Exception:
            pass
