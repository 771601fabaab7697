"""ctypes binding of libseevr_cuda.so (include/seevr.h, include/seevr_scene.h).

The library is built in-tree by ``python seevr_b200/build.py``.  There is no
fallback: importing this module without the built library raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libseevr_cuda.so"

NUM_BINDINGS = 31
NUM_STAGES = 9
STAGE_NAMES = (  # physics.zig:22-32
    "phys/gravity", "phys/aabb", "phys/broad_phase", "phys/narrow_phase",
    "phys/clear_impulse", "phys/pgs_solve", "phys/integrate", "phys/render_verts",
    "phys/clear_counters",
)

# seevr_status
OK, ERR_INVALID_ARGUMENT, ERR_CAPACITY, ERR_CUDA, ERR_TIMEOUT, ERR_NO_DEVICE, \
    ERR_OUT_OF_MEMORY, ERR_NOT_SUPPORTED = range(8)

BROADPHASE_N2, BROADPHASE_LBVH = 0, 1
NARROWPHASE_MPR, NARROWPHASE_GJK_EPA = 0, 1
SOLVER_SEQUENTIAL, SOLVER_WAVEFRONT, SOLVER_COLORED = 0, 1, 2
FLAG_NO_SYNC, FLAG_CUDA_GRAPH, FLAG_SKIP_RENDER_VERTS = 1, 2, 4
# bits of seevr_physics_read_flags
DEVICE_FLAG_PAIR_OVERFLOW, DEVICE_FLAG_CONTACT_OVERFLOW, DEVICE_FLAG_TIMEOUT, \
    DEVICE_FLAG_SOLVER_GLOBAL, DEVICE_FLAG_CHECK_FAILED, DEVICE_FLAG_GIANT_ISLANDS = \
    1, 2, 4, 8, 16, 32

# binding indices (physics.comp:16-57 + extension 30)
(B_BODY_POS, B_BODY_QUAT, B_BODY_VEL, B_BODY_OMEGA, B_BODY_INV_MASS, B_BODY_INV_INERTIA,
 B_BODY_VERT_START, B_BODY_VERT_COUNT, B_GEOM_BODY_IDX, B_GEOM_DATA, B_GEOM_FRICTION,
 B_GEOM_RESTITUTION, B_HULL_VERTS, B_VERTICES, B_ORIG_VERTICES, B_CONTACT_POS,
 B_CONTACT_NORMAL, B_CONTACT_PEN, B_CONTACT_GEOM_A, B_CONTACT_GEOM_B, B_LAMBDA_N,
 B_COUNTERS, B_BODY_AABB_MIN, B_BODY_AABB_MAX, B_COLLISION_PAIRS, B_AABB_TEMP_MIN,
 B_AABB_TEMP_MAX, B_AABB_TEMP_BODY, B_SUPPORT_OFFSET, B_SUPPORT_LOOKUP,
 B_HULL_RANGE) = range(31)


class Bindings(C.Structure):
    _fields_ = [("ptr", C.c_void_p * NUM_BINDINGS), ("bytes", C.c_uint64 * NUM_BINDINGS)]


class Caps(C.Structure):
    _fields_ = [("max_bodies", C.c_uint32), ("max_hull_verts", C.c_uint32),
                ("max_vertices", C.c_uint32), ("max_pairs", C.c_uint32),
                ("max_contacts", C.c_uint32), ("max_scenes", C.c_uint32)]


class Params(C.Structure):
    _fields_ = [("pgs_iterations", C.c_uint32), ("baumgarte", C.c_float), ("slop", C.c_float),
                ("linear_damping", C.c_float), ("angular_damping", C.c_float),
                ("mpr_eps", C.c_float), ("mpr_tolerance", C.c_float),
                ("mpr_iterations", C.c_uint32), ("mpr_discover_trials", C.c_uint32),
                ("broadphase", C.c_uint32), ("solver", C.c_uint32), ("flags", C.c_uint32),
                ("bundle_bodies", C.c_uint32), ("narrowphase", C.c_uint32)]


BVH_NUM_BINDINGS = 18
(BVH_VERTICES, BVH_INDICES, BVH_CENTROIDS, BVH_MORTON, BVH_MORTON_TEMP, BVH_SORT_INDICES,
 BVH_SORT_TEMP, BVH_SCENE_BOUNDS, BVH_NODE_MIN, BVH_NODE_MAX, BVH_LEFT, BVH_RIGHT, BVH_COUNT,
 BVH_PARENT, BVH_PRIM_INDICES, BVH_FLAGS, BVH_TEMP, BVH_TEMP_U) = range(18)


class BvhBindings(C.Structure):
    _fields_ = [("ptr", C.c_void_p * BVH_NUM_BINDINGS), ("bytes", C.c_uint64 * BVH_NUM_BINDINGS)]


class Profile(C.Structure):
    _fields_ = [("ms", C.c_float * NUM_STAGES), ("calls", C.c_uint32)]


class Tuning(C.Structure):
    """seevr_tuning: launch shapes of the batched step (results unchanged)."""
    _fields_ = [("bundle_bodies", C.c_uint32), ("narrow_blocks_per_sm", C.c_uint32),
                ("broad_tile_rows", C.c_uint32), ("scene_groups", C.c_uint32),
                ("giant_island_contacts", C.c_uint32)]


class AdjointGrads(C.Structure):
    """seevr_adjoint_grads: device pointers of the gradient buffers."""
    _fields_ = [("pos", C.c_void_p), ("quat", C.c_void_p), ("vel", C.c_void_p),
                ("omega", C.c_void_p), ("friction", C.c_void_p)]


class RtBindings(C.Structure):
    """seevr_rt_bindings: the 16 device pointers of raytrace.comp."""
    _fields_ = [("ptr", C.c_void_p * 16)]


class RtParams(C.Structure):
    """seevr_rt_params: raytrace.comp's push constants."""
    _fields_ = [("cam_pos", C.c_float * 3), ("cam_dir", C.c_float * 3),
                ("cam_right", C.c_float * 3), ("cam_up", C.c_float * 3),
                ("width", C.c_uint32), ("height", C.c_uint32), ("frame_num", C.c_uint32),
                ("num_triangles", C.c_uint32)]


class HostState(C.Structure):
    """seevr_host_state: host arrays copied in before and out after a frame."""
    _fields_ = [(n, C.c_void_p) for n in ("pos_in", "quat_in", "vel_in", "omega_in",
                                          "pos_out", "quat_out", "vel_out", "omega_out")]


class SeevrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"seevr status {status}: {message}")
        self.status = status


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run `python seevr_b200/build.py`")
    lib = C.CDLL(str(LIB_PATH))
    P, U32, U64, F, I = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.c_int
    FP = C.POINTER(C.c_float)
    UP = C.POINTER(C.c_uint32)
    sig = {
        "seevr_params_default": (None, [C.POINTER(Params)]),
        "seevr_physics_create": (I, [C.POINTER(Bindings), C.POINTER(Caps), C.POINTER(Params),
                                     C.POINTER(P)]),
        "seevr_physics_set_scenes": (I, [P, UP, U32]),
        "seevr_physics_step": (I, [P, U32, U32, U32, U32, F, FP, C.POINTER(Profile)]),
        "seevr_physics_step_async": (I, [P, U32, U32, U32, U32, F, FP, U32, P]),
        "seevr_physics_read_counters": (I, [P, UP]),
        "seevr_physics_read_flags": (I, [P, UP]),
        "seevr_physics_get_tuning": (I, [P, C.POINTER(Tuning)]),
        "seevr_physics_set_tuning": (I, [P, C.POINTER(Tuning)]),
        "seevr_physics_set_wait_limit": (I, [P, U32]),
        "seevr_physics_upload_state": (I, [P, U32, P, P, P, P]),
        "seevr_physics_download_state": (I, [P, U32, P, P, P, P]),
        "seevr_physics_step_io": (I, [P, U32, U32, U32, U32, F, FP, C.POINTER(HostState), P]),
        "seevr_physics_destroy": (None, [P]),
        "seevr_physics_kernel_launches": (U64, [P]),
        "seevr_physics_read_lbvh": (I, [P, U32, UP, UP, FP]),
        "seevr_physics_adjoint_substep": (I, [P, U32, U32, F, FP, C.POINTER(AdjointGrads)]),
        "seevr_raytrace": (I, [C.POINTER(RtBindings), C.POINTER(RtParams), P]),
        "seevr_raytrace_fov_scale": (F, []),
        "seevr_physics_step_noalloc": (I, [C.POINTER(Bindings), C.POINTER(Params), U32, U32,
                                           U32, U32, U32, U32, F, FP, P]),
        "seevr_physics_noalloc_flags": (U32, []),
        "seevr_bvh_create": (I, [C.POINTER(BvhBindings), U32, C.POINTER(P)]),
        "seevr_bvh_build": (I, [P, U32]),
        "seevr_bvh_destroy": (None, [P]),
        "seevr_status_string": (C.c_char_p, [I]),
        "seevr_last_error": (C.c_char_p, []),
        "seevr_abi_version": (I, []),
        # scene builder
        "seevr_scene_create": (P, []),
        "seevr_scene_destroy": (None, [P]),
        "seevr_scene_begin": (None, [P]),
        "seevr_scene_add_material": (U32, [P, FP, F, F, FP, F, F]),
        "seevr_scene_add_box": (U32, [P, FP, FP, FP, F, F, U32]),
        "seevr_scene_add_sphere": (U32, [P, FP, F, FP, U32, F, F, U32]),
        "seevr_scene_add_hull": (U32, [P, FP, FP, U32, FP, F, F, U32]),
        "seevr_scene_set_body_quat": (None, [P, U32, FP]),
        "seevr_scene_set_body_vel": (None, [P, U32, FP, FP]),
        "seevr_scene_set_geom_friction": (None, [P, U32, F]),
        "seevr_scene_gen_pile": (None, [P, U64, U32, U32, U32]),
        "seevr_scene_gen_pile_in": (None, [P, U64, U32, U32, U32, FP, FP]),
        "seevr_scene_gen_large": (None, [P, U64, U32, U32]),
        "seevr_scene_gen_batch": (None, [P, U32, U32, U32, U32, U64]),
        "seevr_scene_gen_rollout": (None, [P, U32, U32, U32, U64]),
        "seevr_scene_gen_towers": (None, [P, U64, U32, U32, F]),
        "seevr_scene_gen_towers_stacked": (None, [P, U64, U32, U32, F, F]),
        "seevr_scene_gen_batch_seeds": (None, [P, C.POINTER(C.c_uint64), U32, U32, U32, U32]),
        "seevr_scene_array": (P, [P, I]),
        "seevr_scene_count": (U64, [P, I]),
        "seevr_scene_save": (I, [P, C.c_char_p]),
        "seevr_scene_load": (P, [C.c_char_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != OK:
        msg = lib.seevr_last_error().decode(errors="replace")
        raise SeevrError(status, msg or lib.seevr_status_string(status).decode())


def default_params() -> Params:
    p = Params()
    lib.seevr_params_default(C.byref(p))
    return p


def fptr(values, n: int):
    """ctypes float[n] from a sequence."""
    arr = (C.c_float * n)(*[float(v) for v in values])
    return arr
