"""TEST INFRASTRUCTURE — ctypes wrapper of oracle/liboracle.so, the CPU
restatement of seeVR's physics.comp / bvh.comp (seevr_oracle.hpp).

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker.  Parity is unpinned against reference outputs (the
reference has no tests or fixtures and cannot run here); see the header of
seevr_oracle.hpp.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_f = C.POINTER(C.c_float)
_u = C.POINTER(C.c_uint32)
_d = C.POINTER(C.c_double)
_u64 = C.POINTER(C.c_uint64)


class OracleScene(C.Structure):
    _fields_ = [("num_bodies", C.c_uint32), ("num_geoms", C.c_uint32),
                ("num_hull_verts", C.c_uint32), ("num_vertices", C.c_uint32),
                ("num_scenes", C.c_uint32),
                ("body_pos", _f), ("body_quat", _f), ("body_vel", _f), ("body_omega", _f),
                ("body_inv_mass", _f), ("body_inv_inertia", _f),
                ("body_vert_start", _u), ("body_vert_count", _u), ("geom_body_idx", _u),
                ("geom_data", _f), ("geom_friction", _f), ("geom_restitution", _f),
                ("hull_verts", _f), ("orig_verts", _f),
                ("support_offset", _u), ("support_lookup", _u), ("scene_body_offset", _u),
                ("hull_range", _u)]


class OracleParams(C.Structure):
    _fields_ = [("pgs_iterations", C.c_uint32), ("baumgarte", C.c_float), ("slop", C.c_float),
                ("lin_damp", C.c_float), ("ang_damp", C.c_float), ("eps", C.c_float),
                ("tol", C.c_float), ("mpr_iterations", C.c_uint32),
                ("discover_trials", C.c_uint32), ("max_pairs", C.c_uint32),
                ("max_contacts", C.c_uint32), ("narrowphase", C.c_uint32)]


class OracleOut(C.Structure):
    _fields_ = [("pos", _d), ("quat", _d), ("vel", _d), ("omega", _d),
                ("aabb_min", _d), ("aabb_max", _d), ("verts", _d), ("pairs", _u),
                ("c_pos", _d), ("c_normal", _d), ("c_pen", _d), ("lambda_", _d),
                ("c_a", _u), ("c_b", _u), ("counters", C.c_uint32 * 2),
                ("ops", C.c_uint64 * 10)]


OP_NAMES = ("support_brute", "support_brute_verts", "support_lookup", "mpr_calls",
            "mpr_support_calls", "pgs_contact_iters", "pgs_friction_iters", "aabb_verts",
            "broad_tests", "body_substeps")


def _load():
    if not LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    lib = C.CDLL(str(LIB_PATH))
    lib.oracle_run.restype = C.c_int
    lib.oracle_run.argtypes = [C.POINTER(OracleScene), C.POINTER(OracleParams), C.c_int,
                               C.c_uint32, C.c_uint32, C.c_float, _f, C.c_int, C.c_int,
                               C.POINTER(OracleOut), _u64, C.c_int]
    lib.oracle_run_f64_state.restype = C.c_int
    lib.oracle_run_f64_state.argtypes = [C.POINTER(OracleScene), C.POINTER(OracleParams),
                                         C.c_uint32, C.c_uint32, C.c_float, _f, _d, _d, _d, _d,
                                         _d, C.c_int, C.POINTER(OracleOut), _u64, C.c_int]
    lib.oracle_raytrace.restype = None
    lib.oracle_raytrace.argtypes = [_f, _u, _f, _f, _u, _u, _u, _u, _u, _u, _f, _f, _f, _f, _f,
                                    _f, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_int,
                                    _f]
    lib.oracle_morton.argtypes = [_f, C.c_uint32, _u, _f]
    lib.oracle_radix_sort.argtypes = [_u, C.c_uint32, _u, _u]
    lib.oracle_karras.argtypes = [_u, C.c_uint32, _u, _u, _u]
    lib.oracle_angle_bin64f.restype = C.c_uint32
    lib.oracle_angle_bin64f.argtypes = [C.c_float, C.c_float]
    lib.oracle_num_threads.restype = C.c_int
    return lib


lib = _load()


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _scene(a: dict, update_verts: bool, use_hull_range: bool) -> OracleScene:
    nb = len(a["body_inv_mass"])
    ng = len(a["geom_body_idx"])
    nhv = len(a["hull_verts"])
    nv = len(a["orig_vertices"]) if update_verts else 0
    off = a.get("scene_body_offset")
    ns = len(off) - 1 if off is not None and len(off) > 1 else 1
    return OracleScene(nb, ng, nhv, nv, ns,
                       _p(a["body_pos"], _f), _p(a["body_quat"], _f), _p(a["body_vel"], _f),
                       _p(a["body_omega"], _f), _p(a["body_inv_mass"], _f),
                       _p(a["body_inv_inertia"], _f), _p(a["body_vert_start"], _u),
                       _p(a["body_vert_count"], _u), _p(a["geom_body_idx"], _u),
                       _p(a["geom_data"], _f), _p(a["geom_friction"], _f),
                       _p(a["geom_restitution"], _f), _p(a["hull_verts"], _f),
                       _p(a["orig_vertices"], _f) if nv else None,
                       _p(a["support_offset"], _u), _p(a["support_lookup"], _u),
                       _p(off, _u) if off is not None and len(off) > 1 else None,
                       _p(a["hull_range"], _u) if use_hull_range and "hull_range" in a else None)


def _params(pgs_iterations, max_pairs, max_contacts, consts) -> OracleParams:
    return OracleParams(pgs_iterations, consts.get("baumgarte", 0.2), consts.get("slop", 0.005),
                        consts.get("lin_damp", 0.999), consts.get("ang_damp", 0.998),
                        consts.get("eps", 1e-6), consts.get("tol", 1e-6),
                        consts.get("mpr_iterations", 50), consts.get("discover_trials", 15),
                        max_pairs, max_contacts, consts.get("narrowphase", 0))


def _outputs(nb: int, nv: int, max_pairs: int, max_contacts: int):
    out = {
        "pos": np.zeros((nb, 3)), "quat": np.zeros((nb, 4)), "vel": np.zeros((nb, 3)),
        "omega": np.zeros((nb, 3)), "aabb_min": np.zeros((nb, 3)), "aabb_max": np.zeros((nb, 3)),
        "verts": np.zeros((max(nv, 1), 3)), "pairs": np.zeros((max_pairs, 2), np.uint32),
        "c_pos": np.zeros((max_contacts, 3)), "c_normal": np.zeros((max_contacts, 3)),
        "c_pen": np.zeros(max_contacts), "lambda": np.zeros(max_contacts),
        "c_a": np.zeros(max_contacts, np.uint32), "c_b": np.zeros(max_contacts, np.uint32),
    }
    o = OracleOut(_p(out["pos"], _d), _p(out["quat"], _d), _p(out["vel"], _d),
                  _p(out["omega"], _d), _p(out["aabb_min"], _d), _p(out["aabb_max"], _d),
                  _p(out["verts"], _d), _p(out["pairs"], _u), _p(out["c_pos"], _d),
                  _p(out["c_normal"], _d), _p(out["c_pen"], _d), _p(out["lambda"], _d),
                  _p(out["c_a"], _u), _p(out["c_b"], _u))
    return out, o


def _finish(out: dict, o: OracleOut, nv: int, max_pairs: int, max_contacts: int) -> dict:
    npairs, ncont = int(o.counters[0]), int(o.counters[1])
    out["num_pairs"], out["num_contacts"] = npairs, ncont
    out["pairs"] = out["pairs"][: min(npairs, max_pairs)]
    for k in ("c_pos", "c_normal", "c_pen", "lambda", "c_a", "c_b"):
        out[k] = out[k][: min(ncont, max_contacts)]
    out["verts"] = out["verts"][:nv]
    out["ops"] = dict(zip(OP_NAMES, [int(x) for x in o.ops]))
    return out


LOCK_MODES = {None: 0, "record": 1, "replay": 2}


def _sig(a: dict, on: bool):
    """Per-scene branch-hash output array, or None."""
    if not on:
        return None
    off = a.get("scene_body_offset")
    ns = len(off) - 1 if off is not None and len(off) > 1 else 1
    return np.zeros(ns, np.uint64)


def _done(rc: int, name: str, out: dict, o, nv, max_pairs, max_contacts, sig) -> dict:
    if rc == 3:
        raise RuntimeError(f"{name}: the replayed run left its recorded branches")
    if rc != 0:
        raise RuntimeError(f"{name} failed ({rc})")
    out = _finish(out, o, nv, max_pairs, max_contacts)
    if sig is not None:
        out["branch_sig"] = sig
    return out


def run(arrays: dict, *, frames=1, substeps=10, dt=1.0 / 60.0, gravity=(0.0, -9.81, 0.0),
        pgs_iterations=4, max_pairs=10000, max_contacts=4000, precision=32,
        update_verts=True, threads=0, use_hull_range=True, branches=False, lock=None,
        **consts) -> dict:
    """Run `frames` Physics.step calls on a copy of the scene `arrays`
    (Data.arrays()).  Returns final state and last-substep outputs (float64).
    branches=True adds "branch_sig": per scene, a hash of the run's
    structural decisions (support vertices chosen, pairs, contacts).
    lock="record" records every branch decision of the run; lock="replay"
    follows the last recording instead of deciding (same threads layout)."""
    a = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
    nb = len(a["body_inv_mass"])
    nv = len(a["orig_vertices"]) if update_verts else 0
    s = _scene(a, update_verts, use_hull_range)
    P = _params(pgs_iterations, max_pairs, max_contacts, consts)
    out, o = _outputs(nb, nv, max_pairs, max_contacts)
    g = (C.c_float * 3)(*gravity)
    sig = _sig(a, branches)
    rc = lib.oracle_run(C.byref(s), C.byref(P), precision, frames, substeps, dt, g,
                        1 if nv else 0, threads, C.byref(o), _p(sig, _u64), LOCK_MODES[lock])
    return _done(rc, "oracle_run", out, o, nv, max_pairs, max_contacts, sig)


def run_f64_state(arrays: dict, *, pos=None, quat=None, vel=None, omega=None, friction=None,
                  frames=1, substeps=10, dt=1.0 / 60.0, gravity=(0.0, -9.81, 0.0),
                  pgs_iterations=4, max_pairs=10000, max_contacts=4000,
                  use_hull_range=True, threads=0, branches=False, lock=None,
                  **consts) -> dict:
    """FP64 run whose initial pos/quat/vel/omega and friction come from
    float64 arrays (None: the scene's float values), for finite differences
    finer than a float ulp.  threads > 0: one instance per scene in
    parallel.  branches and lock as run()."""
    a = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
    nb = len(a["body_inv_mass"])
    s = _scene(a, False, use_hull_range)
    P = _params(pgs_iterations, max_pairs, max_contacts, consts)
    out, o = _outputs(nb, 0, max_pairs, max_contacts)
    d = lambda x: None if x is None else np.ascontiguousarray(x, dtype=np.float64)
    keep = [d(pos), d(quat), d(vel), d(omega), d(friction)]
    g = (C.c_float * 3)(*gravity)
    sig = _sig(a, branches)
    rc = lib.oracle_run_f64_state(C.byref(s), C.byref(P), frames, substeps, dt, g,
                                  *[_p(x, _d) for x in keep], threads, C.byref(o),
                                  _p(sig, _u64), LOCK_MODES[lock])
    return _done(rc, "oracle_run_f64_state", out, o, 0, max_pairs, max_contacts, sig)


def raytrace(verts, idx, node_min, node_max, left, right, count, prim, tri_geom, geom_material,
             albedo, roughness, metallic, emission, ior, cam, width, height, frame, fov,
             threads=0) -> np.ndarray:
    """CPU restatement of raytrace.comp: (height, width, 4) float32 image."""
    f = lambda x: np.ascontiguousarray(x, dtype=np.float32).reshape(-1)
    u = lambda x: np.ascontiguousarray(x).reshape(-1).view(np.uint32)
    args = [f(verts), u(idx), f(node_min), f(node_max), u(left), u(right), u(count), u(prim),
            u(tri_geom), u(geom_material), f(albedo), f(roughness), f(metallic), f(emission),
            f(ior), f(cam)]
    img = np.zeros((height, width, 4), np.float32)
    ptrs = [_p(x, _f if x.dtype == np.float32 else _u) for x in args]
    lib.oracle_raytrace(*ptrs, width, height, frame, fov, threads, _p(img, _f))
    return img


def morton(centroids: np.ndarray):
    c = np.ascontiguousarray(centroids, dtype=np.float32).reshape(-1, 3)
    codes = np.zeros(len(c), np.uint32)
    bounds = np.zeros(6, np.float32)
    lib.oracle_morton(_p(c, _f), len(c), _p(codes, _u), _p(bounds, _f))
    return codes, bounds


def radix_sort(codes: np.ndarray):
    k = np.ascontiguousarray(codes, dtype=np.uint32)
    s = np.zeros_like(k)
    perm = np.zeros_like(k)
    lib.oracle_radix_sort(_p(k, _u), len(k), _p(s, _u), _p(perm, _u))
    return s, perm


def karras(sorted_codes: np.ndarray):
    m = np.ascontiguousarray(sorted_codes, dtype=np.uint32)
    n = len(m)
    left = np.zeros(2 * n - 1, np.uint32)
    right = np.zeros(2 * n - 1, np.uint32)
    parent = np.zeros(2 * n - 1, np.uint32)
    lib.oracle_karras(_p(m, _u), n, _p(left, _u), _p(right, _u), _p(parent, _u))
    return left, right, parent


def angle_bin64(y: float, x: float) -> int:
    """The support lookup's angle bin (0-63) of atan2(y, x) in [0, 2 pi),
    FP32 (seevr_oracle.hpp angle_bin64)."""
    return int(lib.oracle_angle_bin64f(y, x))
