"""seevr_physics_step_noalloc, the physics step for callers that cannot
allocate device memory (a renderer that owns and pre-sizes all device
memory, a real-time loop that must not allocate after start-up, or code
enqueuing work during a global-mode stream capture).  Its scratch is a
static device array inside the library instead of cudaMalloc'd buffers.

The test drives it through the C ABI and checks, on two calls in a row,
that it produces exactly what seevr_physics_step produces for the same
scene (the tolerance of the other parity tests: equal float32 values).
It lives in its own file, collected last, and passes alone in a fresh
process as well as after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from helpers import DT, G, read_back
from seevr_b200 import Caps, Data, Physics, make_params
from seevr_b200 import _lib as L

pytestmark = pytest.mark.gpu

KEYS = ("pos", "quat", "vel", "omega", "aabb_min", "aabb_max", "pairs", "c_pos", "c_normal",
        "c_pen", "lambda", "c_a", "c_b", "verts")


def test_noalloc_step_matches_step_on_two_calls(cuda):
    import torch

    d = Data.pile(seed=21, n_boxes=24, n_spheres=24, lo=(-3, 0, -3), hi=(3, 4, 3))
    caps = Caps.for_data(d)
    assert d.num_bodies <= 4096 and caps.max_pairs <= 32768 and caps.max_contacts <= 16384
    ref = d.upload(cuda, caps)
    mine = d.upload(cuda, caps)
    params = make_params(pgs_iterations=10)
    ph = Physics(ref, params)
    nb, nv, nhv = ref.num_bodies, ref.num_vertices, ref.num_hull_verts
    # settle for a while so that the compared calls see contacts
    for _ in range(40):
        ph.step(nb, nv, nhv, 10, DT, G)
    torch.cuda.synchronize()
    for name in ("body_pos", "body_quat", "body_vel", "body_omega"):
        mine[name].copy_(ref[name])
    torch.cuda.synchronize()
    bind = mine.bindings()
    for call in range(2):
        ph.step(nb, nv, nhv, 10, DT, G)
        st = L.lib.seevr_physics_step_noalloc(C.byref(bind), C.byref(params), caps.max_pairs,
                                              caps.max_contacts, nb, nv, nhv, 10, DT,
                                              L.fptr(G, 3), None)
        L.check(st)
        torch.cuda.synchronize()
        a, b = read_back(ref), read_back(mine)
        assert a["num_contacts"] > 0, "the compared calls must exercise the solver"
        assert (a["num_pairs"], a["num_contacts"]) == (b["num_pairs"], b["num_contacts"]), call
        for k in KEYS:
            assert np.array_equal(a[k], b[k]), (call, k)
    ph.deinit()


def test_noalloc_rejects_sizes_beyond_its_limits(cuda):
    d = Data.pile(seed=1, n_boxes=2, n_spheres=2)
    buf = d.upload(cuda)
    bind = buf.bindings()
    p = make_params()
    st = L.lib.seevr_physics_step_noalloc(C.byref(bind), C.byref(p), 10000, 4000, 5000, 0,
                                          d.num_hull_verts, 1, DT, L.fptr(G, 3), None)
    assert st == L.ERR_INVALID_ARGUMENT
    assert b"at most 4096 bodies" in L.lib.seevr_last_error()
    st = L.lib.seevr_physics_step_noalloc(C.byref(bind), C.byref(p), 40000, 4000, d.num_bodies,
                                          0, d.num_hull_verts, 1, DT, L.fptr(G, 3), None)
    assert st == L.ERR_INVALID_ARGUMENT


def _noalloc_frames(d, cuda, frames, pgs, solver, caps):
    """`frames` calls of the no-allocation step on a fresh upload of d."""
    import torch

    buf = d.upload(cuda, caps)
    bind = buf.bindings()
    p = make_params(pgs_iterations=pgs, solver=solver, flags=4)  # no render vertices
    for _ in range(frames):
        L.check(L.lib.seevr_physics_step_noalloc(C.byref(bind), C.byref(p), caps.max_pairs,
                                                 caps.max_contacts, buf.num_bodies, 0,
                                                 buf.num_hull_verts, 10, DT, L.fptr(G, 3),
                                                 None))
    torch.cuda.synchronize()
    return read_back(buf)


@pytest.mark.parametrize("scene,frames,pgs,solver", [
    # 36 towers of 32 boxes, 1,153 bodies: above the 1,024 bodies of the
    # warp solver, so one block solves the scene with its bodies in shared
    # memory (the handle's step would use its island solver instead)
    ("towers", 3, 30, 0), ("towers", 3, 30, 1),
    # a 2,601-body pile: above the 2,048 bodies of the shared-memory
    # broadphase and solver, so pairs come from the global-memory
    # all-pairs kernel and the block solver sweeps in global memory
    ("pile", 30, 4, 1),
])
def test_noalloc_large_scenes_bit_exact(cuda, scene, frames, pgs, solver):
    import pyoracle

    if scene == "towers":
        d = Data.towers(seed=1, towers=36, height=32, spacing=2.0)
        assert 1024 < d.num_bodies <= 2048
    else:
        d = Data.pile(seed=11, n_boxes=1300, n_spheres=1300, lo=(-16, 0, -16), hi=(18, 3, 18))
        assert 2048 < d.num_bodies <= 4096
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    assert caps.max_pairs <= 32768 and caps.max_contacts <= 16384
    ref = pyoracle.run(d.arrays(), frames=frames, substeps=10, dt=DT, gravity=G,
                       pgs_iterations=pgs, max_pairs=caps.max_pairs,
                       max_contacts=caps.max_contacts, update_verts=False)
    assert ref["num_contacts"] > 300
    got = _noalloc_frames(d, cuda, frames, pgs, solver, caps)
    # the 2,601-body scene's bundle exceeds shared memory: the block solver
    # sweeps in global memory (status bit 3); the towers' 1,153 bodies fit
    solver_global = (L.lib.seevr_physics_noalloc_flags() >> 3) & 1
    assert solver_global == (1 if scene == "pile" else 0)
    assert (got["num_pairs"], got["num_contacts"]) == (ref["num_pairs"], ref["num_contacts"])
    for k in ("pos", "quat", "vel", "omega", "aabb_min", "aabb_max", "pairs", "c_pos",
              "c_normal", "c_pen", "lambda", "c_a", "c_b"):
        r = np.asarray(ref[k])
        r = r.astype(np.float32) if r.dtype == np.float64 else r
        assert np.array_equal(got[k], r), k
