"""Launch-shape tuning (seevr_physics_set_tuning, seevr_b200.tune.autotune):
shapes change speed only, so every setting must give the same state bit for
bit, and the tuner must leave the body state as it found it."""
import numpy as np
import pytest

from helpers import DT, G, read_back
from seevr_b200 import Caps, Data, Physics, SeevrError, make_params
from seevr_b200.tune import autotune

pytestmark = pytest.mark.gpu


def _batch():
    return Data.batch(num_scenes=48, min_bodies=8, max_bodies=128, seed_base=31)


def _run(d, cuda, tuning=None, frames=10):
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    buf = d.upload(cuda, caps)
    ph = Physics(buf, make_params(pgs_iterations=10, flags=4))
    if tuning:
        ph.set_tuning(**tuning)
    for _ in range(frames):
        ph.step(buf.num_bodies, buf.num_vertices, buf.num_hull_verts, 10, DT, G)
    out = read_back(buf)
    ph.deinit()
    return out


def test_tuning_leaves_results_unchanged(cuda):
    d = _batch()
    ref = _run(d, cuda)
    for t in ({"narrow_blocks_per_sm": 2}, {"broad_tile_rows": 8}, {"broad_tile_rows": 512},
              {"bundle_bodies": 64}, {"bundle_bodies": 4096, "narrow_blocks_per_sm": 7},
              {"scene_groups": 2}, {"scene_groups": 3, "bundle_bodies": 64},
              {"scene_groups": 8, "narrow_blocks_per_sm": 3}):
        got = _run(d, cuda, t)
        assert (got["num_pairs"], got["num_contacts"]) == (ref["num_pairs"], ref["num_contacts"])
        for k in ("pos", "quat", "vel", "omega", "aabb_min", "aabb_max", "pairs", "c_pos",
                  "c_normal", "c_pen", "c_a", "c_b", "lambda", "verts"):
            assert np.array_equal(got[k], ref[k]), (t, k)


@pytest.mark.parametrize("groups", [2, 4])
def test_scene_groups_in_the_frame_graph(cuda, groups):
    """Scene groups on their own streams inside the captured frame graph:
    every output of the batch equals the single-group graph step's, frame
    after frame, and the flags and counters are those of the whole batch."""
    import torch

    d = Data.batch(num_scenes=96, min_bodies=8, max_bodies=256, seed_base=41)
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    outs = []
    for g in (1, groups):
        buf = d.upload(cuda, caps)
        ph = Physics(buf, make_params(pgs_iterations=10, flags=2))
        ph.set_tuning(scene_groups=g)
        assert ph.get_tuning()["scene_groups"] == g
        ph.step_async(buf.num_bodies, buf.num_vertices, buf.num_hull_verts, 10, DT, G, frames=70)
        torch.cuda.synchronize()
        outs.append((read_back(buf), ph.read_flags(), ph.read_counters()))
        ph.deinit()
    (a, fa, ca), (b, fb, cb) = outs
    assert a["num_contacts"] > 50 and ca == cb and fa == fb
    for k in ("pos", "quat", "vel", "omega", "aabb_min", "aabb_max", "pairs", "c_pos",
              "c_normal", "c_pen", "c_a", "c_b", "lambda", "verts"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("groups,flags,pinned", [(1, 2, True), (4, 2, True), (4, 0, True),
                                                  (4, 2, False)])
def test_step_io_equals_upload_step_download(cuda, groups, flags, pinned):
    """seevr_physics_step_io: host copies per scene group around each group's
    frame (page-locked arrays; frame graph or launched kernels) or one after
    another (pageable arrays) give the state that upload_state, the step and
    download_state give, frame after frame, with each input array also the
    output; the bound buffers hold the same state."""
    import torch

    d = Data.batch(num_scenes=64, min_bodies=8, max_bodies=256, seed_base=43)
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    keys = ("pos", "quat", "vel", "omega")
    finals = []
    for use_io in (False, True):
        buf = d.upload(cuda, caps)
        ph = Physics(buf, make_params(pgs_iterations=10, flags=flags))
        ph.set_tuning(scene_groups=groups)
        nb, nv, nhv = buf.num_bodies, buf.num_vertices, buf.num_hull_verts
        st = read_back(buf)
        host = {k: np.ascontiguousarray(st[k], dtype=np.float32) for k in keys}
        if use_io and pinned:
            host = {k: torch.from_numpy(v).pin_memory() for k, v in host.items()}
        for _ in range(40):  # the bodies land: contacts at the last frames
            if use_io:
                ph.step_io(nb, nv, nhv, 10, DT, G, inputs=host, outputs=host)
            else:
                ph.upload_state(nb, *[host[k] for k in keys])
                ph.step_async(nb, nv, nhv, 10, DT, G, frames=1)
                torch.cuda.synchronize()
                ph.download_state(nb, *[host[k] for k in keys])
        torch.cuda.synchronize()
        dev = read_back(buf)
        ph.deinit()
        out = {k: (v.numpy() if hasattr(v, "numpy") else v) for k, v in host.items()}
        for k in keys:
            assert np.array_equal(out[k], dev[k]), (use_io, k)
        finals.append((out, dev["num_contacts"]))
    (a, ca), (b, cb) = finals
    assert ca > 20 and ca == cb
    for k in keys:
        assert np.array_equal(a[k], b[k]), k


def test_scene_groups_overflow_is_reported(cuda):
    """The merged counters are the batch's true totals: a pair cap below them
    raises ERR_CAPACITY as without groups."""
    d = _batch()
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    ref = _run(d, cuda, frames=1)
    caps.max_pairs = max(ref["num_pairs"] // 2, 1)
    buf = d.upload(cuda, caps)
    ph = Physics(buf, make_params(pgs_iterations=10, flags=4))
    ph.set_tuning(scene_groups=3)
    with pytest.raises(SeevrError) as e:
        ph.step(buf.num_bodies, buf.num_vertices, buf.num_hull_verts, 10, DT, G)
    assert e.value.status == 2  # ERR_CAPACITY
    assert ph.read_counters()[0] == ref["num_pairs"]
    ph.deinit()


def test_tuning_limits_and_defaults(cuda):
    d = _batch()
    buf = d.upload(cuda, Caps.for_data(d))
    ph = Physics(buf, make_params(pgs_iterations=10))
    assert ph.get_tuning() == {"bundle_bodies": 512, "narrow_blocks_per_sm": 7,
                               "broad_tile_rows": 64, "scene_groups": 1,
                               "giant_island_contacts": 4096}
    for bad in ({"narrow_blocks_per_sm": 8}, {"broad_tile_rows": 4},
                {"broad_tile_rows": 4096}, {"bundle_bodies": (1 << 24) + 1},
                {"scene_groups": 9}):
        with pytest.raises(SeevrError):
            ph.set_tuning(**bad)
    ph.set_tuning(bundle_bodies=256, broad_tile_rows=128)
    assert ph.get_tuning() == {"bundle_bodies": 256, "narrow_blocks_per_sm": 7,
                               "broad_tile_rows": 128, "scene_groups": 1,
                               "giant_island_contacts": 4096}
    ph.deinit()


def test_autotune_restores_state_and_sets_best(cuda):
    import torch

    d = _batch()
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    buf = d.upload(cuda, caps)
    ph = Physics(buf, make_params(pgs_iterations=10, flags=4))
    for _ in range(20):  # settle: contacts present
        ph.step(buf.num_bodies, buf.num_vertices, buf.num_hull_verts, 10, DT, G)
    before = read_back(buf)
    res = autotune(ph, buf, 10, DT, G, frames=1, repeats=1,
                   candidates={"narrow_blocks_per_sm": [4, 7], "broad_tile_rows": [32, 64],
                               "bundle_bodies": [256, 512]})
    torch.cuda.synchronize()
    after = read_back(buf)
    for k in ("pos", "quat", "vel", "omega"):
        assert np.array_equal(after[k], before[k]), k
    assert ph.get_tuning() == res["best"]
    assert len(res["trials"]) >= 4 and res["ms_per_frame"] > 0
    ph.deinit()
