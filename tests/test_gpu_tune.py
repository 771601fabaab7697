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
              {"bundle_bodies": 64}, {"bundle_bodies": 4096, "narrow_blocks_per_sm": 7}):
        got = _run(d, cuda, t)
        for k in ("pos", "quat", "vel", "omega", "pairs", "c_a", "c_b", "lambda"):
            assert np.array_equal(got[k], ref[k]), (t, k)


def test_tuning_limits_and_defaults(cuda):
    d = _batch()
    buf = d.upload(cuda, Caps.for_data(d))
    ph = Physics(buf, make_params(pgs_iterations=10))
    assert ph.get_tuning() == {"bundle_bodies": 512, "narrow_blocks_per_sm": 7,
                               "broad_tile_rows": 64}
    for bad in ({"narrow_blocks_per_sm": 8}, {"broad_tile_rows": 4},
                {"broad_tile_rows": 4096}, {"bundle_bodies": (1 << 24) + 1}):
        with pytest.raises(SeevrError):
            ph.set_tuning(**bad)
    ph.set_tuning(bundle_bodies=256, broad_tile_rows=128)
    assert ph.get_tuning() == {"bundle_bodies": 256, "narrow_blocks_per_sm": 7,
                               "broad_tile_rows": 128}
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
