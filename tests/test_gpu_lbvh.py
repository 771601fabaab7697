"""LBVH broadphase on the GPU: pair lists bit-exact against the all-pairs
broadphase, Morton codes and the sort permutation bit-exact against the
oracle's restatement of bvh.comp (30-bit codes, stable 4-bit LSD sort)."""
import numpy as np
import pytest

import pyoracle
from helpers import DT, G, gpu_run, read_back
from seevr_b200 import BROADPHASE_LBVH, BROADPHASE_N2, Caps, Data, Physics, make_params

pytestmark = pytest.mark.gpu


def run(d, cuda, broadphase, frames=1, substeps=2):
    import torch

    buf = d.upload(cuda, Caps.for_data(d))
    ph = Physics(buf, make_params(pgs_iterations=4, broadphase=broadphase, flags=4))
    for _ in range(frames):
        ph.step(buf.num_bodies, 0, buf.num_hull_verts, substeps, DT, G)
    torch.cuda.synchronize()
    out = read_back(buf)
    lb = ph.read_lbvh(buf.num_bodies) if broadphase == BROADPHASE_LBVH else None
    ph.deinit()
    return out, lb


@pytest.mark.parametrize("n", [2, 3, 100, 4097])
def test_lbvh_pairs_equal_all_pairs_small(cuda, n):
    d = Data.large(seed=n, n_bodies=n - 1)
    a, _ = run(d, cuda, BROADPHASE_N2, frames=3)
    b, _ = run(d, cuda, BROADPHASE_LBVH, frames=3)
    assert a["num_pairs"] == b["num_pairs"]
    assert np.array_equal(a["pairs"], b["pairs"])
    for k in ("pos", "quat", "vel", "omega"):
        assert np.array_equal(a[k], b[k]), k


def test_lbvh_pairs_equal_all_pairs_large_scene(cuda):
    """Config-1 scale: 32,768 bodies (40% boxes, 40% spheres, 20% hulls)."""
    d = Data.large(seed=0, n_bodies=32768)
    a, _ = run(d, cuda, BROADPHASE_N2)
    b, _ = run(d, cuda, BROADPHASE_LBVH)
    assert a["num_pairs"] == b["num_pairs"] > 0
    assert np.array_equal(a["pairs"], b["pairs"])
    for k in ("pos", "quat", "vel", "omega", "aabb_min", "aabb_max"):
        assert np.array_equal(a[k], b[k]), k


def test_lbvh_dense_pile_pairs(cuda):
    """A settled pile has many overlaps per body (rows longer than one
    32-entry write chunk are exercised by the ground body's row)."""
    d = Data.pile(seed=9, n_boxes=200, n_spheres=200, lo=(-6, 0, -6), hi=(6, 6, 6))
    assert d.placement_failures == 0
    a, _ = run(d, cuda, BROADPHASE_N2, frames=40, substeps=10)
    b, _ = run(d, cuda, BROADPHASE_LBVH, frames=40, substeps=10)
    assert a["num_pairs"] > 300
    assert np.array_equal(a["pairs"], b["pairs"])
    assert np.array_equal(a["pos"], b["pos"])


def test_lbvh_morton_and_permutation_match_oracle(cuda):
    d = Data.large(seed=3, n_bodies=20000)
    out, (codes, order, bounds) = run(d, cuda, BROADPHASE_LBVH, frames=1, substeps=1)
    centroids = (out["aabb_min"] + out["aabb_max"]) * np.float32(0.5)
    ref_codes, ref_bounds = pyoracle.morton(centroids)
    assert np.array_equal(bounds, ref_bounds)
    ref_sorted, ref_perm = pyoracle.radix_sort(ref_codes)
    assert np.array_equal(codes, ref_sorted)
    assert np.array_equal(order, ref_perm)
