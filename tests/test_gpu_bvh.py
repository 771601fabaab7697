"""Triangle LBVH (BVH.build, bvh.zig:63-172) on the GPU against the oracle's
restatement of bvh.comp: centroids, Morton codes, the sort permutation and
the Karras hierarchy bit-exact; node boxes equal to the unions of their
leaves' triangle boxes."""
import numpy as np
import pytest

import pyoracle
from seevr_b200 import Data
from seevr_b200.bvh import BVH

pytestmark = pytest.mark.gpu


def tri_arrays(d: Data):
    v = d.array("vertices").astype(np.float32)
    idx = d.array("indices").astype(np.uint32)
    return v, idx


@pytest.mark.parametrize("n_scene", ["pile", "large"])
def test_triangle_bvh_matches_oracle(cuda, n_scene):
    import torch

    d = Data.pile(seed=4, n_boxes=40, n_spheres=40) if n_scene == "pile" else \
        Data.large(seed=2, n_bodies=3000)
    v, idx = tri_arrays(d)
    T = len(idx)
    bvh = BVH(torch.from_numpy(v).to(cuda), torch.from_numpy(idx.view(np.int32)).to(cuda))
    bvh.build(T)
    torch.cuda.synchronize()
    g = lambda k: bvh[k].cpu().numpy()
    # centroids (bvh.comp:74-76): ((a + b) + c) / 3 in float32
    tri = v[idx.astype(np.int64)]
    cen = ((tri[:, 0] + tri[:, 1]) + tri[:, 2]) / np.float32(3.0)
    assert np.array_equal(g("centroids")[: 3 * T].reshape(T, 3), cen)
    codes, bounds = pyoracle.morton(cen)
    assert np.array_equal(g("scene_bounds"), bounds)
    s, perm = pyoracle.radix_sort(codes)
    assert np.array_equal(g("morton")[:T].view(np.uint32), s)
    assert np.array_equal(g("sort_indices")[:T].view(np.uint32), perm)
    assert np.array_equal(g("prim_indices")[:T].view(np.uint32), perm)
    left, right, parent = pyoracle.karras(s)
    nodes = 2 * T - 1
    assert np.array_equal(g("left")[:nodes].view(np.uint32)[: T - 1], left[: T - 1])
    assert np.array_equal(g("right")[:nodes].view(np.uint32)[: T - 1], right[: T - 1])
    assert np.array_equal(g("parent")[:nodes].view(np.uint32), parent)
    # boxes: leaves = triangle bounds, internal = union of children (exact)
    nmin = g("node_min")[: 3 * nodes].reshape(nodes, 3)
    nmax = g("node_max")[: 3 * nodes].reshape(nodes, 3)
    lt = tri[perm.astype(np.int64)]
    assert np.array_equal(nmin[T - 1:], lt.min(axis=1))
    assert np.array_equal(nmax[T - 1:], lt.max(axis=1))
    L = left[: T - 1].astype(np.int64)
    R = right[: T - 1].astype(np.int64)
    assert np.array_equal(nmin[: T - 1], np.minimum(nmin[L], nmin[R]))
    assert np.array_equal(nmax[: T - 1], np.maximum(nmax[L], nmax[R]))
    assert np.all(g("count")[T - 1: nodes] == 1) and np.all(g("count")[: T - 1] == 0)
    bvh.deinit()


def test_triangle_bvh_single_triangle(cuda):
    import torch

    v = torch.tensor([[0, 0, 0], [1, 0, 0], [0, 1, 0]], dtype=torch.float32, device=cuda)
    i = torch.tensor([[0, 1, 2]], dtype=torch.int32, device=cuda)
    bvh = BVH(v, i)
    bvh.build(1)
    assert bvh["parent"][0].item() == -1  # 0xFFFFFFFF
    assert bvh["node_max"][:3].tolist() == [1.0, 1.0, 0.0]
    bvh.deinit()
