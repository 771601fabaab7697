"""GPU parity: the sm_100a step through the C ABI against the FP32 oracle.

The library is built with -fmad=false and keeps the oracle's operation
order, so the bar is bit-exact (equal float32 values) for body state, AABBs,
pair lists, contacts, impulses and render vertices.  Where a test compares
against the FP64 oracle the tolerance is written in the test.
"""
import numpy as np
import pytest

import pyoracle
from helpers import DT, G, assert_bit_exact, gpu_run, max_rel_err, read_back
from seevr_b200 import (Caps, Data, Physics, SeevrError, SOLVER_SEQUENTIAL, SOLVER_WAVEFRONT,
                        make_params)

pytestmark = pytest.mark.gpu


def oracle(d, frames=1, substeps=10, pgs=4, caps=None, threads=0, precision=32, **kw):
    caps = caps or Caps.for_data(d)
    return pyoracle.run(d.arrays(), frames=frames, substeps=substeps, dt=DT, gravity=G,
                        pgs_iterations=pgs, max_pairs=caps.max_pairs,
                        max_contacts=caps.max_contacts, threads=threads, precision=precision,
                        **kw)


@pytest.mark.parametrize("solver", [SOLVER_SEQUENTIAL, SOLVER_WAVEFRONT])
def test_small_pile_bit_exact(cuda, solver):
    d = Data.pile(seed=1, n_boxes=24, n_spheres=24)
    ref = oracle(d, frames=3, pgs=4)
    got = gpu_run(d, cuda, frames=3, pgs=4, solver=solver)
    assert_bit_exact(got, ref)


def low_pile(seed, n):
    """Bodies spawned just above the ground in a 6 m wide column, about 2 m^3
    per body: contacts form within the first frames."""
    d = Data.pile(seed=seed, n_boxes=n // 2, n_spheres=n - n // 2, lo=(-3, 0, -3),
                  hi=(3, max(3.0, n / 18.0), 3))
    assert d.placement_failures == 0
    return d


def test_pile_with_contacts_bit_exact(cuda):
    d = low_pile(5, 48)
    ref = oracle(d, frames=30, pgs=10)
    assert ref["num_contacts"] > 10
    got = gpu_run(d, cuda, frames=30, pgs=10)
    assert_bit_exact(got, ref)


def test_large_scene_many_contacts_bit_exact(cuda):
    """About 860 bodies in one scene (one warp, velocities in global memory) with
    more contacts than the solver setup keeps in registers (256 per warp):
    the memory path of the level assignment and ordering."""
    d = Data.pile(seed=6, n_boxes=450, n_spheres=450, lo=(-8, 0, -8), hi=(8, 5, 8))
    assert 512 < d.num_bodies <= 1024
    ref = oracle(d, frames=60, pgs=10)
    assert ref["num_contacts"] > 300
    got = gpu_run(d, cuda, frames=60, pgs=10)
    assert_bit_exact(got, ref)


def test_scene_above_tile_limit_bit_exact(cuda):
    """2,601 bodies in one scene: above the 2,048 bodies the
    shared-memory broadphase stages, so pairs come from the global-memory
    all-pairs kernel, and above 1,024 bodies, so contacts are solved per
    island."""
    d = Data.pile(seed=11, n_boxes=1300, n_spheres=1300, lo=(-16, 0, -16), hi=(18, 3, 18))
    assert d.num_bodies > 2048
    ref = oracle(d, frames=30, pgs=4)
    assert ref["num_pairs"] > 1000 and ref["num_contacts"] > 300
    got = gpu_run(d, cuda, frames=30, pgs=4)
    assert_bit_exact(got, ref)


def test_config0_pile_bit_exact(cuda):
    """512 bodies (256 boxes + 256 16-segment spheres) + ground, 30 PGS
    iterations, 4 frames."""
    d = Data.pile(seed=0)
    ref = oracle(d, frames=4, pgs=30)
    got = gpu_run(d, cuda, frames=4, pgs=30)
    assert_bit_exact(got, ref)


def test_sequential_equals_wavefront_many_contacts(cuda):
    d = low_pile(2, 128)
    a = gpu_run(d, cuda, frames=90, pgs=8, solver=SOLVER_SEQUENTIAL, update_verts=False)
    b = gpu_run(d, cuda, frames=90, pgs=8, solver=SOLVER_WAVEFRONT, update_verts=False)
    assert a["num_contacts"] > 20
    for k in ("pos", "quat", "vel", "omega", "lambda"):
        assert np.array_equal(a[k], b[k]), k


def test_batch_bit_exact_against_oracle(cuda):
    d = Data.batch(num_scenes=48, min_bodies=8, max_bodies=96, seed_base=11)
    ref = oracle(d, frames=3, pgs=6, threads=8)
    got = gpu_run(d, cuda, frames=3, pgs=6)
    assert_bit_exact(got, ref)


@pytest.mark.parametrize("frames", [2, 20])
def test_bundle_size_does_not_change_results(cuda, frames):
    """bundle_bodies only changes how scenes are grouped per solver warp:
    one bundle of every scene (about 68,000 bodies, more than 16-bit
    bundle-local indices hold; velocities in global memory), the default
    512 and 64 (one scene per bundle) give the same state bit for bit."""
    d = Data.batch(num_scenes=300, min_bodies=200, max_bodies=256, seed_base=21)
    assert d.num_bodies > 65536
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    runs = [gpu_run(d, cuda, frames=frames, pgs=10, caps=caps, update_verts=False,
                    params=make_params(pgs_iterations=10, flags=4, bundle_bodies=bb))
            for bb in (1 << 20, 0, 64)]
    for r in runs[1:]:
        for k in ("pos", "quat", "vel", "omega", "lambda"):
            assert np.array_equal(r[k], runs[0][k]), k


def test_golden_fixtures_bit_exact(cuda):
    """The CUDA path reproduces the committed golden fixtures (tests/golden)
    bit for bit: body state, pairs, contacts and impulses."""
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import make_golden

    for name, (make, frames, pgs) in sorted(make_golden.CASES.items()):
        z = np.load(Path(__file__).resolve().parent / "golden" / f"{name}.npz")
        d = make(Data)
        assert make_golden.scene_digest(d.arrays()) == str(z["scene_sha256"]), name
        got = gpu_run(d, cuda, frames=frames, pgs=pgs)
        assert got["num_pairs"] == int(z["num_pairs"]), name
        assert got["num_contacts"] == int(z["num_contacts"]), name
        for k in make_golden.KEYS:
            assert np.array_equal(np.asarray(got[k]).view(np.uint8), z[k].view(np.uint8)), (name, k)


def test_scene_in_batch_equals_scene_alone(cuda):
    batch = Data.batch(num_scenes=16, min_bodies=8, max_bodies=64, seed_base=100)
    off = batch.scene_body_offset()
    got = gpu_run(batch, cuda, frames=40, pgs=10, update_verts=False)
    for s in (0, 7, 15):
        alone = Data.batch(num_scenes=1, min_bodies=8, max_bodies=64, seed_base=100 + s)
        one = gpu_run(alone, cuda, frames=40, pgs=10, update_verts=False)
        for k in ("pos", "quat", "vel", "omega"):
            assert np.array_equal(one[k], got[k][off[s]:off[s + 1]]), (s, k)


def test_cuda_graph_equals_direct(cuda):
    d = Data.batch(num_scenes=8, min_bodies=16, max_bodies=64, seed_base=3)
    a = gpu_run(d, cuda, frames=6, pgs=5)
    b = gpu_run(d, cuda, frames=6, pgs=5, graph=True)
    for k in ("pos", "quat", "vel", "omega", "pairs", "verts"):
        assert np.array_equal(a[k], b[k]), k


def test_geom_data_path_equals_hull_range_path(cuda):
    d = Data.pile(seed=4, n_boxes=20, n_spheres=20)
    a = gpu_run(d, cuda, frames=3, use_hull_range=True)
    b = gpu_run(d, cuda, frames=3, use_hull_range=False)
    for k in ("pos", "quat", "aabb_min", "aabb_max", "pairs"):
        assert np.array_equal(a[k], b[k]), k


def test_overflow_reported_and_canonical_prefix_kept(cuda):
    d = Data()
    g = d.add_material((.5, .5, .5), .9, 0, (0, 0, 0), 0, 0.0)
    m = d.add_material((.8, .2, .2), .4, 0, (0, 0, 0), 0, 1000.0)
    d.add_box((0, -0.25, 0), (50, 0.25, 50), (.3, .3, .3), 0.5, 0.2, g)
    for i in range(30):  # a row of boxes all resting in the ground: 30 pairs, 30 contacts
        d.add_box((1.2 * i, 0.49, 0.0), (0.5, 0.5, 0.5), (1, 0, 0), .5, .2, m)
    caps = Caps(max_bodies=31, max_hull_verts=d.num_hull_verts, max_vertices=d.num_vertices,
                max_pairs=7, max_contacts=5)
    ref = oracle(d, frames=1, substeps=1, caps=caps)
    got = gpu_run(d, cuda, frames=1, substeps=1, caps=caps)
    assert isinstance(got["error"], SeevrError) and got["error"].status == 2
    assert got["num_pairs"] == ref["num_pairs"] == 30
    assert_bit_exact(got, ref)


def test_fp32_state_error_against_fp64(cuda):
    """One frame of the 512-body pile: GPU FP32 vs FP64 oracle (error
    reference).  Tolerance 1e-5 relative on positions."""
    d = Data.pile(seed=0)
    got = gpu_run(d, cuda, frames=1, pgs=30)
    ref64 = oracle(d, frames=1, pgs=30, precision=64)
    assert max_rel_err(got["pos"], ref64["pos"]) < 1e-5
    assert max_rel_err(got["vel"], ref64["vel"]) < 1e-4


def test_large_scene_pairs_against_brute_force(cuda):
    """32,768-body scene (40% boxes, 40% spheres, 20% hulls): the pair list
    of the last substep is sorted, unique, overlapping and complete against
    an independent all-pairs test on the GPU's own AABBs."""
    import torch

    d = Data.large(seed=0, n_bodies=32768)
    got = gpu_run(d, cuda, frames=1, substeps=2, update_verts=False)
    pairs = got["pairs"].astype(np.int64)
    assert len(pairs) == got["num_pairs"] > 0
    assert np.all(pairs[:, 0] < pairs[:, 1])
    key = pairs[:, 0] * 1_000_000 + pairs[:, 1]
    assert np.all(np.diff(key) > 0)  # strictly increasing: canonical and unique
    mn = torch.from_numpy(got["aabb_min"]).to(cuda)
    mx = torch.from_numpy(got["aabb_max"]).to(cuda)
    inv_mass = torch.from_numpy(d.array("body_inv_mass")).to(cuda)
    n = mn.shape[0]
    count = 0
    for i0 in range(0, n, 2048):
        i1 = min(n, i0 + 2048)
        a_mn, a_mx = mn[i0:i1, None, :], mx[i0:i1, None, :]
        ov = ~((a_mx < mn[None]) | (mx[None] < a_mn)).any(-1)
        ii = torch.arange(i0, i1, device=cuda)[:, None]
        jj = torch.arange(n, device=cuda)[None, :]
        both_static = (inv_mass[i0:i1, None] <= 0) & (inv_mass[None, :] <= 0)
        count += int((ov & (jj > ii) & ~both_static).sum())
    assert count == got["num_pairs"]


def test_large_scene_bit_exact_small_substeps(cuda):
    """4,096 bodies of the large-scene mix (boxes, spheres, hulls) against the
    oracle."""
    d = Data.large(seed=1, n_bodies=4096)
    ref = oracle(d, frames=1, substeps=3)
    got = gpu_run(d, cuda, frames=1, substeps=3)
    assert_bit_exact(got, ref)


def test_profile_mode_and_launch_count(cuda):
    import ctypes

    import torch
    from seevr_b200 import Physics, Profile, make_params

    d = Data.pile(seed=0, n_boxes=16, n_spheres=16)
    buf = d.upload(cuda)
    ph = Physics(buf, make_params())
    prof = Profile()
    ph.step(buf.num_bodies, buf.num_vertices, buf.num_hull_verts, 10, DT, G, prof)
    torch.cuda.synchronize()
    assert prof.calls == 1
    assert prof.ms[1] > 0 and prof.ms[2] > 0 and prof.ms[5] > 0
    assert ph.kernel_launches >= 10 * 8
    ph.deinit()


def test_batch_with_a_nan_body_matches_oracle(cuda):
    """A body whose quaternion is NaN gets NaN bounds, as the reference's
    reduction (seeded with the first vertex's NaN) does, and the reference's
    predicate then counts it as overlapping every body of its scene.  Every
    output, NaNs included, equals the oracle's."""
    import torch

    d = Data.batch(num_scenes=16, min_bodies=8, max_bodies=64, seed_base=77)
    off = d.scene_body_offset()
    k = int(off[3]) + 1
    a = d.arrays()
    a["body_quat"][k] = np.nan
    ref = pyoracle.run(a, frames=2, substeps=10, dt=DT, gravity=G, pgs_iterations=4,
                       max_pairs=Caps.for_data(d).max_pairs,
                       max_contacts=Caps.for_data(d).max_contacts)
    buf = d.upload(cuda)
    buf.tensors["body_quat"][4 * k: 4 * k + 4] = float("nan")
    ph = Physics(buf, make_params(pgs_iterations=4))
    for _ in range(2):
        ph.step(buf.num_bodies, buf.num_vertices, buf.num_hull_verts, 10, DT, G)
    torch.cuda.synchronize()
    got = read_back(buf)
    ph.deinit()
    assert np.isnan(got["quat"][k]).all() and np.isnan(got["aabb_min"][k]).all()
    assert ref["num_pairs"] > 0
    assert (got["num_pairs"], got["num_contacts"]) == (ref["num_pairs"], ref["num_contacts"])
    for key in ("pos", "quat", "vel", "omega", "aabb_min", "aabb_max", "pairs", "c_pos",
                "c_normal", "c_pen", "lambda", "verts"):
        g = np.asarray(got[key])
        r = np.asarray(ref[key]).astype(g.dtype)
        assert g.shape == r.shape, key
        assert np.array_equal(g, r, equal_nan=g.dtype.kind == "f"), key


def test_synchronous_step_replaying_the_graph_equals_eager(cuda):
    """seevr_physics_step with SEEVR_FLAG_CUDA_GRAPH replays the captured
    frame before its wait; every output equals the kernel-by-kernel step's,
    frame after frame, and the oracle's."""
    d = low_pile(9, 40)
    eager = gpu_run(d, cuda, frames=12, pgs=10)
    graph = gpu_run(d, cuda, frames=12, pgs=10, params=make_params(pgs_iterations=10, flags=2))
    for k in ("pos", "quat", "vel", "omega", "aabb_min", "aabb_max", "pairs", "c_pos", "c_normal",
              "c_pen", "lambda", "verts"):
        assert np.array_equal(eager[k], graph[k]), k
    assert_bit_exact(graph, oracle(d, frames=12, pgs=10))
