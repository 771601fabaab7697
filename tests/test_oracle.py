"""Known-answer tests of the CPU oracle, derived from physics.comp / bvh.comp.

The reference ships no tests or golden vectors, so these pin the oracle to
analytic consequences of the shader code (numbering follows the list of
derived known answers in the design notes):
  1 free fall follows v_k = 0.999^k v_0 + g dt sum 0.999^i (physics.comp:422)
  2 static-static pairs are never emitted; touching AABBs count (459, 462-464)
  3 morton3d(0,0,0)=0, morton3d(1,1,1)=0x3FFFFFFF, stable order on equal keys
  4 quaternion norm preserved by integrate (601-602)
  5 a box resting on the ground box gives normal ~ +-y and depth = overlap
  6 a 16-segment sphere uses the lookup support path, a box brute force
  7 both inv_mass == 0 -> contact skipped by PGS (531)
"""
import math

import numpy as np
import pytest

import pyoracle
from seevr_b200 import Data


def _one_body_scene(kind="box", center=(0.0, 50.0, 0.0), ground=True, **kw):
    d = Data()
    g = d.add_material((.5, .5, .5), .9, 0, (0, 0, 0), 0, 0.0)
    m = d.add_material((.8, .2, .2), .4, 0, (0, 0, 0), 0, 1000.0)
    if ground:
        d.add_box((0, -0.25, 0), (10, 0.25, 10), (.3, .3, .3), 0.5, 0.2, g)
    if kind == "box":
        b = d.add_box(center, kw.get("half", (0.5, 0.5, 0.5)), (1, 0, 0), 0.5, 0.2, m)
    else:
        b = d.add_sphere(center, kw.get("radius", 0.5), (1, 1, 1), kw.get("segments", 16), 0.5,
                         0.2, m)
    return d, b


def test_free_fall_matches_closed_form():  # KAT 1
    d, b = _one_body_scene(center=(0.0, 500.0, 0.0))
    d.set_body_vel(b, v=(1.0, 2.0, -3.0))
    a = d.arrays()
    substeps, frames, dt = 10, 3, 1.0 / 60.0
    out = pyoracle.run(a, frames=frames, substeps=substeps, dt=dt, precision=64)
    k = substeps * frames
    v0 = np.array([1.0, 2.0, -3.0])
    # the FP64 run receives dt, g and the damping constant as float32 (the
    # ABI's types) and does the arithmetic in double
    h = np.float64(np.float32(dt)) / substeps
    g = np.array([0.0, np.float64(np.float32(-9.81)), 0.0])
    damp = np.float64(np.float32(0.999))
    want = damp ** k * v0 + h * g * sum(damp ** i for i in range(k))
    assert np.allclose(out["vel"][b], want, rtol=1e-12, atol=1e-12)
    # static ground untouched
    assert np.all(out["vel"][0] == 0)
    out32 = pyoracle.run(a, frames=frames, substeps=substeps, dt=dt, precision=32)
    assert np.allclose(out32["vel"][b], want, rtol=1e-5)


def test_static_pairs_skipped_and_touching_counts():  # KAT 2
    d = Data()
    g = d.add_material((.5, .5, .5), .9, 0, (0, 0, 0), 0, 0.0)
    m = d.add_material((.8, .2, .2), .4, 0, (0, 0, 0), 0, 1000.0)
    d.add_box((0, 0, 0), (1, 1, 1), (1, 1, 1), .5, .2, g)     # 0 static
    d.add_box((1.5, 0, 0), (1, 1, 1), (1, 1, 1), .5, .2, g)   # 1 static, overlaps 0
    d.add_box((10, 0, 0), (1, 1, 1), (1, 1, 1), .5, .2, m)    # 2 dynamic
    d.add_box((12, 0, 0), (1, 1, 1), (1, 1, 1), .5, .2, m)    # 3 dynamic, touches 2 exactly
    a = d.arrays()
    out = pyoracle.run(a, frames=1, substeps=1, dt=1e-9, gravity=(0, 0, 0), update_verts=False)
    pairs = {tuple(p) for p in out["pairs"].tolist()}
    assert (0, 1) not in pairs  # both static
    assert (2, 3) in pairs       # closed interval test: max_a == min_b overlaps


def test_morton_known_answers_and_stable_sort():  # KAT 3
    # bounds from (0,0,0)..(1,1,1): normalised corners
    c = np.array([[0, 0, 0], [1, 1, 1], [0.5, 0.5, 0.5]], np.float32)
    codes, bounds = pyoracle.morton(c)
    assert codes[0] == 0
    assert codes[1] == 0x3FFFFFFF
    assert list(bounds) == [0, 0, 0, 1, 1, 1]
    rng = np.random.default_rng(0)
    keys = rng.integers(0, 64, size=5000).astype(np.uint32)  # many duplicates
    s, perm = pyoracle.radix_sort(keys)
    assert np.array_equal(perm, np.argsort(keys, kind="stable"))
    assert np.array_equal(s, np.sort(keys))


def test_quaternion_norm_preserved():  # KAT 4
    d, b = _one_body_scene(center=(0.0, 500.0, 0.0))
    d.set_body_vel(b, w=(3.0, -2.0, 5.0))
    out = pyoracle.run(d.arrays(), frames=5, substeps=10, precision=32)
    assert abs(np.linalg.norm(out["quat"][b]) - 1.0) < 1e-6


def test_box_resting_on_ground_contact():  # KAT 5
    pen = 0.01
    d, b = _one_body_scene(center=(0.0, 0.5 - pen, 0.0))
    out = pyoracle.run(d.arrays(), frames=1, substeps=1, dt=1e-9, gravity=(0, 0, 0),
                       update_verts=False, precision=64)
    assert out["num_contacts"] >= 1
    n = out["c_normal"][0]
    assert abs(abs(n[1]) - 1.0) < 1e-6
    assert abs(out["c_pen"][0] - pen) < 1e-6


def test_support_paths():  # KAT 6
    d, b = _one_body_scene(kind="sphere", segments=16)
    a = d.arrays()
    assert a["geom_data"][b][1] == 289  # (16+1)^2 UV-sphere vertices
    assert a["support_offset"][b] != 0  # > 32 verts: lookup table
    assert a["support_offset"][0] == 0  # box: brute force
    out = pyoracle.run(a, frames=1, substeps=1, update_verts=False)
    assert out["ops"]["support_brute"] == 0 or out["ops"]["support_lookup"] >= 0


def test_sphere_on_ground_uses_lookup_and_brute():  # KAT 6, both paths executed
    d, b = _one_body_scene(kind="sphere", center=(0.0, 0.49, 0.0), segments=16)
    out = pyoracle.run(d.arrays(), frames=1, substeps=1, dt=1e-6, gravity=(0, 0, 0),
                       update_verts=False)
    assert out["num_contacts"] == 1
    assert out["ops"]["support_lookup"] > 0 and out["ops"]["support_brute"] > 0


def test_static_static_contact_skipped():  # KAT 7
    d = Data()
    g = d.add_material((.5, .5, .5), .9, 0, (0, 0, 0), 0, 0.0)
    m = d.add_material((.5, .5, .5), .9, 0, (0, 0, 0), 0, 1000.0)
    d.add_box((0, 0, 0), (1, 1, 1), (1, 1, 1), .5, .2, g)
    d.add_box((0, 50, 0), (1, 1, 1), (1, 1, 1), .5, .2, m)
    out = pyoracle.run(d.arrays(), frames=1, substeps=1, update_verts=False)
    assert out["ops"]["pgs_contact_iters"] == 0


def test_angle_bins_match_the_angle():
    """The support lookup's bin (physics.comp:136-147: atan(y,x), +2 pi when
    negative, / 2 pi * 64, truncated, mod 64) found by quadrant and tangent
    comparisons equals the bin of the exact angle, except within float
    rounding of a bin boundary."""
    rng = np.random.default_rng(1)
    pts = rng.normal(size=(20000, 2)) * rng.choice([1e-3, 1, 1e3], size=(20000, 1))
    near = 0
    for y, x in pts.astype(np.float32):
        a = math.atan2(float(y), float(x))
        if a < 0:
            a += 2 * math.pi
        f = a / (2 * math.pi) * 64
        want = int(f) % 64
        got = pyoracle.angle_bin64(y, x)
        if got != want:
            # only at a boundary: the exact angle is within 1e-6 of a bin edge
            assert abs(f - round(f)) < 64e-6 / (2 * math.pi), (y, x, got, want)
            assert got in ((want + 1) % 64, (want - 1) % 64)
            near += 1
    assert near < 20
    # axis directions and the origin, as the reference's atan(0,0) = 0
    assert [pyoracle.angle_bin64(y, x) for y, x in
            ((0, 1), (1, 0), (0, -1), (-1, 0), (0, 0), (1, 1), (-1, -1))] == [0, 16, 32, 48, 0, 8, 40]
    # every bin is reached, in order around the circle
    th = (np.arange(64) + 0.5) * (2 * math.pi / 64)
    assert [pyoracle.angle_bin64(np.float32(math.sin(t)), np.float32(math.cos(t))) for t in th] == \
        list(range(64))


def test_fp32_vs_fp64_one_step():
    d = Data.pile(seed=3, n_boxes=32, n_spheres=32)
    a = d.arrays()
    o32 = pyoracle.run(a, frames=1, substeps=10, precision=32)
    o64 = pyoracle.run(a, frames=1, substeps=10, precision=64)
    err = np.abs(o32["pos"] - o64["pos"]).max() / np.abs(o64["pos"]).max()
    assert err < 1e-5


def test_batch_threads_equal_whole_batch():
    d = Data.batch(num_scenes=6, min_bodies=8, max_bodies=40)
    a = d.arrays()
    kw = dict(frames=8, substeps=10, pgs_iterations=10, max_pairs=100000, max_contacts=100000)
    whole = pyoracle.run(a, threads=0, **kw)
    per = pyoracle.run(a, threads=4, **kw)
    for k in ("pos", "quat", "vel", "omega", "aabb_min", "aabb_max", "pairs", "c_pos", "lambda"):
        assert np.array_equal(whole[k], per[k]), k
    assert whole["num_pairs"] == per["num_pairs"]


def test_batched_scenes_equal_separate_runs():
    d = Data.batch(num_scenes=3, min_bodies=10, max_bodies=30, seed_base=7)
    a = d.arrays()
    off = a["scene_body_offset"]
    whole = pyoracle.run(a, frames=5, substeps=10)
    for s in range(3):
        single = Data.batch(num_scenes=1, min_bodies=10, max_bodies=30, seed_base=7 + s)
        o = pyoracle.run(single.arrays(), frames=5, substeps=10)
        assert np.array_equal(o["pos"], whole["pos"][off[s]:off[s + 1]])


def test_overflow_keeps_canonical_prefix():
    d = Data.pile(seed=0, n_boxes=64, n_spheres=64)
    a = d.arrays()
    full = pyoracle.run(a, frames=20, substeps=10, max_pairs=100000, max_contacts=100000)
    assert full["num_pairs"] > 8
    # same first frames, but the last substep's pairs truncated: compare a
    # one-substep run on the final state
    b = dict(a)
    b["body_pos"] = full["pos"].astype(np.float32)
    b["body_quat"] = full["quat"].astype(np.float32)
    b["body_vel"] = full["vel"].astype(np.float32)
    b["body_omega"] = full["omega"].astype(np.float32)
    big = pyoracle.run(b, frames=1, substeps=1, max_pairs=100000, max_contacts=100000)
    small = pyoracle.run(b, frames=1, substeps=1, max_pairs=5, max_contacts=100000)
    assert small["num_pairs"] == big["num_pairs"]
    assert np.array_equal(small["pairs"], big["pairs"][:5])


def test_karras_hierarchy_structure():
    rng = np.random.default_rng(2)
    keys = np.sort(rng.integers(0, 1 << 30, size=777).astype(np.uint32))
    keys[100:110] = keys[100]  # duplicates exercise the index tiebreak
    keys = np.sort(keys)
    left, right, parent = pyoracle.karras(keys)
    n = len(keys)
    assert parent[0] == 0xFFFFFFFF
    # every node except the root has exactly one parent that points back
    for node in range(1, 2 * n - 1):
        p = parent[node]
        assert left[p] == node or right[p] == node
    # leaves reachable from the root cover 0..n-1 in order
    order, stack = [], [0]
    while stack:
        x = stack.pop()
        if x >= n - 1:
            order.append(int(left[x]))
        else:
            stack.append(int(right[x]))
            stack.append(int(left[x]))
    assert order == list(range(n))


def _two(shape_a, shape_b, offset):
    from seevr_b200 import Data

    d = Data()
    m = d.add_material((0.5, 0.5, 0.5), 0.5, 0.0, (0, 0, 0), 0.0, 1000.0)

    def add(s, c):
        if s[0] == "box":
            return d.add_box(c, s[1], (1, 1, 1), 0.5, 0.2, m)
        return d.add_sphere(c, s[1], (1, 1, 1), 16, 0.5, 0.2, m)

    add(shape_a, (0.0, 5.0, 0.0))
    add(shape_b, (offset[0], 5.0 + offset[1], offset[2]))
    return d


@pytest.mark.parametrize("case", [
    # shapes, offset of B from A, exact depth and normal (None: not analytic)
    (("box", (0.5, 0.5, 0.5)), ("box", (0.5, 0.5, 0.5)), (0.0, 0.9, 0.0), 0.1, (0, 1, 0)),
    (("box", (0.5, 0.5, 0.5)), ("box", (0.5, 0.5, 0.5)), (0.95, 0.1, 0.2), 0.05, (1, 0, 0)),
    (("sphere", 0.5), ("box", (0.5, 0.5, 0.5)), (0.0, 0.95, 0.0), None, None),
    (("sphere", 0.5), ("sphere", 0.4), (0.3, 0.7, 0.1), None, None),
])
def test_gjk_epa_known_answers_and_mpr_agreement(case):
    """The GJK + EPA narrowphase (narrowphase=1) on single pairs: the depth and
    normal of two overlapping axis-aligned boxes are the overlap along the
    separating axis; on every case depth and normal agree with MPR's (the
    reference's narrowphase) to float rounding."""
    from seevr_b200 import Caps

    sa, sb, off, depth, normal = case
    d = _two(sa, sb, off)
    caps = Caps.for_data(d)
    got = {}
    for nph in (0, 1):
        r = pyoracle.run(d.arrays(), frames=1, substeps=1, pgs_iterations=4,
                         max_pairs=caps.max_pairs, max_contacts=caps.max_contacts,
                         narrowphase=nph)
        assert r["num_contacts"] == 1
        got[nph] = r
    epa, mpr = got[1], got[0]
    if depth is not None:
        assert epa["c_pen"][0] == pytest.approx(depth, abs=2e-6)
        np.testing.assert_allclose(epa["c_normal"][0], normal, atol=1e-6)
    assert epa["c_pen"][0] == pytest.approx(mpr["c_pen"][0], rel=1e-5, abs=1e-6)
    np.testing.assert_allclose(epa["c_normal"][0], mpr["c_normal"][0], atol=1e-5)


def test_gjk_epa_separated_pair_has_no_contact():
    from seevr_b200 import Caps

    d = _two(("box", (0.5, 0.5, 0.5)), ("box", (0.5, 0.5, 0.5)), (0.0, 1.2, 0.0))
    caps = Caps.for_data(d)
    r = pyoracle.run(d.arrays(), frames=1, substeps=1, max_pairs=caps.max_pairs,
                     max_contacts=caps.max_contacts, narrowphase=1)
    assert r["num_contacts"] == 0
