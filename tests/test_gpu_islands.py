"""Island-parallel PGS (scenes above 1,024 bodies) and the coloured solver.

WAVEFRONT on islands must stay bit-identical to the sequential sweep (the
FP32 oracle).  COLORED visits contacts in a different order, so it is assessed
by what it is for: stacks stay up (tower-top drift), and its state stays
close to the sequential one.
"""
import numpy as np
import pytest

import pyoracle
from helpers import DT, G, assert_bit_exact, gpu_run, read_back
from seevr_b200 import (BROADPHASE_LBVH, Caps, Data, Physics, SOLVER_COLORED, SOLVER_SEQUENTIAL,
                        SOLVER_WAVEFRONT, make_params)

pytestmark = pytest.mark.gpu


def towers(n, h):
    return Data.towers(seed=1, towers=n, height=h, spacing=2.0)


def run(d, cuda, frames, solver, pgs=30, lbvh=False):
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    p = make_params(pgs_iterations=pgs, solver=solver, flags=4,
                    broadphase=BROADPHASE_LBVH if lbvh else 0)
    return gpu_run(d, cuda, frames=frames, pgs=pgs, caps=caps, update_verts=False, params=p)


@pytest.mark.parametrize("solver", [SOLVER_WAVEFRONT, SOLVER_SEQUENTIAL])
def test_island_solver_bit_exact_on_towers(cuda, solver):
    """36 towers of 32 boxes (1,153 bodies: above the warp solver's 1,024, so
    the contacts are solved per island, one island per tower)."""
    d = towers(36, 32)
    assert d.num_bodies > 1024
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    ref = pyoracle.run(d.arrays(), frames=3, substeps=10, dt=DT, gravity=G, pgs_iterations=30,
                       max_pairs=caps.max_pairs, max_contacts=caps.max_contacts,
                       update_verts=False)
    assert ref["num_contacts"] > 400
    got = run(d, cuda, 3, solver)
    assert_bit_exact(got, ref, keys=("pos", "quat", "vel", "omega", "pairs", "c_pos", "c_normal",
                                     "c_pen", "lambda", "c_a", "c_b"))


def test_island_solver_bit_exact_on_pile(cuda):
    """A 2,000-body pile in one scene: islands of every size, one large."""
    d = Data.pile(seed=7, n_boxes=1000, n_spheres=1000, lo=(-14, 0, -14), hi=(14, 6, 14))
    assert d.placement_failures == 0
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    ref = pyoracle.run(d.arrays(), frames=40, substeps=10, dt=DT, gravity=G, pgs_iterations=10,
                       max_pairs=caps.max_pairs, max_contacts=caps.max_contacts,
                       update_verts=False)
    assert ref["num_contacts"] > 300
    got = run(d, cuda, 40, SOLVER_WAVEFRONT, pgs=10)
    assert_bit_exact(got, ref, keys=("pos", "quat", "vel", "omega", "lambda", "c_a", "c_b"))


def _tops(st, n, h):
    # the top box of each tower: bodies 1 + t*h + (h-1)
    return np.array([st["pos"][1 + t * h + h - 1, 1] for t in range(n)])


@pytest.mark.parametrize("n", [16, 40])  # warp-bundle path (513 bodies) and island path
def test_coloured_towers_match_sequential_drift(cuda, n):
    """Coloured PGS on towers of 32 stacked boxes: after 1 s the tower tops
    have sunk (contacts settle to the Baumgarte slop, some towers lean) by
    the same mean amount as under the sequential sweep, and no state is
    non-finite."""
    h = 32
    d = towers(n, h)
    st0 = {"pos": d.arrays()["body_pos"].reshape(-1, 3)}
    col = run(d, cuda, 60, SOLVER_COLORED)
    seq = run(d, cuda, 60, SOLVER_WAVEFRONT)
    for k in ("pos", "vel", "omega", "quat"):
        assert np.isfinite(col[k]).all()
    drift_col = np.abs(_tops(col, n, h) - _tops(st0, n, h))
    drift_seq = np.abs(_tops(seq, n, h) - _tops(st0, n, h))
    print("tower-top drift after 1 s: coloured max %.4f mean %.4f, sequential max %.4f mean %.4f"
          % (drift_col.max(), drift_col.mean(), drift_seq.max(), drift_seq.mean()))
    assert abs(drift_col.mean() - drift_seq.mean()) < 0.02
    assert drift_col.mean() < 0.3


def test_coloured_batch_close_to_sequential(cuda):
    """48 scenes, bundle path: coloured vs sequential order after one frame
    (the same contacts, a different Gauss-Seidel order)."""
    d = Data.batch(num_scenes=48, min_bodies=8, max_bodies=128, seed_base=3)
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    col = gpu_run(d, cuda, frames=20, pgs=30, caps=caps, update_verts=False,
                  params=make_params(pgs_iterations=30, solver=SOLVER_COLORED, flags=4))
    seq = gpu_run(d, cuda, frames=20, pgs=30, caps=caps, update_verts=False,
                  params=make_params(pgs_iterations=30, solver=SOLVER_WAVEFRONT, flags=4))
    assert np.isfinite(col["vel"]).all()
    assert np.abs(col["pos"] - seq["pos"]).max() < 0.05



@pytest.mark.parametrize("n", [36])
def test_giant_island_grid_solve_on_towers(cuda, n):
    """The grid-wide coloured solve (giant.cu) on 36 towers of 32 boxes,
    with the threshold lowered to 16 contacts so that every tower's island
    takes it (flag bit 5): deterministic (two runs equal bit for bit),
    finite, and the tower tops sink by the same mean as under the
    sequential order after 1 s (as the warp-coloured solve does)."""
    from seevr_b200 import _lib as L

    h = 32
    d = towers(n, h)
    st0 = {"pos": d.arrays()["body_pos"].reshape(-1, 3)}
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    runs = []
    for solver in (SOLVER_COLORED, SOLVER_COLORED, SOLVER_WAVEFRONT):
        buf = d.upload(cuda, caps)
        ph = Physics(buf, make_params(pgs_iterations=30, solver=solver, flags=4))
        ph.set_tuning(giant_island_contacts=16)
        flags = 0
        for _ in range(60):
            ph.step(buf.num_bodies, 0, buf.num_hull_verts, 10, DT, G)
            flags |= ph.read_flags()
        r = read_back(buf)
        r["flags"] = flags
        runs.append(r)
        ph.deinit()
    col1, col2, seq = runs
    assert col1["flags"] & L.DEVICE_FLAG_GIANT_ISLANDS, col1["flags"]
    assert not (col1["flags"] & L.DEVICE_FLAG_TIMEOUT), col1["flags"]
    assert not (seq["flags"] & L.DEVICE_FLAG_GIANT_ISLANDS)
    for k in ("pos", "quat", "vel", "omega", "lambda"):
        assert np.array_equal(col1[k], col2[k]), k
        assert np.isfinite(col1[k]).all(), k
    drift_col = np.abs(_tops(col1, n, h) - _tops(st0, n, h))
    drift_seq = np.abs(_tops(seq, n, h) - _tops(st0, n, h))
    print("tower-top drift after 1 s: grid-coloured mean %.4f max %.4f, sequential mean %.4f "
          "max %.4f" % (drift_col.mean(), drift_col.max(), drift_seq.mean(), drift_seq.max()))
    assert abs(drift_col.mean() - drift_seq.mean()) < 0.02
    assert drift_col.mean() < 0.3
