"""GPU parity on the benchmarked workload itself.

The bench steps 4,096 scenes of 8-512 bodies (half boxes, half 16-segment
spheres) at 30 PGS iterations from a state pre-rolled 90 frames, with the
frame replayed from a CUDA graph.  Scene s of that batch is generated from
its own splitmix64 stream seeded s, so Data.batch(40, seed_base=64) is
exactly scenes 64-103 of the bench batch: 6,486 bodies, ten scenes of 257 to
477 bodies, so the default 512-body solver bundles hold both merged small
scenes and single large ones.  The CUDA graph path must equal the FP32
oracle bit for bit after the bench's pre-roll, in every output the step
writes.
"""
import os

import numpy as np
import pytest

import pyoracle
from helpers import DT, G, assert_bit_exact, gpu_run
from seevr_b200 import Caps, Data, make_params

pytestmark = pytest.mark.gpu

PREROLL = 90  # the bench's untimed settling frames


def test_bench_scenes_after_preroll_bit_exact(cuda):
    d = Data.batch(num_scenes=40, min_bodies=8, max_bodies=512, segments=16, seed_base=64)
    n = np.diff(d.scene_body_offset())
    assert (n >= 257).sum() >= 4 and n.max() > 400 and n.min() < 16
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    frames = PREROLL + 2
    params = make_params(pgs_iterations=30, flags=2)  # CUDA graph, as the bench
    got = gpu_run(d, cuda, frames=frames, pgs=30, caps=caps, graph=True, params=params)
    ref = pyoracle.run(d.arrays(), frames=frames, substeps=10, dt=DT, gravity=G,
                       pgs_iterations=30, max_pairs=caps.max_pairs,
                       max_contacts=caps.max_contacts, threads=os.cpu_count() or 1)
    assert ref["num_contacts"] > 1000, ref["num_contacts"]
    assert got["flags"] == 0, got["flags"]
    assert_bit_exact(got, ref)
