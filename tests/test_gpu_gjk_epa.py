"""The GJK + EPA narrowphase (seevr_params.narrowphase = GJK_EPA) on the GPU
against its CPU restatement in the oracle: every output of the step equal
bit for bit, on a settling pile of boxes and 16-segment spheres and on a
batch of scenes replayed from a CUDA graph.  The reference's shader has only
MPR; the oracle tests pin GJK + EPA to MPR's depths and normals and to
analytic overlaps (tests/test_oracle.py)."""
import pytest

import pyoracle
from helpers import DT, G, assert_bit_exact, gpu_run
from seevr_b200 import NARROWPHASE_GJK_EPA, Caps, Data, SeevrError, Physics, make_params

pytestmark = pytest.mark.gpu


def _oracle(d, caps, frames, pgs):
    return pyoracle.run(d.arrays(), frames=frames, substeps=10, dt=DT, gravity=G,
                        pgs_iterations=pgs, max_pairs=caps.max_pairs,
                        max_contacts=caps.max_contacts, threads=8, narrowphase=1)


def test_gjk_epa_pile_bit_exact(cuda):
    d = Data.pile(seed=5, n_boxes=24, n_spheres=24, lo=(-3, 0, -3), hi=(3, 3, 3))
    caps = Caps.for_data(d)
    ref = _oracle(d, caps, 30, 10)
    assert ref["num_contacts"] > 10
    p = make_params(pgs_iterations=10, narrowphase=NARROWPHASE_GJK_EPA)
    got = gpu_run(d, cuda, frames=30, pgs=10, caps=caps, params=p)
    assert_bit_exact(got, ref)


def test_gjk_epa_batch_graph_bit_exact(cuda):
    d = Data.batch(num_scenes=32, min_bodies=8, max_bodies=128, seed_base=7)
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    ref = _oracle(d, caps, 70, 10)
    assert ref["num_contacts"] > 50
    p = make_params(pgs_iterations=10, flags=2, narrowphase=NARROWPHASE_GJK_EPA)
    got = gpu_run(d, cuda, frames=70, pgs=10, caps=caps, graph=True, params=p)
    assert_bit_exact(got, ref)


def test_gjk_epa_adjoint_is_not_supported(cuda):
    import torch

    from seevr_b200.grad import rollout

    d = Data.pile(seed=1, n_boxes=2, n_spheres=2)
    buf = d.upload(cuda, Caps.for_data(d))
    ph = Physics(buf, make_params(pgs_iterations=4, flags=4, narrowphase=NARROWPHASE_GJK_EPA))
    nb = buf.num_bodies
    v0 = buf["body_vel"][: nb * 3].clone().reshape(nb, 3).requires_grad_()
    pos, _, _, _ = rollout(ph, vel0=v0, frames=1, substeps=2)
    with pytest.raises(SeevrError):
        pos.sum().backward()
    torch.cuda.synchronize()
    ph.deinit()
