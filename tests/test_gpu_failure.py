"""Failure paths on the GPU, made without a fault: the bounded device-side
waits (decoupled look-back of the scans and sorts) are given a limit of 0
polls, so a look-back gives up at the first tile it finds unpublished.  The
step must come back with SEEVR_ERR_TIMEOUT instead of hanging, write nothing
outside its buffers (the stages after a scan that gave up are skipped), and
leave the handle usable: with the default limit restored it reproduces a
fresh handle's step bit for bit."""
import numpy as np
import pytest

from helpers import DT, G, read_back
from seevr_b200 import Caps, Data, Physics, SeevrError, make_params
from seevr_b200 import _lib as L

pytestmark = pytest.mark.gpu

STATE = (("body_pos", 3), ("body_quat", 4), ("body_vel", 3), ("body_omega", 3))


def _batch(cuda):
    # about 125,000 bodies: the per-row pair scan has ~60 tiles and the
    # contact scan ~100, so look-backs race their predecessors every substep
    d = Data.batch(num_scenes=1024, min_bodies=8, max_bodies=512, seed_base=5)
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    return d, caps, d.upload(cuda, caps)


def test_wait_limit_zero_times_out_and_handle_recovers(cuda):
    import torch

    d, caps, buf = _batch(cuda)
    nb, nhv = buf.num_bodies, buf.num_hull_verts
    ph = Physics(buf, make_params(pgs_iterations=10, flags=4))
    for _ in range(30):  # pre-roll until the scenes hold contacts
        ph.step(nb, 0, nhv, 10, DT, G)
    torch.cuda.synchronize()
    saved = {n: buf[n][: nb * c].clone() for n, c in STATE}

    ph.set_wait_limit(0)
    outcomes = []
    for _ in range(5):
        try:
            ph.step(nb, 0, nhv, 10, DT, G)
            outcomes.append(L.OK)
        except SeevrError as e:
            outcomes.append(e.status)
    torch.cuda.synchronize()
    assert set(outcomes) <= {L.OK, L.ERR_TIMEOUT}, outcomes
    assert L.ERR_TIMEOUT in outcomes, outcomes
    for n, c in STATE:
        assert torch.isfinite(buf[n][: nb * c]).all(), n

    # the same handle, default limit, from the saved state ...
    ph.set_wait_limit(1 << 22)
    for n, c in STATE:
        buf[n][: nb * c].copy_(saved[n])
    ph.step(nb, 0, nhv, 10, DT, G)
    torch.cuda.synchronize()
    a = read_back(buf)
    ph.deinit()
    # ... equals a fresh handle from the same state
    buf2 = d.upload(cuda, caps)
    for n, c in STATE:
        buf2[n][: nb * c].copy_(saved[n])
    ph2 = Physics(buf2, make_params(pgs_iterations=10, flags=4))
    ph2.step(nb, 0, nhv, 10, DT, G)
    torch.cuda.synchronize()
    b = read_back(buf2)
    ph2.deinit()
    assert a["num_contacts"] > 1000
    for k in ("pos", "quat", "vel", "omega", "pairs", "lambda", "c_a", "c_b"):
        assert np.array_equal(a[k], b[k]), k


def test_async_timeout_is_reported_by_read_flags(cuda):
    """Graph-replayed frames do not return a status: the timeout bit is
    reported by read_flags, and the stages that consume scans stay skipped
    until it is read."""
    import torch

    d, caps, buf = _batch(cuda)
    nb, nhv = buf.num_bodies, buf.num_hull_verts
    ph = Physics(buf, make_params(pgs_iterations=10, flags=2 | 4))
    ph.step_async(nb, 0, nhv, 10, DT, G, frames=30)
    torch.cuda.synchronize()
    assert ph.read_flags() & L.DEVICE_FLAG_TIMEOUT == 0
    ph.set_wait_limit(0)
    ph.step_async(nb, 0, nhv, 10, DT, G, frames=5)
    torch.cuda.synchronize()
    with pytest.raises(SeevrError) as e:
        ph.read_flags()
    assert e.value.status == L.ERR_TIMEOUT
    ph.set_wait_limit(1 << 22)
    ph.step_async(nb, 0, nhv, 10, DT, G, frames=2)
    torch.cuda.synchronize()
    assert ph.read_flags() & L.DEVICE_FLAG_TIMEOUT == 0
    ph.deinit()


def _check_mode_handle(buf, params):
    import os

    os.environ["SEEVR_CHECK"] = "1"  # read when the handle is created
    try:
        return Physics(buf, params)
    finally:
        del os.environ["SEEVR_CHECK"]


def test_bounds_check_mode_leaves_results_unchanged(cuda):
    """SEEVR_CHECK=1 validates every index the kernels dereference; on a
    valid batch the step's results are those of a handle without it."""
    d = Data.batch(num_scenes=48, min_bodies=8, max_bodies=96, seed_base=11)
    caps = Caps.for_data(d)
    outs = []
    for check in (False, True):
        buf = d.upload(cuda, caps)
        p = make_params(pgs_iterations=6)
        ph = _check_mode_handle(buf, p) if check else Physics(buf, p)
        for _ in range(20):
            ph.step(buf.num_bodies, buf.num_vertices, buf.num_hull_verts, 10, DT, G)
        outs.append(read_back(buf))
        ph.deinit()
    assert outs[0]["num_contacts"] > 0
    for k in ("pos", "quat", "vel", "omega", "pairs", "lambda", "verts"):
        assert np.array_equal(outs[0][k], outs[1][k]), k


@pytest.mark.parametrize("corrupt", ["hull_range", "geom_body", "support_offset"])
def test_bounds_check_mode_reports_bad_indices(cuda, corrupt):
    """A bad index in the caller's arrays is caught before any kernel uses
    it: the step returns ERR_INVALID_ARGUMENT naming the check, and the
    handle steps normally once the array is repaired."""
    import torch

    d = Data.batch(num_scenes=8, min_bodies=16, max_bodies=64, seed_base=3)
    caps = Caps.for_data(d)
    buf = d.upload(cuda, caps)
    nb = buf.num_bodies
    off = buf.scene_body_offset
    body = int(off[3]) + 2  # a sphere or box of scene 3
    ph = _check_mode_handle(buf, make_params(pgs_iterations=4))
    name = {"hull_range": "hull_range", "geom_body": "geom_body_idx",
            "support_offset": "support_offset"}[corrupt]
    saved = buf[name].clone()
    if corrupt == "hull_range":
        buf[name][2 * body + 1] = buf.num_hull_verts + 5   # count past the hull vertices
    elif corrupt == "geom_body":
        buf[name][body] = int(off[5])                       # a body of scene 5
    else:
        buf[name][body] = buf["support_lookup"].numel() - 10  # table runs past the binding
    torch.cuda.synchronize()
    before = buf["body_pos"][: nb * 3].clone()
    with pytest.raises(SeevrError) as e:
        ph.step(nb, buf.num_vertices, buf.num_hull_verts, 10, DT, G)
    assert e.value.status == L.ERR_INVALID_ARGUMENT
    assert "bounds check" in str(e.value) and f"index {body}" in str(e.value), str(e.value)
    # the stages that would index the bad array did not run
    assert torch.equal(before, buf["body_pos"][: nb * 3])
    buf[name].copy_(saved)
    torch.cuda.synchronize()
    ph.step(nb, buf.num_vertices, buf.num_hull_verts, 10, DT, G)
    ph.deinit()
