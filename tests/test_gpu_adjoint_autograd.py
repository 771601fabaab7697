"""The CUDA adjoint against torch autograd of plain FP64 operations.

One substep of the step is restated with torch operations in float64:
gravity and damping (physics.comp:418-428), the contact constants and the
unrolled projected Gauss-Seidel sweep with its clamps (physics.comp:500-583)
and integration (physics.comp:586-604).  Within one substep the contacts'
points, normals and depths depend only on the positions and orientations the
substep starts from, so with respect to the initial velocities, angular
velocities and friction coefficients they are constants: the restatement
takes them from the GPU forward (contact buffers after the step) and
autograd differentiates everything else.  The CUDA adjoint
(seevr_physics_adjoint_substep through seevr_b200.grad.rollout) must give
the same gradients, component by component, to the tolerance written in the
test.  A CPU test first pins the restatement to the FP64 oracle.
"""
import numpy as np
import pytest

import pyoracle
from helpers import DT, G, read_back
from seevr_b200 import Caps, Data, Physics, make_params
from seevr_b200.grad import rollout, substep_dt

F32 = lambda x: float(np.float32(x))
BAUMGARTE, SLOP, LIN_DAMP, ANG_DAMP = F32(0.2), F32(0.005), F32(0.999), F32(0.998)


def quat_to_mat(q):
    """physics.comp:74-81, columns of the column-major GLSL mat3."""
    import torch

    x, y, z, w = q
    c0 = torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)])
    c1 = torch.stack([2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x)])
    c2 = torch.stack([2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)])
    return torch.stack([c0, c1, c2], dim=1)  # R[:, k] = column k


def apply_inv_i(R, inv_i, v):
    """physics.comp:90-94: R (inv_i * (R^T v))."""
    return R @ (inv_i * (R.T @ v))


def substep_reference(a, st, contacts, pgs, sub, v0, w0, mu):
    """One substep in float64 torch operations; v0, w0 [nb,3] and mu [nb]
    are the differentiated inputs, everything else constant."""
    import torch

    f64 = lambda x: torch.tensor(np.asarray(x, np.float64))
    nb = len(a["body_inv_mass"])
    inv_m = f64(a["body_inv_mass"])
    inv_i = f64(a["body_inv_inertia"].reshape(nb, 3))
    rest = f64(a["geom_restitution"])
    pos = f64(st["pos"])
    quat = f64(st["quat"])
    g = torch.tensor([F32(x) for x in G], dtype=torch.float64)
    dyn = inv_m > 0
    # step 0: gravity and damping of dynamic bodies
    vel = torch.where(dyn[:, None], v0 * LIN_DAMP + g * sub, v0)
    om = torch.where(dyn[:, None], w0 * ANG_DAMP, w0)
    R = [quat_to_mat(quat[i]) for i in range(nb)]
    fixed = [bool(inv_m[i] == 0 and (inv_i[i] == 0).all()) for i in range(nb)]
    V = [vel[i] for i in range(nb)]
    W = [om[i] for i in range(nb)]
    cons = []
    for c in range(len(contacts["c_a"])):
        A, B = int(contacts["c_a"][c]), int(contacts["c_b"][c])
        n = f64(contacts["c_normal"][c])
        cp = f64(contacts["c_pos"][c])
        ra, rb = cp - pos[A], cp - pos[B]
        ua = V[A] + torch.linalg.cross(W[A], ra)
        ub = V[B] + torch.linalg.cross(W[B], rb)
        vn = torch.dot(ub - ua, n)
        e = torch.maximum(rest[A], rest[B])
        pen = float(contacts["c_pen"][c])
        bias = BAUMGARTE * max(pen - SLOP, 0.0) / sub + e * torch.clamp(-vn, min=0.0)
        ran, rbn = torch.linalg.cross(ra, n), torch.linalg.cross(rb, n)
        kn = inv_m[A] + inv_m[B] + torch.dot(ran, apply_inv_i(R[A], inv_i[A], ran)) + \
            torch.dot(rbn, apply_inv_i(R[B], inv_i[B], rbn))
        cons.append((A, B, n, ra, rb, bias, kn, torch.sqrt(mu[A] * mu[B])))
    lam = [torch.zeros((), dtype=torch.float64) for _ in cons]
    for _ in range(pgs):
        for c, (A, B, n, ra, rb, bias, kn, mu_c) in enumerate(cons):
            ima, imb = inv_m[A], inv_m[B]
            if ima == 0 and imb == 0:  # physics.comp:531
                continue
            va, wa, vb, wb = V[A], W[A], V[B], W[B]
            vn = torch.dot(vb + torch.linalg.cross(wb, rb) - va - torch.linalg.cross(wa, ra), n)
            new_ln = torch.clamp(lam[c] + (-vn + bias) / kn, min=0.0)
            d_ln = new_ln - lam[c]
            lam[c] = new_ln
            imp = d_ln * n
            va = va - ima * imp
            vb = vb + imb * imp
            wa = wa - apply_inv_i(R[A], inv_i[A], torch.linalg.cross(ra, imp))
            wb = wb + apply_inv_i(R[B], inv_i[B], torch.linalg.cross(rb, imp))
            dv = vb + torch.linalg.cross(wb, rb) - va - torch.linalg.cross(wa, ra)
            vt = dv - torch.dot(dv, n) * n
            vt_len = torch.linalg.norm(vt)
            if vt_len > 1e-6:
                td = vt / vt_len
                rat, rbt = torch.linalg.cross(ra, td), torch.linalg.cross(rb, td)
                kt = ima + imb + torch.dot(rat, apply_inv_i(R[A], inv_i[A], rat)) + \
                    torch.dot(rbt, apply_inv_i(R[B], inv_i[B], rbt))
                d_lt = torch.minimum(vt_len / kt, mu_c * new_ln)
                it = d_lt * td
                va = va + ima * it
                vb = vb - imb * it
                wa = wa + apply_inv_i(R[A], inv_i[A], torch.linalg.cross(ra, it))
                wb = wb - apply_inv_i(R[B], inv_i[B], torch.linalg.cross(rb, it))
            if not fixed[A]:
                V[A], W[A] = va, wa
            if not fixed[B]:
                V[B], W[B] = vb, wb
    vel = torch.stack(V)
    om = torch.stack(W)
    # step 6: integrate (explicit xyzw quaternion derivative, renormalised)
    x1, q1 = [], []
    for i in range(nb):
        if not dyn[i]:
            x1.append(pos[i])
            q1.append(quat[i])
            continue
        x1.append(pos[i] + vel[i] * sub)
        qx, qy, qz, qw = quat[i]
        ox, oy, oz = om[i]
        dq = torch.stack([ox * qw + oy * qz - oz * qy, -ox * qz + oy * qw + oz * qx,
                          ox * qy - oy * qx + oz * qw, -ox * qx - oy * qy - oz * qz])
        q = quat[i] + 0.5 * dq * sub
        q1.append(q / torch.linalg.norm(q))
    return torch.stack(x1), torch.stack(q1), vel, om


def settled(seed, pgs):
    d = Data.pile(seed=seed, n_boxes=12, n_spheres=12, lo=(-1.5, 0, -1.5), hi=(1.5, 4, 1.5))
    assert d.placement_failures == 0
    a = d.arrays()
    caps = Caps.for_data(d)
    r = pyoracle.run(a, frames=40, substeps=10, dt=DT, gravity=G, pgs_iterations=pgs,
                     max_pairs=caps.max_pairs, max_contacts=caps.max_contacts,
                     update_verts=False)
    st = {k: r[k].astype(np.float32) for k in ("pos", "quat", "vel", "omega")}
    st["friction"] = np.asarray(a["geom_friction"], np.float32).copy()
    rng = np.random.default_rng(seed)
    st["friction"][1:] = rng.uniform(0.2, 0.8, len(st["friction"]) - 1).astype(np.float32)
    return d, a, caps, st


@pytest.mark.parametrize("pgs", [1, 4, 30])
@pytest.mark.parametrize("seed", [3, 11])
def test_restatement_equals_fp64_oracle_substep(seed, pgs):
    """CPU check of the restatement itself: from the same state and with the
    FP64 oracle's contacts, it reproduces the FP64 oracle's substep to
    float64 rounding."""
    import torch

    d, a, caps, st = settled(seed, pgs)
    sub = substep_dt(DT, 10)
    r = pyoracle.run_f64_state(a, pos=st["pos"].astype(np.float64),
                               quat=st["quat"].astype(np.float64),
                               vel=st["vel"].astype(np.float64),
                               omega=st["omega"].astype(np.float64),
                               friction=st["friction"].astype(np.float64), frames=1, substeps=1,
                               dt=sub, gravity=G, pgs_iterations=pgs, max_pairs=caps.max_pairs,
                               max_contacts=caps.max_contacts)
    assert r["num_contacts"] >= 8
    contacts = {k: r[k] for k in ("c_a", "c_b", "c_pos", "c_normal", "c_pen")}
    out = substep_reference(a, st, contacts, pgs, sub,
                            torch.tensor(st["vel"], dtype=torch.float64),
                            torch.tensor(st["omega"], dtype=torch.float64),
                            torch.tensor(st["friction"], dtype=torch.float64))
    for o, k in zip(out, ("pos", "quat", "vel", "omega")):
        np.testing.assert_allclose(o.numpy(), r[k], rtol=0, atol=1e-12, err_msg=k)


@pytest.mark.gpu
@pytest.mark.parametrize("pgs", [1, 4, 10, 30])
@pytest.mark.parametrize("seed", [3, 11])
def test_adjoint_matches_fp64_autograd_of_plain_ops(cuda, seed, pgs):
    import torch

    d, a, caps, st = settled(seed, pgs)
    nb = d.num_bodies
    sub = substep_dt(DT, 10)
    # the GPU forward of the substep: its contacts
    buf = d.upload(cuda, caps)
    for k, c in (("pos", 3), ("quat", 4), ("vel", 3), ("omega", 3)):
        buf["body_" + k][: nb * c].copy_(torch.tensor(st[k].reshape(-1)))
    buf["geom_friction"][:nb].copy_(torch.tensor(st["friction"]))
    ph = Physics(buf, make_params(pgs_iterations=pgs, flags=4))
    ph.step(nb, 0, buf.num_hull_verts, 1, sub, G)
    torch.cuda.synchronize()
    contacts = read_back(buf)
    assert contacts["num_contacts"] >= 8, contacts["num_contacts"]
    # the CUDA adjoint of the same substep
    rng = np.random.default_rng(100 + seed)
    w = {k: rng.standard_normal((nb, c)) for k, c in (("pos", 3), ("quat", 4), ("vel", 3),
                                                      ("omega", 3))}
    ins = {k: torch.tensor(st[k], device=cuda, requires_grad=True)
           for k in ("vel", "omega", "friction")}
    out = rollout(ph, torch.tensor(st["pos"], device=cuda), torch.tensor(st["quat"], device=cuda),
                  ins["vel"], ins["omega"], ins["friction"], frames=1, substeps=1, dt=sub,
                  gravity=G)
    loss = sum((torch.tensor(w[k], device=cuda, dtype=torch.float32) * o).sum()
               for k, o in zip(("pos", "quat", "vel", "omega"), out))
    loss.backward()
    gpu = {k: v.grad.double().cpu().numpy().reshape(nb, -1) for k, v in ins.items()}
    ph.deinit()
    # torch autograd of the plain-ops restatement
    v0 = torch.tensor(st["vel"], dtype=torch.float64, requires_grad=True)
    w0 = torch.tensor(st["omega"], dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(st["friction"], dtype=torch.float64, requires_grad=True)
    x1, q1, v1, o1 = substep_reference(a, st, contacts, pgs, sub, v0, w0, mu)
    ref_loss = sum((torch.tensor(w[k]) * o).sum()
                   for k, o in zip(("pos", "quat", "vel", "omega"), (x1, q1, v1, o1)))
    ref_loss.backward()
    ref = {"vel": v0.grad.numpy(), "omega": w0.grad.numpy(), "friction": mu.grad.numpy()[:, None]}
    # the restated forward follows the GPU's: final velocities agree to FP32 rounding
    np.testing.assert_allclose(v1.detach().numpy(), out[2].detach().cpu().numpy(),
                               rtol=0, atol=1e-5)
    report = {}
    for k in ref:
        scale = np.abs(ref[k]).max()
        err = np.abs(gpu[k] - ref[k])
        report[k] = (float(scale), float(err.max() / scale),
                     float((err / np.maximum(np.abs(ref[k]), 1e-3 * scale)).max()))
    print(f"seed {seed}, {pgs} PGS iterations, {contacts['num_contacts']} contacts "
          "(group: largest |grad|, normwise err, max componentwise rel err):", report)
    for k in ref:
        scale = np.abs(ref[k]).max()
        if k == "friction" and pgs >= 30:
            # at 30 iterations dL/dmu is what is left of per-iteration terms
            # that cancel as the sweep converges toward sticking (the largest
            # is 1e-6 to 1e-5 here, against about 1 for the velocities); the
            # FP32 forward's rounding, amplified by that cancellation, bounds
            # the agreement with the FP64 forward: normwise 1e-4 of the group
            assert np.abs(gpu[k] - ref[k]).max() <= 1e-4 * scale, (k, report)
            continue
        # every component within 1e-3 of the autograd value, relative to its
        # own size (floored at 1e-3 of the group's largest gradient)
        bad = np.abs(gpu[k] - ref[k]) > 1e-3 * np.maximum(np.abs(ref[k]), 1e-3 * scale)
        assert not bad.any(), (k, np.argwhere(bad)[:4].tolist(), gpu[k][bad][:4],
                               ref[k][bad][:4], report)
