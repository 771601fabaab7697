"""Differentiable rollouts of the physics step (reverse mode).

    buf = Data.rollout(num_scenes=32, bodies=64).upload("cuda:0")
    ph = Physics(buf, make_params(pgs_iterations=30))
    n = buf.num_bodies
    vel0 = buf.tensors["body_vel"][: 3 * n].clone().reshape(n, 3).requires_grad_()
    pos, quat, vel, omega = rollout(ph, vel0=vel0, frames=4)
    loss(pos).backward()          # vel0.grad: dL/d initial velocities

The forward runs the regular step one substep at a time (a frame of k
substeps is exactly k calls of one substep with dt / k), ordered on the
current stream, and keeps a checkpoint of (pos, quat, vel, omega) before
each.  The backward restores
each checkpoint in reverse order and calls seevr_physics_adjoint_substep,
which recomputes that substep's contacts and PGS sweep on the GPU and
propagates dL/d(state) back through it, accumulating dL/d friction.
Contact selection and the solver's clamps are piecewise constant, so the
gradient is that of the branch the forward took.  No counterpart in the
reference, whose step has no reverse mode.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .physics import Physics


def _names():
    return ("body_pos", 3), ("body_quat", 4), ("body_vel", 3), ("body_omega", 3)


class _Rollout:
    """torch.autograd.Function over a Physics handle (built lazily so that
    importing this module does not import torch)."""

    fn = None

    @classmethod
    def get(cls):
        if cls.fn is not None:
            return cls.fn
        import torch

        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, ph, cfg, pos0, quat0, vel0, omega0, friction):
                nb, nhv, steps, sub_dt, gravity = cfg
                t = ph.buffers.tensors
                ins = (pos0, quat0, vel0, omega0)
                views = [t[name][: nb * k] for name, k in _names()]
                with torch.no_grad():
                    for v, x in zip(views, ins):
                        v.copy_(x.detach().reshape(-1))
                    t["geom_friction"][:nb].copy_(friction.detach().reshape(-1))
                    # checkpoints and substeps stay ordered on one stream,
                    # with no host round trip until the end
                    stream = torch.cuda.current_stream(ph.buffers.device)
                    ckpt = []
                    for _ in range(steps):
                        ckpt.append(torch.cat([v.clone() for v in views]))
                        ph.step_async(nb, 0, nhv, 1, sub_dt, gravity, frames=1, stream=stream)
                    outs = [v.clone().reshape(x.shape) for v, x in zip(views, ins)]
                    torch.cuda.synchronize(ph.buffers.device)
                    if ph.read_flags() & (L.DEVICE_FLAG_PAIR_OVERFLOW | L.DEVICE_FLAG_CONTACT_OVERFLOW):
                        raise L.SeevrError(L.ERR_CAPACITY,
                                           "pairs or contacts exceeded the caps during the rollout")
                ctx.ph, ctx.cfg, ctx.ckpt = ph, cfg, ckpt
                ctx.shapes = [x.shape for x in ins] + [friction.shape]
                return tuple(outs)

            @staticmethod
            def backward(ctx, gpos, gquat, gvel, gomega):
                ph = ctx.ph
                nb, nhv, steps, sub_dt, gravity = ctx.cfg
                t = ph.buffers.tensors
                dev = ph.buffers.device
                # the reverse pass carries FP64 gradients from substep to substep
                g = []
                for gx, (name, k) in zip((gpos, gquat, gvel, gomega), _names()):
                    g.append(torch.zeros(nb * k, dtype=torch.float64, device=dev) if gx is None
                             else gx.detach().reshape(-1).to(torch.float64).contiguous().clone())
                gf = torch.zeros(max(nb, 1), dtype=torch.float64, device=dev)
                gr = L.AdjointGrads(g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr(),
                                    g[3].data_ptr(), gf.data_ptr())
                views = [t[name][: nb * k] for name, k in _names()]
                sizes = [nb * k for _, k in _names()]
                with torch.no_grad():
                    for ck in reversed(ctx.ckpt):
                        for v, part in zip(views, torch.split(ck, sizes)):
                            v.copy_(part)
                        torch.cuda.current_stream(dev).synchronize()
                        L.check(L.lib.seevr_physics_adjoint_substep(
                            ph._h, nb, nhv, sub_dt, L.fptr(gravity, 3), C.byref(gr)))
                ctx.ckpt = None
                sh = ctx.shapes
                f = lambda x, shape: x.reshape(shape).to(torch.float32)
                return (None, None, f(g[0], sh[0]), f(g[1], sh[1]), f(g[2], sh[2]),
                        f(g[3], sh[3]), f(gf[:nb], sh[4]))

        cls.fn = Fn
        return Fn


def substep_dt(dt: float, substeps: int) -> float:
    """The substep length the step uses (physics.zig:90), in float32."""
    return float(np.float32(np.float32(dt) / np.float32(substeps)))


def rollout(ph: Physics, pos0=None, quat0=None, vel0=None, omega0=None, friction=None, *,
            frames: int = 1, substeps: int = 10, dt: float = 1.0 / 60.0,
            gravity=(0.0, -9.81, 0.0)):
    """Run `frames` frames of `substeps` substeps from the given initial state
    (torch tensors on the handle's device; None = the bound buffers' current
    values) and return the final (pos, quat, vel, omega), differentiable
    with respect to all five inputs.  Raises SeevrError (ERR_CAPACITY) when
    pairs or contacts exceeded the caps in any substep."""
    import torch

    b = ph.buffers
    nb = b.num_bodies
    t = b.tensors
    cur = lambda name, k: t[name][: nb * k].clone().reshape(nb, k)
    pos0 = cur("body_pos", 3) if pos0 is None else pos0
    quat0 = cur("body_quat", 4) if quat0 is None else quat0
    vel0 = cur("body_vel", 3) if vel0 is None else vel0
    omega0 = cur("body_omega", 3) if omega0 is None else omega0
    friction = t["geom_friction"][:nb].clone() if friction is None else friction
    for x in (pos0, quat0, vel0, omega0, friction):
        if x.dtype != torch.float32 or x.device != t["body_pos"].device:
            raise ValueError("rollout inputs must be float32 tensors on the handle's device")
    cfg = (nb, b.num_hull_verts, frames * substeps, substep_dt(dt, substeps),
           tuple(float(x) for x in gravity))
    return _Rollout.get().apply(ph, cfg, pos0, quat0, vel0, omega0, friction)
