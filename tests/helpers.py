"""Shared test helpers: run a scene on the GPU through the C ABI and read the
outputs back in the oracle's layout."""
from __future__ import annotations

import numpy as np

from seevr_b200 import Caps, Data, Physics, make_params

DT = 1.0 / 60.0
G = (0.0, -9.81, 0.0)


def gpu_run(d: Data, device, frames=1, substeps=10, pgs=4, solver=1, caps: Caps | None = None,
            graph=False, use_hull_range=True, update_verts=True, params=None):
    import torch

    buf = d.upload(device, caps)
    flags = 0 if update_verts else 4
    p = params or make_params(pgs_iterations=pgs, solver=solver, flags=flags | (2 if graph else 0))
    ph = Physics(buf, p, use_hull_range=use_hull_range)
    nv = buf.num_vertices if update_verts else 0
    err = None
    if graph:
        ph.step_async(buf.num_bodies, nv, buf.num_hull_verts, substeps, DT, G, frames=frames)
        torch.cuda.synchronize()
    else:
        for _ in range(frames):
            try:
                ph.step(buf.num_bodies, nv, buf.num_hull_verts, substeps, DT, G)
            except Exception as e:  # capacity overflow is reported after the step
                err = e
    torch.cuda.synchronize()
    out = read_back(buf)
    out["error"] = err
    out["launches"] = ph.kernel_launches
    out["flags"] = ph.read_flags()
    ph.deinit()
    return out


def read_back(buf) -> dict:
    nb = buf.num_bodies
    t = buf.tensors

    def f(name, n, comp):
        return t[name][: n * comp].cpu().numpy().reshape(n, comp) if comp > 1 else \
            t[name][:n].cpu().numpy()

    cnt = t["counters"][:2].cpu().numpy().view(np.uint32)
    npairs = int(min(cnt[0], buf.caps.max_pairs))
    nc = int(min(cnt[1], buf.caps.max_contacts))
    return {
        "pos": f("body_pos", nb, 3), "quat": f("body_quat", nb, 4), "vel": f("body_vel", nb, 3),
        "omega": f("body_omega", nb, 3), "aabb_min": f("body_aabb_min", nb, 3),
        "aabb_max": f("body_aabb_max", nb, 3),
        "verts": t["vertices"][: buf.num_vertices * 3].cpu().numpy().reshape(-1, 3),
        "pairs": t["collision_pairs"][: npairs * 2].cpu().numpy().view(np.uint32).reshape(-1, 2),
        "num_pairs": int(cnt[0]), "num_contacts": int(cnt[1]),
        "c_pos": t["contact_pos"][: nc * 3].cpu().numpy().reshape(-1, 3),
        "c_normal": t["contact_normal"][: nc * 3].cpu().numpy().reshape(-1, 3),
        "c_pen": t["contact_pen"][:nc].cpu().numpy(),
        "lambda": t["lambda_n"][:nc].cpu().numpy(),
        "c_a": t["contact_geom_a"][:nc].cpu().numpy().view(np.uint32),
        "c_b": t["contact_geom_b"][:nc].cpu().numpy().view(np.uint32),
    }


STATE_KEYS = ("pos", "quat", "vel", "omega")
ALL_KEYS = STATE_KEYS + ("aabb_min", "aabb_max", "pairs", "c_pos", "c_normal", "c_pen", "lambda",
                         "c_a", "c_b", "verts")


def assert_bit_exact(gpu: dict, ref: dict, keys=ALL_KEYS):
    """FP32 GPU results against the FP32 oracle (float64 holding float32
    values): equal value for value."""
    assert gpu["num_pairs"] == ref["num_pairs"], (gpu["num_pairs"], ref["num_pairs"])
    assert gpu["num_contacts"] == ref["num_contacts"], (gpu["num_contacts"], ref["num_contacts"])
    for k in keys:
        g = np.asarray(gpu[k])
        r = np.asarray(ref[k])
        if r.dtype == np.float64:
            r = r.astype(np.float32)
        assert g.shape == r.shape, (k, g.shape, r.shape)
        if not np.array_equal(g, r):
            bad = np.argwhere(g != r)
            raise AssertionError(f"{k}: {len(bad)} mismatches, first at {bad[:3].tolist()}: "
                                 f"gpu {g[tuple(bad[0])]} oracle {r[tuple(bad[0])]}")


def max_rel_err(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
