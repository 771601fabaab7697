"""Autotuner for the batched step's launch shapes.

The shapes (seevr_physics_set_tuning: solver bundle size, narrowphase
resident blocks per SM, broadphase rows per block) change speed only, never
results, and the best values depend on the workload: scene sizes, contact
density, hull sizes.  `autotune` therefore times candidates on the caller's
own handle and state.  It saves the body state, and for each candidate
restores it, runs one untimed frame, then times `frames` frames with CUDA
events on its stream (the best of `repeats` runs); the search is coordinate
descent over the parameters in turn, starting from the values in use.  At
the end the state is restored and the fastest shapes stay set.
"""
from __future__ import annotations

from typing import Callable

# scene groups first: the shapes of the other stages' kernels are best
# chosen at the group size they will run at
DEFAULT_CANDIDATES = {
    "scene_groups": [1, 2, 4, 6, 8],
    "narrow_blocks_per_sm": [4, 5, 6, 7],
    "broad_tile_rows": [32, 64, 128, 256],
    "bundle_bodies": [256, 512, 1024],
}


def search(candidates: dict, start: dict, measure: Callable[[dict], float],
           passes: int = 1) -> tuple[dict, list]:
    """Coordinate descent: for each parameter in turn, time every candidate
    value with the others fixed and keep the fastest (the current value
    wins ties).  Returns the best setting and the (setting, ms) trials."""
    best = dict(start)
    trials = []
    cache = {}

    def timed(setting):
        key = tuple(sorted(setting.items()))
        if key not in cache:
            cache[key] = measure(dict(setting))
            trials.append((dict(setting), cache[key]))
        return cache[key]

    best_ms = timed(best)
    for _ in range(passes):
        changed = False
        for name, values in candidates.items():
            for v in values:
                if v == best[name]:
                    continue
                trial = dict(best, **{name: v})
                ms = timed(trial)
                if ms < best_ms:
                    best, best_ms, changed = trial, ms, True
        if not changed:
            break
    return best, trials


def autotune(ph, buf, substeps: int, dt: float, gravity=(0.0, -9.81, 0.0), frames: int = 2,
             repeats: int = 2, candidates: dict | None = None, passes: int = 1) -> dict:
    """Time launch shapes on `ph` (a Physics bound to `buf`) and set the
    fastest.  Returns {"best": setting, "ms_per_frame": ..., "trials": [...]}.
    Body state is restored before every trial and at the end."""
    import torch

    cands = dict(candidates if candidates is not None else DEFAULT_CANDIDATES)
    if buf.num_scenes <= 1:
        cands.pop("bundle_bodies", None)  # one scene is one bundle
    nb, nv, nhv = buf.num_bodies, buf.num_vertices, buf.num_hull_verts
    t = buf.tensors
    names = (("body_pos", 3), ("body_quat", 4), ("body_vel", 3), ("body_omega", 3))
    saved = {n: t[n][: nb * c].clone() for n, c in names}
    stream = torch.cuda.Stream(t["body_pos"].device)
    start = ph.get_tuning()

    def restore():
        torch.cuda.synchronize()
        for n, c in names:
            t[n][: nb * c].copy_(saved[n])
        torch.cuda.synchronize()

    def measure(setting):
        ph.set_tuning(**setting)
        best = float("inf")
        for _ in range(repeats):
            restore()
            with torch.cuda.stream(stream):
                ph.step_async(nb, nv, nhv, substeps, dt, gravity, frames=1, stream=stream)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ph.step_async(nb, nv, nhv, substeps, dt, gravity, frames=frames, stream=stream)
                e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / frames)
        return best

    try:
        best, trials = search(cands, {k: start[k] for k in cands}, measure, passes)
    finally:
        restore()
    ph.set_tuning(**dict(start, **best))
    ms = min(m for s, m in trials if s == best)
    return {"best": ph.get_tuning(), "ms_per_frame": ms, "trials": trials}
