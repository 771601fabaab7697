"""Benchmark of the physics step: body-substeps/s of the batched CUDA-graph
step over 4,096 independent scenes, beside the plain single-scene drop-in
looped per scene and the CPU oracle.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one frame (Physics.step: 10 substeps, 30 PGS iterations) of the
whole batch.  The scenes are pre-rolled (--preroll frames, untimed) so the
timed frames contain a settling pile rather than free fall.  Under torchrun
each rank runs its own 4,096 scenes (weak scaling, no collective in the
step); rank 0 prints one JSON line.

Besides the headline the line carries: the whole-step and per-stage
roofline, the CPU oracle on a sample of the same scenes and state with the
GPU's results on that sample compared bit for bit, the plain drop-in, the
512-body drop-in scene (120 frames at 4 and 30 PGS iterations), the
32,768-body scene with the LBVH and all-pairs broadphases, the
differentiable rollout, and the stacked towers.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = ("body-substeps/s batched vs plain step, same B200, ≤1e-4 state err; adjoint/s")
UNIT = "body-substeps/s"
DT = 1.0 / 60.0
G = (0.0, -9.81, 0.0)
STATE = (("pos", "body_pos", 3), ("quat", "body_quat", 4), ("vel", "body_vel", 3),
         ("omega", "body_omega", 3))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scenes", type=int, default=4096)
    ap.add_argument("--min-bodies", type=int, default=8)
    ap.add_argument("--max-bodies", type=int, default=512)
    ap.add_argument("--segments", type=int, default=16)
    ap.add_argument("--substeps", type=int, default=10)
    ap.add_argument("--pgs", type=int, default=30)
    ap.add_argument("--preroll", type=int, default=90)
    ap.add_argument("--sample-stride", type=int, default=16,
                    help="CPU legs run every n-th scene of the batch (same histogram)")
    ap.add_argument("--plain-scenes", type=int, default=32)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adjoint-scenes", type=int, default=1024)
    ap.add_argument("--adjoint-bodies", type=int, default=64)
    ap.add_argument("--adjoint-frames", type=int, default=60)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--towers", type=int, default=1024)
    ap.add_argument("--tower-height", type=int, default=256)
    ap.add_argument("--tower-frames", type=int, default=300)
    ap.add_argument("--tower-overlap", type=float, default=0.002)
    ap.add_argument("--tower-wavefront-frames", type=int, default=40)
    ap.add_argument("--no-towers", action="store_true")
    ap.add_argument("--no-config0", action="store_true")
    ap.add_argument("--config0-frames", type=int, default=120)
    ap.add_argument("--no-config1", action="store_true")
    ap.add_argument("--config1-bodies", type=int, default=32768)
    ap.add_argument("--config1-frames", type=int, default=60)
    ap.add_argument("--no-raytrace", action="store_true")
    ap.add_argument("--rt-width", type=int, default=640)
    ap.add_argument("--rt-height", type=int, default=480)
    ap.add_argument("--prof-frames", type=int, default=3)
    ap.add_argument("--bundle-bodies", type=int, default=0,
                    help="solver bundle size in bodies (0: the library default)")
    ap.add_argument("--scene-groups", type=int, default=0,
                    help="scene ranges stepped on their own streams (0: the library default)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the library's launch shapes instead of timing candidates on "
                         "the settled state before the timed region")
    return ap.parse_args()


def workload_config(a, world):
    """The workload both arms report (identical keys and values)."""
    return {
        "workload": (f"batched scenes: {a.scenes} independent scenes per GPU, dynamic bodies "
                     f"log-uniform {a.min_bodies}-{a.max_bodies} (half boxes with half-extents "
                     f"U(0.2,0.6) m, half {a.segments}-segment UV spheres r U(0.2,0.5) m) on a "
                     f"static ground box, {a.substeps} substeps x {a.pgs} PGS iterations per "
                     f"60 Hz frame, after {a.preroll} untimed frames of settling"),
        "scenes": a.scenes, "min_bodies": a.min_bodies, "max_bodies": a.max_bodies,
        "sphere_segments": a.segments, "substeps": a.substeps, "pgs_iterations": a.pgs,
        "preroll_frames": a.preroll, "dt": DT, "seed": "scene s of rank r: seed r*scenes+s",
        "l2": "inputs larger than L2: the hull vertices (888 MB at 4,096 scenes) are read "
              "every substep, no flush needed",
        "broadphase": "all-pairs per scene", "solver": "wavefront (bit-identical to sequential)",
        "parallelism": f"scenes sharded x{world}",
    }


# ---------------------------------------------------------------------------
# clocks during the timed region
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()  # the timed region starts once sampling has begun
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# the sample of scenes the CPU legs run
def sample_seeds(a, rank):
    """Every `sample_stride`-th scene of this rank's batch: the body-count
    histogram of the sample follows the batch's."""
    stride = max(1, a.sample_stride)
    return [rank * a.scenes + s for s in range(0, a.scenes, stride)]


def sample_data(a, rank):
    from seevr_b200 import Data

    return Data.batch_seeds(sample_seeds(a, rank), min_bodies=a.min_bodies,
                            max_bodies=a.max_bodies, segments=a.segments)


def sample_state(a, full_off, state, rank):
    """Rows of `state` (per-body arrays of the full batch) that belong to the
    sampled scenes, concatenated in sample order."""
    rows = np.concatenate([np.arange(full_off[s - rank * a.scenes],
                                     full_off[s - rank * a.scenes + 1])
                           for s in sample_seeds(a, rank)])
    return {k: v[rows] for k, v in state.items()}


def oracle_frames(arrays, state, frames, a, threads):
    """The CPU oracle: `frames` frames of the scenes in `arrays` from
    `state`; returns (dynamic body-substeps, seconds, out)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    arr = dict(arrays)
    if state is not None:
        for key, name, _ in STATE:
            arr[name] = np.ascontiguousarray(state[key], dtype=np.float32)
    nb = len(arr["body_inv_mass"])
    ndyn = int((arr["body_inv_mass"] > 0).sum())
    t0 = time.perf_counter()
    out = pyoracle.run(arr, frames=frames, substeps=a.substeps, dt=DT, gravity=G,
                       pgs_iterations=a.pgs, max_pairs=max(8 * nb, 10000),
                       max_contacts=max(4 * nb, 4000), threads=threads)
    secs = time.perf_counter() - t0
    return ndyn * a.substeps * frames, secs, out


def reference_arm(a, rank, world):
    """The reference's path on the host cores: the CPU restatement of
    physics.comp (the reference's own Vulkan/GLSL step cannot run here), on
    every `sample_stride`-th scene of the batch, pre-rolled on the CPU like
    the GPU arm's batch, then `warmup` + `steps` frames timed per step."""
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    d = sample_data(a, rank)
    arrays = d.arrays()
    _, _, out = oracle_frames(arrays, None, a.preroll, a, threads)
    st = {k: out[k].astype(np.float32) for k, _, _ in STATE}
    for _ in range(a.warmup):
        _, _, out = oracle_frames(arrays, st, 1, a, threads)
        st = {k: out[k].astype(np.float32) for k, _, _ in STATE}
    work, secs = 0, 0.0
    for _ in range(a.steps):
        w_, s_, out = oracle_frames(arrays, st, 1, a, threads)
        st = {k: out[k].astype(np.float32) for k, _, _ in STATE}
        work += w_
        secs += s_
    value = work / secs
    n = np.diff(d.scene_body_offset())
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": secs / a.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": workload_config(a, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"every {a.sample_stride}th of the {a.scenes} scenes "
                                   f"({len(n)} scenes, mean {n.mean():.1f} bodies per scene "
                                   f"against {d_batch_mean(a):.1f} in the batch), pre-rolled "
                                   f"{a.preroll} frames on the CPU, {a.steps} frames timed, "
                                   f"OpenMP over scenes"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("reference GLSL/Vulkan step unavailable on this box (no graphics stack, no Zig "
                 "toolchain); timed its CPU restatement"),
    }
    print(json.dumps(line))
    return 0


def d_batch_mean(a):
    from seevr_b200 import Data

    d = Data.batch(num_scenes=a.scenes, min_bodies=a.min_bodies, max_bodies=a.max_bodies,
                   segments=a.segments, seed_base=0)
    return float(np.diff(d.scene_body_offset()).mean())


# ---------------------------------------------------------------------------
def read_state(buf, nb):
    return {k: buf[n][: nb * c].cpu().numpy().reshape(nb, c).copy() for k, n, c in STATE}


def ours(a, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from seevr_b200 import (FLAG_CUDA_GRAPH, Caps, Data, Physics, Profile, STAGE_NAMES,
                            make_params)

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    d = Data.batch(num_scenes=a.scenes, min_bodies=a.min_bodies, max_bodies=a.max_bodies,
                   segments=a.segments, seed_base=rank * a.scenes)
    nb, nhv, nv, ndyn = d.num_bodies, d.num_hull_verts, d.num_vertices, d.num_dynamic
    off = d.scene_body_offset()
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    buf = d.upload(dev, caps)
    ph = Physics(buf, make_params(pgs_iterations=a.pgs, flags=FLAG_CUDA_GRAPH,
                                  bundle_bodies=a.bundle_bodies))
    if a.scene_groups:
        ph.set_tuning(**(ph.get_tuning() | {"scene_groups": a.scene_groups}))
    stream = torch.cuda.Stream(dev)

    def frames(n):
        ph.step_async(nb, nv, nhv, a.substeps, DT, G, frames=n, stream=stream)

    # pre-roll (untimed) and warm-up
    with torch.cuda.stream(stream):
        frames(a.preroll)
    stream.synchronize()
    if a.autotune:  # launch shapes timed on the settled state (restored afterwards)
        from seevr_b200.tune import autotune
        autotune(ph, buf, a.substeps, DT, G, frames=2, repeats=2)
    frames(a.warmup)
    stream.synchronize()
    t0_state = read_state(buf, nb)  # the state the timed region starts from

    # ---- timed region: K graph replays, CUDA events on the launching stream
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ph.kernel_launches
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        frames(a.steps)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = ph.kernel_launches - launches0
    flags = ph.read_flags()
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    work = torch.tensor([float(ndyn)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(work, op=dist.ReduceOp.SUM)
    ms_max = float(t.item())
    total_dyn = float(work.item())
    value = total_dyn * a.substeps * a.steps / (ms_max / 1e3)
    ms_per_step = ms_max / a.steps
    pairs, contacts = ph.read_counters()
    end_state = read_state(buf, nb)

    # ---- e2e: the same K frames from the same state through the C ABI,
    # the state copied in from pinned host memory and back out every frame
    # (seevr_physics_step_io, the host waiting for each frame's state), and
    # the same with three separate calls (upload_state, step_async,
    # download_state)
    def e2e_frame(one_call, host):
        if one_call:
            ph.step_io(nb, nv, nhv, a.substeps, DT, G, inputs=host, outputs=host)
        else:
            ph.upload_state(nb, host["pos"], host["quat"], host["vel"], host["omega"])
            ph.step_async(nb, nv, nhv, a.substeps, DT, G, frames=1)
            ph.download_state(nb, host["pos"], host["quat"], host["vel"], host["omega"])

    def e2e_run(one_call):
        host = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)).pin_memory()
                for k, v in t0_state.items()}
        # one untimed frame captures the frame graph with these host arrays;
        # the arrays are then reset (the four arrays are the whole state the
        # frame reads from the host)
        e2e_frame(one_call, host)
        torch.cuda.synchronize()
        for k, v in t0_state.items():
            host[k].copy_(torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        tw = time.perf_counter()
        for _ in range(a.steps):
            e2e_frame(one_call, host)
        e2e_s = time.perf_counter() - tw
        et = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        same = all(np.array_equal(host[k].numpy(), end_state[k]) for k in host)
        return total_dyn * a.substeps * a.steps / float(et.item()), same, host

    e2e_sep, e2e_sep_same, _ = e2e_run(False)
    e2e_value, e2e_same, host = e2e_run(True)
    h2d = d2h = sum(host[k].numel() * 4 for k in host)

    # ---- per-stage device times of one frame (profiling mode, separate
    # handle with the timed handle's launch shapes and scene groups, whose
    # stages then run one group after another; the state continues from the
    # end of the e2e frames)
    ph_prof = Physics(buf, make_params(pgs_iterations=a.pgs, bundle_bodies=a.bundle_bodies))
    ph_prof.set_tuning(**ph.get_tuning())
    prof = Profile()
    for _ in range(a.prof_frames):
        ph_prof.step(nb, nv, nhv, a.substeps, DT, G, prof)
    ph_prof.deinit()
    stage_ms = {STAGE_NAMES[i]: prof.ms[i] / a.prof_frames for i in range(len(STAGE_NAMES))}
    tuning = ph.get_tuning()
    ph.deinit()

    peak, peak_kind = measured_peaks()
    roof = roofline(stage_ms, ms_per_step, nb, nhv, nv, pairs, contacts, a.substeps, peak,
                    peak_kind, a)

    extras = {}
    if rank == 0:
        if a.plain_scenes > 0:
            extras["plain"] = plain_dropin(a, d, t0_state, dev)
        if world == 1 and not a.no_cpu_baseline:
            extras["cpu_baseline"], extras["parity"] = cpu_baseline(a, off, t0_state, dev, rank)
        if world == 1 and not a.no_config0:
            extras["config0"] = config0_leg(a, dev)
        if world == 1 and not a.no_config1:
            extras["config1"] = config1_leg(a, dev)
        if world == 1 and not a.no_raytrace:
            extras["raytrace"] = raytrace_leg(a, dev)
    del buf
    torch.cuda.empty_cache()
    adj = None if a.no_adjoint else adjoint_leg(a, rank, world, dev)
    tow = None if a.no_towers or world > 1 else towers_leg(a, rank, world, dev)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded splitmix64 scenes)",
            "config": workload_config(a, world),
            "tuning": tuning | {"autotuned": bool(a.autotune)},
            "bodies": nb, "dynamic_bodies": ndyn, "hull_verts": nhv, "render_verts": nv,
            "clocks": clk.summary(),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "how": ("the timed region's frames from its starting state, each through "
                            "seevr_physics_step_io with pinned host arrays (copied per scene "
                            "group beside the other groups' kernels) and a wait for its "
                            "state, wall clock, max over ranks"),
                    "same_final_state_as_timed_region": e2e_same,
                    "separate_calls": {
                        "value": e2e_sep,
                        "how": "seevr_physics_upload_state / step_async / download_state per frame",
                        "same_final_state_as_timed_region": e2e_sep_same}},
            "gpu_launches": launches,
            "device_flags": flags,
            "roofline": roof,
            "cpu_baseline": extras.get("cpu_baseline"),
            "parity": extras.get("parity"),
            "plain": extras.get("plain"),
            "config0": extras.get("config0"),
            "config1": extras.get("config1"),
            "raytrace": extras.get("raytrace"),
            "adjoint": adj,
            "towers": tow,
            "stage_ms_per_frame": stage_ms,
            "stage_ms_how": ("CUDA events around each stage of one frame on a handle with the "
                             "timed handle's launch shapes, the scene groups one after another "
                             "(the timed frames overlap them, so the sum exceeds ms_per_step)"),
            "last_substep": {"pairs": pairs, "contacts": contacts},
        }
        print(json.dumps(line))
    return 0


def adjoint_leg(a, rank, world, dev):
    """Differentiable rollout: --adjoint-scenes scenes of --adjoint-bodies
    bodies (half boxes, half spheres, v and omega N(0,1), friction
    U(0.2,0.8)), --adjoint-frames frames of 10 substeps x 30 PGS iterations.
    Loss: sum over scenes of the squared distance of the scene's first
    dynamic body's final position to a target drawn in a 2 m cube.  One
    forward + backward yields every scene's gradient with respect to its
    initial velocities, angular velocities and friction coefficients."""
    import torch
    import torch.distributed as dist

    from seevr_b200 import FLAG_CUDA_GRAPH, FLAG_SKIP_RENDER_VERTS, Caps, Data, Physics, make_params
    from seevr_b200.grad import rollout

    d = Data.rollout(num_scenes=a.adjoint_scenes, bodies=a.adjoint_bodies, segments=a.segments,
                     seed_base=(1 << 32) + rank * a.adjoint_scenes)
    nb = d.num_bodies
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    buf = d.upload(dev, caps)
    # the forward's substeps replay a captured one-substep graph
    ph = Physics(buf, make_params(pgs_iterations=a.pgs, flags=FLAG_SKIP_RENDER_VERTS | FLAG_CUDA_GRAPH,
                                  bundle_bodies=a.adjoint_bodies + 1))
    off = d.scene_body_offset()
    first = torch.tensor(off[:-1].astype(np.int64) + 1, device=dev)  # body 0 is the ground
    rng = np.random.default_rng(7 + rank)
    target = torch.tensor(rng.uniform(-1.0, 1.0, (a.adjoint_scenes, 3)) + [0.0, 1.0, 0.0],
                          dtype=torch.float32, device=dev)
    t = buf.tensors
    init = {k: t[n][: nb * c].clone().reshape(nb, c) for k, n, c in STATE}
    fr0 = t["geom_friction"][:nb].clone()

    def one(frames):
        v0 = init["vel"].clone().requires_grad_()
        w0 = init["omega"].clone().requires_grad_()
        mu = fr0.clone().requires_grad_()
        pos, _, _, _ = rollout(ph, init["pos"], init["quat"], v0, w0, mu, frames=frames,
                               substeps=a.substeps, dt=DT, gravity=G)
        loss = ((pos[first] - target) ** 2).sum()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loss.backward()
        torch.cuda.synchronize()
        return t1, v0.grad, w0.grad, mu.grad

    one(1)  # warm-up: work arrays, first-call paths
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record()
    t1, gv, gw, gmu = one(a.adjoint_frames)
    e1.record()
    e1.synchronize()
    fwd_s, bwd_s = t1 - t0, time.perf_counter() - t1
    ms = e0.elapsed_time(e1)
    tt = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    total = a.adjoint_scenes * world
    finite = bool(torch.isfinite(gv).all() and torch.isfinite(gw).all() and
                  torch.isfinite(gmu).all())
    ph.deinit()
    return {
        "value": total / (float(tt.item()) / 1e3), "unit": "scene-gradients/s",
        "scenes": total, "bodies_per_scene": a.adjoint_bodies + 1,
        "frames": a.adjoint_frames, "substeps": a.substeps, "pgs_iterations": a.pgs,
        "forward_s": fwd_s, "backward_s": bwd_s, "grads_finite": finite,
        "wrt": "initial velocities, angular velocities, friction",
        "timing": "CUDA events around one forward + backward, max over ranks",
    }


def towers_leg(a, rank, world, dev):
    """Stacked boxes: --towers towers of --tower-height unit boxes (jitter
    N(0, 0.01) m, friction 0.6, no restitution, each box sunk
    --tower-overlap m into the one below so that every stack contact exists
    from the first substep) on one static ground, one scene, LBVH
    broadphase, island-parallel PGS, 10 substeps x 30 iterations per frame.
    Coloured order runs --tower-frames frames, timed in segments of 20
    frames (the towers sink, merge into heaps that the grid-wide coloured
    solve takes, and collapse); wavefront (= sequential) order runs the
    first --tower-wavefront-frames frames, where both orders still see the
    same stacks, since after the collapse one warp per island takes about
    two seconds per frame.  Throughput, contacts and the tower tops'
    drift for both."""
    import torch

    from seevr_b200 import (BROADPHASE_LBVH, FLAG_CUDA_GRAPH, FLAG_SKIP_RENDER_VERTS, Caps, Data,
                            Physics, SOLVER_COLORED, SOLVER_WAVEFRONT, make_params)

    h = a.tower_height
    d = Data.towers(seed=rank, towers=a.towers, height=h, spacing=2.0, overlap=a.tower_overlap)
    nb, nhv = d.num_bodies, d.num_hull_verts
    caps = Caps.for_data(d, pairs_per_body=4.0, contacts_per_body=4.0)
    buf = d.upload(dev, caps)
    init = {k: buf.tensors[k].clone() for k in ("body_pos", "body_quat", "body_vel", "body_omega")}
    tops = torch.arange(a.towers, device=dev) * h + h  # top box of each tower (body 0: ground)
    top0 = init["body_pos"].reshape(-1, 3)[tops, 1].clone()
    stream = torch.cuda.Stream(dev)
    out = {}
    for name, solver, frames in (("coloured", SOLVER_COLORED, a.tower_frames),
                                 ("wavefront", SOLVER_WAVEFRONT, a.tower_wavefront_frames)):
        for k, v in init.items():
            buf.tensors[k].copy_(v)
        ph = Physics(buf, make_params(pgs_iterations=a.pgs, solver=solver,
                                      broadphase=BROADPHASE_LBVH,
                                      flags=FLAG_CUDA_GRAPH | FLAG_SKIP_RENDER_VERTS))
        torch.cuda.synchronize()
        ph.step_async(nb, 0, nhv, a.substeps, DT, G, frames=1, stream=stream)  # capture
        stream.synchronize()
        c_first = ph.read_counters()[1]
        for k, v in init.items():
            buf.tensors[k].copy_(v)
        torch.cuda.synchronize()
        seg, segments, flags, total = 20, [], 0, 0.0
        for f0 in range(0, frames, seg):
            n = min(seg, frames - f0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ph.step_async(nb, 0, nhv, a.substeps, DT, G, frames=n, stream=stream)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            total += ms
            flags |= ph.read_flags()
            segments.append({"frames": f"{f0 + 1}-{f0 + n}", "ms_per_frame": ms / n,
                             "contacts_last_substep": ph.read_counters()[1]})
        top = buf.tensors["body_pos"][: nb * 3].reshape(-1, 3)[tops, 1]
        drift = (top - top0).abs()
        rate = lambda ms_pf: (nb - 1) * a.substeps / (ms_pf / 1e3)
        out[name] = {"value": (nb - 1) * a.substeps * frames / (total / 1e3), "frames": frames,
                     "ms_per_frame": total / frames,
                     "first_segment_rate": rate(segments[0]["ms_per_frame"]),
                     "last_segment_rate": rate(segments[-1]["ms_per_frame"]),
                     "slowest_segment_rate": rate(max(x["ms_per_frame"] for x in segments)),
                     "segments": segments,
                     "contacts_first_frame": c_first,
                     "top_drift_mean_m": float(drift.mean()),
                     "top_drift_max_m": float(drift.max()),
                     "towers_standing": int((drift < 0.5).sum()),
                     "finite": bool(torch.isfinite(buf.tensors["body_pos"][: nb * 3]).all()),
                     "device_flags": flags,
                     "grid_solved_giant_islands": bool(flags & 32)}
        ph.deinit()
    return {"unit": UNIT, "bodies": nb, "towers": a.towers, "height": h,
            "overlap_m": a.tower_overlap, "substeps": a.substeps,
            "pgs_iterations": a.pgs, "broadphase": "LBVH",
            "solver_work": "islands: a warp each, islands above 4,096 contacts grid-wide "
                           "(coloured order)",
            "contact_model": "one MPR contact per touching pair (physics.comp:475-491)",
            "note": "PGS passes support one box up a stack per iteration: 256-box towers sink "
                    "and collapse under either order", **out}


def plain_dropin(a, d, state, dev):
    """Plain single-scene step (the Physics.step drop-in, synchronous) looped
    over the first scenes; also the state error of the batched step against
    it after one frame from the same state."""
    import torch

    from seevr_b200 import Caps, Data, Physics, make_params

    off = d.scene_body_offset()
    n = min(a.plain_scenes, a.scenes)
    # the batched step over the same scenes for one frame, from `state`
    sub_batch = Data.batch(num_scenes=n, min_bodies=a.min_bodies, max_bodies=a.max_bodies,
                           segments=a.segments, seed_base=0)
    b1 = int(off[n])
    bbuf = sub_batch.upload(dev)
    for key, name, c in STATE:
        bbuf[name][: b1 * c].copy_(torch.from_numpy(state[key][:b1].reshape(-1)))
    bph = Physics(bbuf, make_params(pgs_iterations=a.pgs))
    bph.step(b1, sub_batch.num_vertices, sub_batch.num_hull_verts, a.substeps, DT, G)
    batched_pos = bbuf["body_pos"][: b1 * 3].cpu().numpy().reshape(-1, 3)
    batched_vel = bbuf["body_vel"][: b1 * 3].cpu().numpy().reshape(-1, 3)
    bph.deinit()

    total_ms, work, err = 0.0, 0, 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for s in range(n):
        one = Data.batch(num_scenes=1, min_bodies=a.min_bodies, max_bodies=a.max_bodies,
                         segments=a.segments, seed_base=s)
        lo, hi = int(off[s]), int(off[s + 1])
        buf = one.upload(dev, Caps.for_data(one))
        for key, name, c in STATE:
            buf[name][: (hi - lo) * c].copy_(torch.from_numpy(state[key][lo:hi].reshape(-1)))
        ph = Physics(buf, make_params(pgs_iterations=a.pgs))
        ph.step(hi - lo, one.num_vertices, one.num_hull_verts, a.substeps, DT, G)  # warm
        for key, name, c in STATE:
            buf[name][: (hi - lo) * c].copy_(torch.from_numpy(state[key][lo:hi].reshape(-1)))
        torch.cuda.synchronize()
        e0.record(torch.cuda.current_stream())
        ph.step(hi - lo, one.num_vertices, one.num_hull_verts, a.substeps, DT, G)
        e1.record(torch.cuda.current_stream())
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        work += one.num_dynamic * a.substeps
        pos = buf["body_pos"][: (hi - lo) * 3].cpu().numpy().reshape(-1, 3)
        vel = buf["body_vel"][: (hi - lo) * 3].cpu().numpy().reshape(-1, 3)
        scale = max(np.abs(pos).max(), 1e-30)
        err = max(err, float(np.abs(pos - batched_pos[lo:hi]).max() / scale),
                  float(np.abs(vel - batched_vel[lo:hi]).max() / max(np.abs(vel).max(), 1e-30)))
        ph.deinit()
    return {"value": work / (total_ms / 1e3), "unit": UNIT, "scenes": n,
            "how": "one handle per scene, synchronous Physics.step, looped over scenes",
            "batched_vs_plain_max_rel_state_err": err}


# Figures of single-kernel ncu captures (not measured by this run): per
# main kernel of each stage, DRAM bytes (read + write) per launch and issue
# and warp utilisation, captured on a 1,024-scene batch of the same
# distributions (123,288 bodies, 118,480 pairs and 28,231 contacts at the
# captured substep) and scaled to a run by its bodies (body stage,
# broadphase, solver, render vertices) or pairs (narrowphase).  Captured as
#   ncu --metrics <NCU_METRICS> --clock-control none -k regex:<kernel>
#       -s <pre-roll and warm-up launches> -c 2 --csv <NCU_SMALL>
# after the same command exited 0 without ncu; each figure is the mean of
# the two captured launches.
NCU_SMALL = ("python bench.py --scenes 1024 --steps 2 --warmup 1 --preroll 90 --no-cpu-baseline "
             "--no-adjoint --no-towers --no-config0 --no-config1 --no-raytrace --plain-scenes 0 "
             "--no-autotune --prof-frames 1")
NCU_METRICS = ("gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum,"
               "sm__inst_executed.sum,sm__issue_active.avg.pct_of_peak_sustained_elapsed,"
               "sm__warps_active.avg.pct_of_peak_sustained_active,"
               "smsp__thread_inst_executed_per_inst_executed.ratio,lts__t_sector_hit_rate.pct,"
               "l1tex__t_sector_hit_rate.pct,launch__registers_per_thread,"
               "gpu__dram_throughput.avg.pct_of_peak_sustained_elapsed")
NCU_CAPTURED = {"bodies": 123288, "pairs": 118480, "contacts": 28231}
NCU_CAPTURE = {
    "phys/aabb": {"kernel": "k_body_stage", "skip": 1001, "scale": "bodies",
                  "dram_bytes_per_launch": 247286528, "duration_us": 60.2,
                  "issue_active_pct": 44.7, "warps_active_pct": 38.1, "lanes_per_inst": 27.9,
                  "registers": 64},
    "phys/broad_phase": {"kernel": "k_broad_tile<0> + k_broad_tile<1>", "skip": 1820,
                         "scale": "bodies", "dram_bytes_per_launch": 10507520,
                         "duration_us": 56.8, "issue_active_pct": 40.5,
                         "warps_active_pct": 56.3, "lanes_per_inst": 29.5, "registers": 63},
    "phys/narrow_phase": {"kernel": "k_narrow<0, 7>", "skip": 910, "scale": "pairs",
                          "dram_bytes_per_launch": 96512384, "duration_us": 128.1,
                          "issue_active_pct": 33.5, "warps_active_pct": 32.8,
                          "lanes_per_inst": 8.1, "registers": 72},
    "phys/pgs_solve": {"kernel": "k_solver_warp", "skip": 910, "scale": "bodies",
                       "dram_bytes_per_launch": 10583040, "duration_us": 286.9,
                       "issue_active_pct": 9.1, "warps_active_pct": 2.8, "lanes_per_inst": 16.2,
                       "registers": 141},
    "phys/render_verts": {"kernel": "k_render_verts", "skip": 91, "scale": "bodies",
                          "dram_bytes_per_launch": 394073344, "duration_us": 98.7,
                          "issue_active_pct": 35.3, "warps_active_pct": 39.8,
                          "lanes_per_inst": 30.0, "registers": 62},
}


def ncu_scaled(stage, nb, pairs):
    """The captured DRAM bytes per launch of a stage's main kernel, scaled
    from the captured batch to this run by bodies or pairs."""
    c = NCU_CAPTURE[stage]
    f = (pairs / NCU_CAPTURED["pairs"]) if c["scale"] == "pairs" else (nb / NCU_CAPTURED["bodies"])
    return c["dram_bytes_per_launch"] * f


def roofline(stage_ms, ms_per_step, nb, nhv, nv, pairs, contacts, substeps, peak, peak_kind, a):
    """Whole-step HBM roofline (algorithmic bytes per frame over the timed
    frame) and one entry per stage with the bound that limits it.

    Algorithmic bytes per substep (the minimum traffic of each stage as the
    reference sequence moves it; pairs and contacts of the last substep):
      body stage  = integrate 84N + gravity 52N + AABB 60N + 12 per hull vertex
      broadphase  = 28N + 8P;  narrowphase = 64P + 36C;  impulse clear = 4C;
      solver      = 100N + 44C;  and per frame the render vertices 28N + 24V.
    """
    per_substep = {
        "phys/aabb": ("k_body_stage", "hbm", 196 * nb + 12 * nhv),
        "phys/broad_phase": ("k_broad_tile (count, scan, write)", "issue: compare pipe",
                             28 * nb + 8 * pairs),
        "phys/narrow_phase": ("k_narrow (+ scan, scatter)", "latency: dependent gathers, "
                              "divergence", 64 * pairs + 36 * contacts),
        "phys/clear_impulse": ("memset", "hbm", 4 * contacts),
        "phys/pgs_solve": ("k_solver_warp", "latency: dependent chain of the largest bundle",
                           100 * nb + 44 * contacts),
    }
    once = {"phys/render_verts": ("k_render_verts", "hbm", 28 * nb + 24 * nv)}
    frame_bytes = substeps * (324 * nb + 12 * nhv + 72 * pairs + 84 * contacts) + \
        28 * nb + 24 * nv
    achieved = frame_bytes / (ms_per_step / 1e3) / 1e9
    total_stage = max(sum(stage_ms.values()), 1e-9)
    stages = []
    for k, ms in sorted(stage_ms.items(), key=lambda kv: -kv[1]):
        if ms <= 0:
            continue
        kern, bound, algo = per_substep.get(k) or once.get(k) or ("", "", 0)
        launch_ms = ms / (substeps if k in per_substep else 1)
        gbs = algo / (launch_ms / 1e3) / 1e9 if launch_ms > 0 else 0.0
        e = {"stage": k, "kernel": kern, "bound": bound, "share": ms / total_stage,
             "launch_ms": launch_ms, "algorithmic_bytes_per_launch": algo,
             "achieved_gbs": gbs, "hbm_frac": gbs / peak}
        if k in NCU_CAPTURE:
            e["ncu"] = dict(NCU_CAPTURE[k])
            e["ncu"]["dram_bytes_per_launch_scaled"] = ncu_scaled(k, nb, pairs)
        stages.append(e)
    # per frame: the stage kernels' captured DRAM bytes per launch, scaled to
    # this run, times their launches per frame (the impulse clear is a
    # memset of 4 bytes per contact, counted at its algorithmic size)
    traffic = sum(substeps * ncu_scaled(k, nb, pairs) for k in per_substep
                  if k in NCU_CAPTURE) + substeps * 4 * contacts + \
        ncu_scaled("phys/render_verts", nb, pairs)
    return {"bound": "hbm", "kernel": f"whole frame ({substeps} substeps + render vertices)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_kind, "traffic": traffic,
            "traffic_source": ("per frame: the stage kernels' ncu-captured DRAM bytes per launch "
                               "(stages[].ncu, a 1,024-scene capture scaled by bodies or pairs) "
                               "times their launches"),
            "traffic_over_algorithmic": traffic / frame_bytes,
            "ncu_command": f"ncu --metrics {NCU_METRICS} --clock-control none "
                           f"-k regex:<kernel> -s <skip> -c 2 --csv {NCU_SMALL}",
            "algorithmic_bytes_per_frame": frame_bytes,
            "dominant_stage": stages[0]["stage"] if stages else None,
            "stages": stages}


def cpu_baseline(a, full_off, state, dev, rank):
    """The CPU oracle on every `sample_stride`-th scene of the batch from the
    state the timed region starts from, and the CUDA path on the same scenes
    from the same state for the same frames, compared bit for bit."""
    import torch

    threads = os.cpu_count() or 1
    d = sample_data(a, rank)
    arrays = d.arrays()
    st = sample_state(a, full_off, state, rank)
    work, secs, out = oracle_frames(arrays, st, 1, a, threads)
    frames = 1
    if secs < a.cpu_seconds / 2:
        frames = max(1, min(a.steps, int(a.cpu_seconds / max(secs, 1e-3))))
        work, secs, out = oracle_frames(arrays, st, frames, a, threads)
    n = np.diff(d.scene_body_offset())
    cpu = {"value": work / secs, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"every {a.sample_stride}th of the {a.scenes} scenes ({len(n)} scenes, "
                     f"{n.sum()} bodies, {n.max()} in the largest), {frames} frame(s) from the "
                     f"state the timed region starts from, OpenMP over scenes"}
    got = gpu_frames(d, st, frames, a, dev)
    keys = ("pos", "quat", "vel", "omega", "pairs", "c_a", "c_b", "c_pos", "c_normal", "c_pen",
            "lambda")
    same = {k: bool(np.array_equal(got[k], np.asarray(out[k]).astype(got[k].dtype)))
            for k in keys}
    parity = {"scenes": int(len(n)), "bodies": int(n.sum()), "largest_scene": int(n.max()),
              "scenes_over_256_bodies": int((n > 256).sum()), "frames": frames,
              "pairs": int(out["num_pairs"]), "contacts": int(out["num_contacts"]),
              "counters_equal": (got["num_pairs"], got["num_contacts"]) ==
                                (int(out["num_pairs"]), int(out["num_contacts"])),
              "bit_exact": all(same.values()) and (got["num_pairs"], got["num_contacts"]) ==
                           (int(out["num_pairs"]), int(out["num_contacts"])),
              "keys": same,
              "against": "FP32 CPU oracle, same scenes, same starting state, same frames; "
                         "the GPU runs them as one batched CUDA-graph handle"}
    del got
    torch.cuda.empty_cache()
    return cpu, parity


def gpu_frames(d, state, frames, a, dev):
    """The batched CUDA-graph step on the scenes of `d` from `state` for
    `frames` frames; the outputs the oracle also returns."""
    import torch

    from seevr_b200 import FLAG_CUDA_GRAPH, FLAG_SKIP_RENDER_VERTS, Caps, Physics, make_params

    nb = d.num_bodies
    caps = Caps(nb, max(d.num_hull_verts, 1), max(d.num_vertices, 1), max(8 * nb, 10000),
                max(4 * nb, 4000), max(d.num_scenes, 1))
    buf = d.upload(dev, caps)
    for key, name, c in STATE:
        buf[name][: nb * c].copy_(torch.from_numpy(np.ascontiguousarray(state[key]).reshape(-1)))
    ph = Physics(buf, make_params(pgs_iterations=a.pgs, bundle_bodies=a.bundle_bodies,
                                  flags=FLAG_CUDA_GRAPH | FLAG_SKIP_RENDER_VERTS))
    ph.step_async(nb, 0, d.num_hull_verts, a.substeps, DT, G, frames=frames)
    torch.cuda.synchronize()
    ph.deinit()
    t = buf.tensors
    cnt = t["counters"][:2].cpu().numpy().view(np.uint32)
    npairs, nc = int(min(cnt[0], caps.max_pairs)), int(min(cnt[1], caps.max_contacts))
    out = read_state(buf, nb)
    out.update({
        "num_pairs": int(cnt[0]), "num_contacts": int(cnt[1]),
        "pairs": t["collision_pairs"][: npairs * 2].cpu().numpy().view(np.uint32).reshape(-1, 2),
        "c_pos": t["contact_pos"][: nc * 3].cpu().numpy().reshape(-1, 3),
        "c_normal": t["contact_normal"][: nc * 3].cpu().numpy().reshape(-1, 3),
        "c_pen": t["contact_pen"][:nc].cpu().numpy(),
        "lambda": t["lambda_n"][:nc].cpu().numpy(),
        "c_a": t["contact_geom_a"][:nc].cpu().numpy().view(np.uint32),
        "c_b": t["contact_geom_b"][:nc].cpu().numpy().view(np.uint32),
    })
    return out


def config0_leg(a, dev):
    """The plain drop-in scene: 256 boxes + 256 16-segment spheres on the
    ground (seed 0), 120 frames of synchronous Physics.step at the
    reference's 4 and at 30 PGS iterations, beside the single-threaded CPU
    oracle over the same frames; the final states are compared."""
    import torch

    from seevr_b200 import FLAG_CUDA_GRAPH, Caps, Data, Physics, make_params

    out = {"scene": "256 boxes + 256 spheres (16 segments), seed 0, ground box",
           "frames": a.config0_frames,
           "how": "synchronous Physics.step per frame (the drop-in), replaying the frame's CUDA "
                  "graph (gpu) and launching each kernel (gpu_eager)"}
    d = Data.pile(seed=0)
    caps = Caps.for_data(d)
    for pgs in (4, 30):
        b = dict(a.__dict__)
        b["pgs"] = pgs
        work, secs, ref = oracle_frames(d.arrays(), None, a.config0_frames,
                                        argparse.Namespace(**b), 1)
        res = {"cpu_oracle_1_thread": work / secs, "unit": UNIT}
        for key, flags in (("gpu", FLAG_CUDA_GRAPH), ("gpu_eager", 0)):
            buf = d.upload(dev, caps)
            nb, nv, nhv = buf.num_bodies, buf.num_vertices, buf.num_hull_verts
            ph = Physics(buf, make_params(pgs_iterations=pgs, flags=flags))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(a.config0_frames):
                ph.step(nb, nv, nhv, a.substeps, DT, G)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            pairs, contacts = ph.read_counters()
            gpu_state = read_state(buf, nb)
            ph.deinit()
            exact = all(np.array_equal(gpu_state[k], ref[k].astype(np.float32)) for k, _, _ in STATE)
            res[key] = work / (ms / 1e3)
            res[f"{key}_ms_per_frame"] = ms / a.config0_frames
            res[f"{key}_final_state_bit_exact"] = bool(exact)
            res["pairs_last_substep"], res["contacts_last_substep"] = pairs, contacts
            del buf
        out[f"pgs{pgs}"] = res
    return out


def config1_leg(a, dev):
    """The large scene: --config1-bodies bodies (40% boxes, 40% spheres, 20%
    hulls of 16-32 points) in a 64 m cube with velocities N(0,1), stepped
    --config1-frames frames with the LBVH broadphase and with the all-pairs
    broadphase from the same state: time per frame and per stage, and the
    final pair lists and states compared."""
    import torch

    from seevr_b200 import (BROADPHASE_LBVH, BROADPHASE_N2, FLAG_CUDA_GRAPH, Caps, Data, Physics,
                            Profile, STAGE_NAMES, make_params)

    d = Data.large(seed=0, n_bodies=a.config1_bodies)
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    out = {"bodies": d.num_bodies, "frames": a.config1_frames,
           "scene": "40% boxes, 40% 16-segment spheres, 20% hulls of 16-32 points, 64 m cube, "
                    "v N(0,1), seed 0"}
    res = {}
    for name, bp in (("lbvh", BROADPHASE_LBVH), ("all_pairs", BROADPHASE_N2)):
        buf = d.upload(dev, caps)
        nb, nv, nhv = buf.num_bodies, buf.num_vertices, buf.num_hull_verts
        ph = Physics(buf, make_params(pgs_iterations=a.pgs, broadphase=bp, flags=FLAG_CUDA_GRAPH))
        stream = torch.cuda.Stream(dev)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ph.step_async(nb, nv, nhv, a.substeps, DT, G, frames=a.config1_frames, stream=stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)  # includes the graph capture of the first frame
        pairs, contacts = ph.read_counters()
        st = read_state(buf, nb)
        pl = buf["collision_pairs"][: min(pairs, caps.max_pairs) * 2].cpu().numpy().copy()
        ph.deinit()
        # per-stage times of one more frame in profiling mode
        php = Physics(buf, make_params(pgs_iterations=a.pgs, broadphase=bp))
        prof = Profile()
        php.step(nb, nv, nhv, a.substeps, DT, G, prof)
        php.deinit()
        res[name] = (st, pl)
        out[name] = {"value": d.num_dynamic * a.substeps * a.config1_frames / (ms / 1e3),
                     "unit": UNIT, "ms_per_frame": ms / a.config1_frames,
                     "pairs_last_substep": pairs, "contacts_last_substep": contacts,
                     "stage_ms_next_frame": {STAGE_NAMES[i]: prof.ms[i]
                                             for i in range(len(STAGE_NAMES)) if prof.ms[i] > 0}}
        del buf
        torch.cuda.empty_cache()
    out["pair_lists_equal"] = bool(np.array_equal(res["lbvh"][1], res["all_pairs"][1]))
    out["states_equal"] = all(np.array_equal(res["lbvh"][0][k], res["all_pairs"][0][k])
                              for k, _, _ in STATE)
    return out


def raytrace_leg(a, dev):
    """Raytrace mode on the 512-body drop-in scene after 60 settling frames:
    the triangle LBVH build of its render mesh (BVH.build) and frames of the
    path tracer (16 samples per pixel, up to 16 bounces, raytrace.comp),
    CUDA events around each."""
    import torch

    from seevr_b200 import Caps, Data, Physics, make_params
    from seevr_b200 import _lib as L
    from seevr_b200.bvh import BVH
    from seevr_b200.raytrace import Raytracer

    d = Data.pile(seed=0)
    buf = d.upload(dev, Caps.for_data(d))
    ph = Physics(buf, make_params(pgs_iterations=a.pgs))
    for _ in range(60):
        ph.step(buf.num_bodies, buf.num_vertices, buf.num_hull_verts, a.substeps, DT, G)
    ph.deinit()
    arr = d.arrays()
    ntri = len(arr["indices"])
    verts = buf["vertices"][: buf.num_vertices * 3].clone()
    idx = torch.tensor(arr["indices"].reshape(-1).view(np.int32), device=dev)
    bvh = BVH(verts, idx)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    bvh.build(ntri)  # warm-up
    torch.cuda.synchronize()
    e0.record()
    for _ in range(5):
        bvh.build(ntri)
    e1.record()
    e1.synchronize()
    build_ms = e0.elapsed_time(e1) / 5
    w, h = a.rt_width, a.rt_height
    rt = Raytracer(d, bvh, w, h)
    cam = np.array([0.0, 12.0, 24.0, 0.0, -0.35, -1.0, 1.0, 0.0, 0.0, 0.0, 1.0, -0.35], np.float32)
    cam[3:6] /= np.linalg.norm(cam[3:6])
    cam[9:12] /= np.linalg.norm(cam[9:12])
    rt.render(cam[0:3], cam[3:6], cam[6:9], cam[9:12], ntri)  # warm-up
    torch.cuda.synchronize()
    frames = 5
    e0.record()
    for _ in range(frames):
        rt.render(cam[0:3], cam[3:6], cam[6:9], cam[9:12], ntri)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / frames
    finite = bool(torch.isfinite(rt.image).all())
    bvh.deinit()
    return {"triangles": ntri, "bvh_build_ms": build_ms,
            "bvh_triangles_per_s": ntri / (build_ms / 1e3),
            "width": w, "height": h, "samples_per_pixel": 16, "max_bounces": 16,
            "frame_ms": ms, "pixel_samples_per_s": w * h * 16 / (ms / 1e3),
            "image_finite": finite,
            "scene": "the 512-body drop-in scene after 60 frames, its render mesh "
                     f"(fov scale {L.lib.seevr_raytrace_fov_scale():.6f})"}


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return reference_arm(a, rank, world)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        return ours(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
