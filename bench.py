"""Benchmark of the physics step: body-substeps/s of the batched CUDA-graph
step over 4,096 independent scenes, beside the plain single-scene drop-in
looped per scene and the CPU oracle.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one frame (Physics.step: 10 substeps, 30 PGS iterations) of the
whole batch.  The scenes are pre-rolled (--preroll frames, untimed) so the
timed frames contain a settling pile rather than free fall.  Under torchrun
each rank runs its own 4,096 scenes (weak scaling, no collective in the
step); rank 0 prints one JSON line.
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
    ap.add_argument("--plain-scenes", type=int, default=32)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adjoint-scenes", type=int, default=1024)
    ap.add_argument("--adjoint-bodies", type=int, default=64)
    ap.add_argument("--adjoint-frames", type=int, default=60)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--towers", type=int, default=1024)
    ap.add_argument("--tower-height", type=int, default=256)
    ap.add_argument("--tower-frames", type=int, default=20)
    ap.add_argument("--no-towers", action="store_true")
    ap.add_argument("--prof-frames", type=int, default=3)
    ap.add_argument("--bundle-bodies", type=int, default=0,
                    help="solver bundle size in bodies (0: the library default)")
    ap.add_argument("--autotune", action="store_true",
                    help="time launch shapes on the settled state and use the fastest")
    return ap.parse_args()


def workload_config(a, nb, ndyn, nhv, nv):
    return {
        "workload": (f"batched scenes: {a.scenes} independent scenes per GPU, dynamic bodies "
                     f"log-uniform {a.min_bodies}-{a.max_bodies} (half boxes with half-extents "
                     f"U(0.2,0.6) m, half {a.segments}-segment UV spheres r U(0.2,0.5) m) on a "
                     f"static ground box, {a.substeps} substeps x {a.pgs} PGS iterations per "
                     f"60 Hz frame, after {a.preroll} untimed frames of settling"),
        "scenes": a.scenes, "bodies": nb, "dynamic_bodies": ndyn, "hull_verts": nhv,
        "render_verts": nv, "substeps": a.substeps, "pgs_iterations": a.pgs,
        "preroll_frames": a.preroll, "dt": DT,
        "l2": f"inputs larger than L2: {nhv * 12 / 1e6:.0f} MB of hull vertices read per substep",
        "broadphase": "all-pairs per scene", "solver": "wavefront (bit-identical to sequential)",
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
def oracle_sample(arrays, scenes, frames, a, threads):
    """Run the CPU oracle on the first `scenes` scenes for `frames` frames;
    returns (dynamic body-substeps, seconds, out)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    off = arrays["scene_body_offset"]
    b1 = int(off[scenes])
    hr = arrays["hull_range"]
    h0, h1 = 0, int(hr[b1 - 1][0] + hr[b1 - 1][1])
    vs, vc = arrays["body_vert_start"], arrays["body_vert_count"]
    v1 = int(vs[b1 - 1] + vc[b1 - 1])
    sub = {}
    for k, v in arrays.items():
        if k in ("hull_verts",):
            sub[k] = v[h0:h1]
        elif k in ("orig_vertices", "vertices", "colors"):
            sub[k] = v[:v1]
        elif k in ("support_lookup", "indices"):
            sub[k] = v
        elif k == "scene_body_offset":
            sub[k] = off[: scenes + 1]
        elif len(v) == len(arrays["body_inv_mass"]):
            sub[k] = v[:b1]
        else:
            sub[k] = v
    ndyn = int((sub["body_inv_mass"] > 0).sum())
    t0 = time.perf_counter()
    out = pyoracle.run(sub, frames=frames, substeps=a.substeps, dt=DT, gravity=G,
                       pgs_iterations=a.pgs, max_pairs=max(16 * b1, 10000),
                       max_contacts=max(8 * b1, 4000), threads=threads)
    dt = time.perf_counter() - t0
    return ndyn * a.substeps * frames, dt, out


def reference_arm(a, rank, world):
    """The reference's path on the host cores: the CPU restatement of
    physics.comp (the reference's own Vulkan/GLSL step cannot run here)."""
    if rank != 0:
        return 0
    from seevr_b200 import Data

    threads = os.cpu_count() or 1
    d = Data.batch(num_scenes=a.scenes, min_bodies=a.min_bodies, max_bodies=a.max_bodies,
                   segments=a.segments, seed_base=0)
    arrays = d.arrays()
    scenes = max(8, min(a.scenes, 2 * threads))
    # pre-roll the sample like the GPU arm, then time `steps` frames
    _, _, out = oracle_sample(arrays, scenes, a.preroll, a, threads)
    st = dict(arrays)
    b1 = int(arrays["scene_body_offset"][scenes])
    for key, name in (("pos", "body_pos"), ("quat", "body_quat"), ("vel", "body_vel"),
                      ("omega", "body_omega")):
        x = arrays[name].copy()
        x[:b1] = out[key].astype(np.float32)
        st[name] = x
    for _ in range(a.warmup):
        oracle_sample(st, scenes, 1, a, threads)
    work, secs, _ = oracle_sample(st, scenes, a.steps, a, threads)
    value = work / secs
    nb = d.num_bodies
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": secs / a.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": workload_config(a, nb, d.num_dynamic, d.num_hull_verts, d.num_vertices),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"first {scenes} of {a.scenes} scenes, {a.steps} frames after "
                                   f"{a.preroll} pre-roll frames, one OpenMP thread per scene"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("reference GLSL/Vulkan step unavailable on this box (no graphics stack, no Zig "
                 "toolchain); timed its CPU restatement"),
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
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
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    buf = d.upload(dev, caps)
    ph = Physics(buf, make_params(pgs_iterations=a.pgs, flags=FLAG_CUDA_GRAPH, bundle_bodies=a.bundle_bodies))
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
    pre_state = {k: buf[n][: nb * c].cpu().numpy().reshape(nb, c) for k, n, c in (
        ("pos", "body_pos", 3), ("quat", "body_quat", 4), ("vel", "body_vel", 3),
        ("omega", "body_omega", 3))}
    frames(a.warmup)
    stream.synchronize()

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
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    work = torch.tensor([float(ndyn)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(work, op=dist.ReduceOp.SUM)
    ms_max = float(t.item())
    total_dyn = float(work.item())
    value = total_dyn * a.substeps * a.steps / (ms_max / 1e3)
    ms_per_step = ms_max / a.steps
    counters = ph.read_counters()

    # ---- per-stage device times of one frame (profiling mode)
    ph_prof = Physics(buf, make_params(pgs_iterations=a.pgs, bundle_bodies=a.bundle_bodies))
    prof = Profile()
    for _ in range(a.prof_frames):
        ph_prof.step(nb, nv, nhv, a.substeps, DT, G, prof)
    pairs, contacts = ph_prof.read_counters()
    ph_prof.deinit()
    stage_ms = {STAGE_NAMES[i]: prof.ms[i] / a.prof_frames for i in range(len(STAGE_NAMES))}

    # ---- e2e: host state in pinned memory -> device, frame, device -> host
    host = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32)).pin_memory()
            for k, v in pre_state.items()}
    ph_e2e = Physics(buf, make_params(pgs_iterations=a.pgs, flags=FLAG_CUDA_GRAPH, bundle_bodies=a.bundle_bodies))
    ph_e2e.set_tuning(**ph.get_tuning())  # the same launch shapes as the timed handle
    h2d = d2h = nb * (12 + 16 + 12 + 12)
    ph_e2e.upload_state(nb, host["pos"], host["quat"], host["vel"], host["omega"])
    ph_e2e.step_async(nb, nv, nhv, a.substeps, DT, G, frames=1)  # capture
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(a.e2e_steps):
        ph_e2e.upload_state(nb, host["pos"], host["quat"], host["vel"], host["omega"])
        ph_e2e.step_async(nb, nv, nhv, a.substeps, DT, G, frames=1)
        ph_e2e.download_state(nb, host["pos"], host["quat"], host["vel"], host["omega"])
    e2e_s = time.perf_counter() - t0
    et = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e_value = total_dyn * a.substeps * a.e2e_steps / float(et.item())
    ph_e2e.deinit()

    # ---- plain drop-in: one handle per scene, synchronous Physics.step,
    # looped over a sample of scenes from the same pre-rolled state
    plain = None
    if rank == 0 and a.plain_scenes > 0:
        plain = plain_dropin(a, d, pre_state, dev)

    # ---- roofline of the dominant stage kernel
    peak, peak_kind = measured_peaks()
    roof = roofline(stage_ms, nb, nhv, nv, pairs, contacts, a.substeps, peak, peak_kind,
                    NCU_TRAFFIC_DEFAULT if default_workload(a) else None)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a, d, pre_state)

    adj = None if a.no_adjoint else adjoint_leg(a, rank, world, dev)
    tow = None if a.no_towers or world > 1 else towers_leg(a, rank, world, dev)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded splitmix64 scenes)",
            "config": workload_config(a, nb, ndyn, nhv, nv) | {"parallelism": f"scenes x{world}",
                                                               "tuning": ph.get_tuning(),
                                                               "autotuned": bool(a.autotune)},
            "clocks": clk.summary(),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "plain": plain,
            "adjoint": adj,
            "towers": tow,
            "stage_ms_per_frame": stage_ms,
            "last_substep": {"pairs": pairs, "contacts": contacts},
        }
        print(json.dumps(line))
    ph.deinit()
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

    from seevr_b200 import Caps, Data, Physics, make_params
    from seevr_b200.grad import rollout

    d = Data.rollout(num_scenes=a.adjoint_scenes, bodies=a.adjoint_bodies, segments=a.segments,
                     seed_base=(1 << 32) + rank * a.adjoint_scenes)
    nb = d.num_bodies
    caps = Caps.for_data(d, pairs_per_body=8.0, contacts_per_body=4.0)
    buf = d.upload(dev, caps)
    ph = Physics(buf, make_params(pgs_iterations=a.pgs, flags=4,
                                  bundle_bodies=a.adjoint_bodies + 1))
    off = d.scene_body_offset()
    first = torch.tensor(off[:-1].astype(np.int64) + 1, device=dev)  # body 0 is the ground
    rng = np.random.default_rng(7 + rank)
    target = torch.tensor(rng.uniform(-1.0, 1.0, (a.adjoint_scenes, 3)) + [0.0, 1.0, 0.0],
                          dtype=torch.float32, device=dev)
    t = buf.tensors
    init = {k: t[n][: nb * c].clone().reshape(nb, c) for k, n, c in (
        ("pos", "body_pos", 3), ("quat", "body_quat", 4), ("vel", "body_vel", 3),
        ("omega", "body_omega", 3))}
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
    N(0, 0.01) m, friction 0.6, no restitution) on one static ground, one
    scene, LBVH broadphase, island-parallel PGS, --tower-frames frames of 10
    substeps x 30 iterations.  Coloured vs wavefront (= sequential) order:
    throughput and the tower tops' drift at the end."""
    import torch

    from seevr_b200 import (BROADPHASE_LBVH, FLAG_CUDA_GRAPH, FLAG_SKIP_RENDER_VERTS, Caps, Data,
                            Physics, SOLVER_COLORED, SOLVER_WAVEFRONT, make_params)

    h = a.tower_height
    d = Data.towers(seed=rank, towers=a.towers, height=h, spacing=2.0)
    nb, nhv = d.num_bodies, d.num_hull_verts
    caps = Caps.for_data(d, pairs_per_body=4.0, contacts_per_body=4.0)
    buf = d.upload(dev, caps)
    init = {k: buf.tensors[k].clone() for k in ("body_pos", "body_quat", "body_vel", "body_omega")}
    tops = torch.arange(a.towers, device=dev) * h + h  # top box of each tower (body 0: ground)
    top0 = init["body_pos"].reshape(-1, 3)[tops, 1].clone()
    stream = torch.cuda.Stream(dev)
    out = {}
    for name, solver in (("coloured", SOLVER_COLORED), ("wavefront", SOLVER_WAVEFRONT)):
        for k, v in init.items():
            buf.tensors[k].copy_(v)
        ph = Physics(buf, make_params(pgs_iterations=a.pgs, solver=solver,
                                      broadphase=BROADPHASE_LBVH,
                                      flags=FLAG_CUDA_GRAPH | FLAG_SKIP_RENDER_VERTS))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            ph.step_async(nb, 0, nhv, a.substeps, DT, G, frames=a.tower_frames, stream=stream)
            e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        flags = ph.read_flags()
        top = buf.tensors["body_pos"][: nb * 3].reshape(-1, 3)[tops, 1]
        drift = (top - top0).abs()
        out[name] = {"value": (nb - 1) * a.substeps * a.tower_frames / (ms / 1e3),
                     "ms_per_frame": ms / a.tower_frames,
                     "top_drift_mean_m": float(drift.mean()), "top_drift_max_m": float(drift.max()),
                     "finite": bool(torch.isfinite(buf.tensors["body_pos"][: nb * 3]).all()),
                     "device_flags": flags}
        ph.deinit()
    return {"unit": UNIT, "bodies": nb, "towers": a.towers, "height": h,
            "frames": a.tower_frames, "substeps": a.substeps, "pgs_iterations": a.pgs,
            "broadphase": "LBVH", "solver_work": "islands (one per tower)", **out}


def plain_dropin(a, d, pre_state, dev):
    """Plain single-scene step (the Physics.step drop-in, synchronous) looped
    over the first scenes; also the state error of the batched step against
    it after one frame from the same state."""
    import torch

    from seevr_b200 import Caps, Data, Physics, make_params

    off = d.scene_body_offset()
    n = min(a.plain_scenes, a.scenes)
    # the batched step over the same scenes for one frame, from pre_state
    sub_batch = Data.batch(num_scenes=n, min_bodies=a.min_bodies, max_bodies=a.max_bodies,
                           segments=a.segments, seed_base=0)
    b1 = int(off[n])
    bbuf = sub_batch.upload(dev)
    for key, name, c in (("pos", "body_pos", 3), ("quat", "body_quat", 4), ("vel", "body_vel", 3),
                         ("omega", "body_omega", 3)):
        bbuf[name][: b1 * c].copy_(torch.from_numpy(pre_state[key][:b1].reshape(-1)))
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
        for key, name, c in (("pos", "body_pos", 3), ("quat", "body_quat", 4),
                             ("vel", "body_vel", 3), ("omega", "body_omega", 3)):
            buf[name][: (hi - lo) * c].copy_(torch.from_numpy(pre_state[key][lo:hi].reshape(-1)))
        ph = Physics(buf, make_params(pgs_iterations=a.pgs))
        ph.step(hi - lo, one.num_vertices, one.num_hull_verts, a.substeps, DT, G)  # warm
        for key, name, c in (("pos", "body_pos", 3), ("quat", "body_quat", 4),
                             ("vel", "body_vel", 3), ("omega", "body_omega", 3)):
            buf[name][: (hi - lo) * c].copy_(torch.from_numpy(pre_state[key][lo:hi].reshape(-1)))
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


# DRAM bytes (read + write) per substep launch of each stage's main kernel,
# from one ncu capture of the default workload (4,096 scenes, bodies 8-512,
# 16-segment spheres, 10 substeps x 30 PGS iterations, 20 substeps after the
# 90-frame pre-roll: profiles/launches_batched4096.md).  Reported as
# roofline.traffic only when the bench runs that workload.
NCU_TRAFFIC_DEFAULT = {
    "phys/pgs_solve": ("k_solver_warp", 43545792),
    "phys/narrow_phase": ("k_narrow", 805700000),
    "phys/aabb": ("k_body_stage", 1023200000),
    "phys/broad_phase": ("k_broad_tile (count + write)", 37183770 + 23357722),
}


def default_workload(a):
    return (a.scenes, a.min_bodies, a.max_bodies, a.segments, a.substeps, a.pgs, a.preroll) == \
        (4096, 8, 512, 16, 10, 30, 90)


def roofline(stage_ms, nb, nhv, nv, pairs, contacts, substeps, peak, peak_kind, traffic_table=None):
    """Algorithmic bytes per launch of each stage kernel (last-substep pair and
    contact counts) over its measured time; the dominant stage is reported."""
    per_substep = {
        "phys/aabb": 196 * nb + 12 * nhv,          # integrate 84N + gravity 52N + AABB 60N+12V
        "phys/broad_phase": 28 * nb + 8 * pairs,
        "phys/narrow_phase": 64 * pairs + 36 * contacts,
        "phys/pgs_solve": 100 * nb + 44 * contacts,
        "phys/clear_impulse": 4 * contacts,
    }
    once = {"phys/render_verts": 28 * nb + 24 * nv}
    best = max(stage_ms, key=lambda k: stage_ms[k])
    t_launch = stage_ms[best] / (substeps if best in per_substep else 1)
    algo = per_substep.get(best, once.get(best, 0))
    achieved = algo / (t_launch / 1e3) / 1e9 if t_launch > 0 else 0.0
    measured = (traffic_table or {}).get(best)
    return {"bound": "hbm", "kernel": best, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind,
            "traffic": measured[1] if measured else None,
            "traffic_kernel": measured[0] if measured else None,
            "algorithmic_bytes_per_launch": algo, "launch_ms": t_launch,
            "note": "stage share of the frame: " + ", ".join(
                f"{k.split('/')[1]} {v / max(sum(stage_ms.values()), 1e-9):.0%}"
                for k, v in sorted(stage_ms.items(), key=lambda kv: -kv[1]) if v > 0)}


def cpu_baseline(a, d, pre_state):
    """The CPU oracle on a bounded sample of the same workload and state."""
    threads = os.cpu_count() or 1
    arrays = d.arrays()
    for key, name in (("pos", "body_pos"), ("quat", "body_quat"), ("vel", "body_vel"),
                      ("omega", "body_omega")):
        arrays[name] = pre_state[key].astype(np.float32)
    scenes = max(8, min(a.scenes, 2 * threads))
    work, secs, _ = oracle_sample(arrays, scenes, 1, a, threads)
    frames = 1
    if secs < a.cpu_seconds / 4:
        frames = max(1, min(10, int(a.cpu_seconds / max(secs, 1e-3))))
        work, secs, _ = oracle_sample(arrays, scenes, frames, a, threads)
    return {"value": work / secs, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {scenes} of {a.scenes} scenes, {frames} frame(s) from the same "
                      f"pre-rolled state, OpenMP over scenes"}


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
