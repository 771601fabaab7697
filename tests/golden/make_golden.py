"""Regenerate the golden fixtures in this folder from the CPU oracle.

The reference (seeVR's physics.comp, dispatched from Zig) has no tests or
golden vectors of its own and cannot run here, so these fixtures pin this
project's own chain instead: the seeded scene generator (data.zig's
builders) and the FP32 oracle (physics.comp restated).  A change to either
that alters any result shows up as a mismatch, and the GPU parity test
checks the CUDA path against the same files.

    python tests/golden/make_golden.py      # rewrites the .npz files
"""
import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

DT = 1.0 / 60.0
G = (0.0, -9.81, 0.0)

# name -> (scene factory, frames, PGS iterations): a low pile (the scene of
# a GPU parity test) and a batch of 12 scenes, both run until contacts form
CASES = {
    "lowpile48_30frames_pgs10": (
        lambda Data: Data.pile(seed=5, n_boxes=24, n_spheres=24, lo=(-3, 0, -3), hi=(3, 3.0, 3)),
        30, 10),
    "batch12_60frames_pgs10": (
        lambda Data: Data.batch(num_scenes=12, min_bodies=8, max_bodies=48, seed_base=41), 60, 10),
}
KEYS = ("pos", "quat", "vel", "omega", "pairs", "c_a", "c_b", "c_pos", "c_normal", "c_pen",
        "lambda")


def scene_digest(arrays: dict) -> str:
    h = hashlib.sha256()
    for k in sorted(arrays):
        h.update(k.encode())
        h.update(np.ascontiguousarray(arrays[k]).tobytes())
    return h.hexdigest()


def run_case(name):
    import pyoracle
    from seevr_b200 import Caps, Data

    make, frames, pgs = CASES[name]
    d = make(Data)
    caps = Caps.for_data(d)
    arrays = d.arrays()
    r = pyoracle.run(arrays, frames=frames, substeps=10, dt=DT, gravity=G, pgs_iterations=pgs,
                     max_pairs=caps.max_pairs, max_contacts=caps.max_contacts)
    out = {}
    for k in KEYS:
        x = np.asarray(r[k])
        if x.dtype.kind == "f":  # FP32 results held in doubles: narrowing is exact
            x32 = x.astype(np.float32)
            assert np.array_equal(x32.astype(x.dtype), x), k
            x = x32
        out[k] = x
    out["num_pairs"] = np.asarray(r["num_pairs"])
    out["num_contacts"] = np.asarray(r["num_contacts"])
    out["scene_sha256"] = np.asarray(scene_digest(arrays))
    return d, caps, out


def main():
    for name in CASES:
        _, _, out = run_case(name)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
