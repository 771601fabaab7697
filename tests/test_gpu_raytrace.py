"""GPU path tracer (seevr_raytrace) against its CPU restatement, bit for bit,
on a scene that exercises every material branch of raytrace.comp: diffuse,
metal, glass (reflection, refraction, total internal reflection) and
emission, over the GPU-built triangle BVH."""
import numpy as np
import pytest
import torch

import pyoracle
from seevr_b200 import Data
from seevr_b200.bvh import BVH
from seevr_b200 import _lib as L
from seevr_b200.raytrace import Raytracer

pytestmark = pytest.mark.gpu


def showcase():
    d = Data()
    grey = d.add_material((0.7, 0.7, 0.7), 0.9, 0.0, (0, 0, 0), 0.0, 0.0)
    red = d.add_material((0.8, 0.2, 0.2), 0.4, 0.0, (0, 0, 0), 0.0, 1000.0)
    metal = d.add_material((0.9, 0.9, 0.8), 0.15, 1.0, (0, 0, 0), 0.0, 1000.0)
    glass = d.add_material((0.95, 0.95, 1.0), 0.0, 0.0, (0, 0, 0), 1.5, 1000.0)
    light = d.add_material((1, 1, 1), 0.0, 0.0, (4.0, 3.6, 3.0), 0.0, 0.0)
    d.add_box((0, -0.25, 0), (20, 0.25, 20), (0.7, 0.7, 0.7), 0.5, 0.2, grey)
    d.add_box((0, 6, -2), (2, 0.1, 2), (1, 1, 1), 0.5, 0.2, light)
    d.add_sphere((-1.2, 1.0, -1.0), 1.0, (1, 1, 1), 16, 0.5, 0.2, glass)
    d.add_box((1.5, 0.8, -2.0), (0.8, 0.8, 0.8), (1, 1, 1), 0.5, 0.2, metal)
    rng = np.random.default_rng(3)
    for i in range(12):
        c = (rng.uniform(-4, 4), rng.uniform(0.3, 0.6), rng.uniform(-6, 1))
        d.add_box(c, (0.3, 0.3, 0.3), (1, 1, 1), 0.5, 0.2, red)
    return d


def render_both(d, w, h, frames):
    a = d.arrays()
    dev = torch.device("cuda:0")
    verts = torch.tensor(a["vertices"].reshape(-1), device=dev)
    idx = torch.tensor(a["indices"].reshape(-1).view(np.int32), device=dev)
    ntri = len(a["indices"])
    bvh = BVH(verts, idx)
    bvh.build(ntri)
    rt = Raytracer(d, bvh, w, h)
    cam = np.array([0.0, 2.5, 6.0, 0.0, -0.25, -1.0, 1.0, 0.0, 0.0, 0.0, 1.0, -0.25], np.float32)
    cam[3:6] /= np.linalg.norm(cam[3:6])
    cam[9:12] /= np.linalg.norm(cam[9:12])
    fov = L.lib.seevr_raytrace_fov_scale()
    nodes = {k: bvh[k].cpu().numpy() for k in ("node_min", "node_max", "left", "right", "count",
                                               "prim_indices")}
    out = []
    for f in range(frames):
        gpu = rt.render(cam[0:3], cam[3:6], cam[6:9], cam[9:12], ntri).cpu().numpy().copy()
        ref = pyoracle.raytrace(a["vertices"], a["indices"], nodes["node_min"], nodes["node_max"],
                                nodes["left"], nodes["right"], nodes["count"],
                                nodes["prim_indices"], a["tri_geom"], a["geom_material"],
                                a["mat_albedo"], a["mat_roughness"], a["mat_metallic"],
                                a["mat_emission"], a["mat_ior"], cam, w, h, f, fov, threads=8)
        out.append((gpu, ref))
    bvh.deinit()
    return out


def test_raytrace_bit_exact_against_restatement():
    d = showcase()
    for gpu, ref in render_both(d, 96, 72, frames=2):
        assert np.isfinite(gpu).all()
        bad = np.argwhere(gpu != ref)
        assert len(bad) == 0, (len(bad), bad[:4].tolist())
    # the scene is lit: something brighter than the sky reaches the camera
    assert gpu[..., :3].max() > 1.0
