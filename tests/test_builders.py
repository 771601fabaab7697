"""Scene builders against data.zig's formulas (Data.addBox data.zig:392-485,
Data.addSphere 487-597, buildSupportLookup 299-353): the masses, inertias,
hull sizes and support-lookup choice the Zig host would upload."""
import numpy as np

from seevr_b200 import Data

f32 = np.float32


def _scene():
    d = Data()
    dyn = d.add_material((0.8, 0.2, 0.2), 0.4, 0.0, (0, 0, 0), 1.5, 1000.0)
    static = d.add_material((0.5, 0.5, 0.5), 0.9, 0.0, (0, 0, 0), 1.5, 0.0)
    return d, dyn, static


def test_box_mass_and_inertia():
    d, dyn, static = _scene()
    half = (0.3, 0.5, 0.7)
    b = d.add_box((0, 2, 0), half, (1, 1, 1), 0.5, 0.2, dyn)
    g = d.add_box((0, -0.25, 0), (50, 0.25, 50), (1, 1, 1), 0.5, 0.2, static)
    hx, hy, hz = (f32(x) for x in half)
    mass = f32(1000.0) * (hx * f32(2) * hy * f32(2) * hz * f32(2))   # rho * 8 hx hy hz
    wx, wy, wz = hx * f32(2), hy * f32(2), hz * f32(2)
    inertia = np.array([mass / f32(12) * (wy * wy + wz * wz), mass / f32(12) * (wx * wx + wz * wz),
                        mass / f32(12) * (wx * wx + wy * wy)], np.float32)
    im = d.array("body_inv_mass").ravel()
    ii = d.array("body_inv_inertia").reshape(-1, 3)
    assert im[b] == f32(1) / mass
    assert np.array_equal(ii[b], (f32(1) / inertia).astype(np.float32))
    assert np.array_equal(d.array("body_inertia").reshape(-1, 3)[b], inertia)
    # density 0: static, never moved by gravity or impulses
    assert im[g] == 0 and not ii[g].any()
    assert d.num_dynamic == 1


def test_sphere_mass_inertia_and_hull():
    d, dyn, _ = _scene()
    r, segs = 0.4, 16
    s = d.add_sphere((0, 3, 0), r, (1, 1, 1), segs, 0.5, 0.2, dyn)
    mass = 1000.0 * 4.0 / 3.0 * np.pi * r ** 3                       # rho 4/3 pi r^3
    im = float(d.array("body_inv_mass").ravel()[s])
    assert abs(1.0 / im - mass) <= 2e-6 * mass
    inertia = d.array("body_inertia").reshape(-1, 3)[s]
    assert np.allclose(inertia, 0.4 * mass * r * r, rtol=2e-6)         # 2/5 m r^2
    hull = d.array("hull_range").reshape(-1, 2)[0]
    assert hull[1] == (segs + 1) ** 2                                  # UV grid of (S+1)^2 verts
    v = d.array("hull_verts").reshape(-1, 3)[hull[0]:hull[0] + hull[1]]
    assert np.allclose(np.linalg.norm(v, axis=1), r, rtol=1e-6, atol=1e-6)


def test_support_lookup_only_above_32_vertices():
    d, dyn, _ = _scene()
    d.add_box((0, 1, 0), (0.3, 0.3, 0.3), (1, 1, 1), 0.5, 0.2, dyn)    # 8 vertices
    d.add_sphere((2, 1, 0), 0.3, (1, 1, 1), 16, 0.5, 0.2, dyn)         # 289 vertices
    d.add_sphere((4, 1, 0), 0.3, (1, 1, 1), 4, 0.5, 0.2, dyn)          # 25 vertices
    off = d.array("support_offset").ravel()
    assert off[0] == 0 and off[2] == 0          # brute force
    assert off[1] != 0                          # 3 axes x 64 bins
    lut = d.array("support_lookup").ravel()
    bins = lut[off[1]:off[1] + 192]
    assert bins.size == 192 and bins.max() < 289
