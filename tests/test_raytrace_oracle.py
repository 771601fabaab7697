"""CPU restatement of the path tracer (raytrace.comp): known answers."""
import numpy as np

import pyoracle

FOV = np.float32(np.tan(np.float64(np.float32(np.float32(30.0) * np.float32(3.14159265)) /
                                  np.float32(180.0))))


def one_triangle(v, emission):
    """A scene of one triangle: its tree is a single leaf."""
    v = np.asarray(v, np.float32).reshape(3, 3)
    return dict(verts=v, idx=np.array([0, 1, 2], np.uint32), node_min=v.min(0), node_max=v.max(0),
                left=np.array([0], np.uint32), right=np.array([0], np.uint32),
                count=np.array([1], np.uint32), prim=np.array([0], np.uint32),
                tri_geom=np.array([0], np.uint32), geom_material=np.array([0], np.uint32),
                albedo=np.array([0.5, 0.5, 0.5], np.float32),
                roughness=np.array([0.5], np.float32), metallic=np.array([0.0], np.float32),
                emission=np.asarray(emission, np.float32), ior=np.array([0.0], np.float32))


CAM = np.array([0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 1, 0], np.float32)


def render(scene, w=32, h=24, frame=0):
    return pyoracle.raytrace(**scene, cam=CAM, width=w, height=h, frame=frame, fov=FOV)


def test_emissive_wall_fills_the_view():
    # every primary ray hits the light at bounce 0: the pixel is its emission
    # exactly (16 equal samples of dyadic values sum and divide exactly)
    s = one_triangle([[-100, -100, -1], [100, -100, -1], [0, 100, -1]], [1.0, 0.5, 0.25])
    img = render(s)
    assert np.array_equal(img[..., :3], np.broadcast_to([1.0, 0.5, 0.25], img[..., :3].shape))
    assert (img[..., 3] == 1.0).all()


def test_sky_when_nothing_is_hit():
    # the only triangle is behind the camera: every sample sees the sky,
    # 0.8 * mix(white, (0.5, 0.7, 1.0), (dir.y + 1) / 2), so red falls and
    # blue stays 0.8 from the bottom row to the top row
    s = one_triangle([[-1, -1, 5], [1, -1, 5], [0, 1, 5]], [0, 0, 0])
    img = render(s)
    red = img[..., 0].mean(1)
    assert (np.diff(red) > 0).all()          # rows go down the image: rd.y decreases
    assert np.allclose(img[..., 2], 0.8, atol=1e-6)
    assert (img[..., :3] <= 0.8 + 1e-6).all() and (img[..., :3] >= 0.4 - 1e-6).all()


def test_frame_number_changes_the_samples_only():
    # a diffuse floor under the sky: a new frame number reseeds every pixel,
    # the image statistics stay the same
    s = one_triangle([[-100, -1, 100], [100, -1, 100], [0, -1, -100]], [0, 0, 0])
    a, b = render(s, frame=0), render(s, frame=1)
    assert not np.array_equal(a, b)
    assert abs(a[..., :3].mean() - b[..., :3].mean()) < 0.02
