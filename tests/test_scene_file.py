"""Scene files (seevr_scene_save / seevr_scene_load): the binary dump of the
staging arrays that data.zig builds, used for reproducible benches and
fixtures.  A saved and reloaded scene must hand every binding the same
bytes, render and material tables included."""
import numpy as np
import pytest

from seevr_b200 import Data

COUNTS = range(9)  # bodies, geoms, hull verts, vertices, triangles, support entries,
                   # scenes, materials, dynamic bodies


def _same(a: Data, b: Data):
    for c in COUNTS:
        assert a.count(c) == b.count(c), c
    aa, bb = a.arrays(), b.arrays()
    assert aa.keys() == bb.keys()
    for k in aa:
        assert aa[k].dtype == bb[k].dtype, k
        assert np.array_equal(aa[k].view(np.uint8), bb[k].view(np.uint8)), k


@pytest.mark.parametrize("make", [
    lambda: Data.pile(seed=3, n_boxes=12, n_spheres=12),
    lambda: Data.batch(num_scenes=6, min_bodies=8, max_bodies=40, seed_base=5),
])
def test_save_load_round_trip(tmp_path, make):
    d = make()
    path = tmp_path / "scene.seevr"
    d.save(path)
    _same(d, Data.load(path))


def test_reloaded_scene_saves_identically(tmp_path):
    d = Data.pile(seed=4, n_boxes=5, n_spheres=5)
    p1, p2 = tmp_path / "a.seevr", tmp_path / "b.seevr"
    d.save(p1)
    Data.load(p1).save(p2)
    assert p1.read_bytes() == p2.read_bytes()


def test_bad_files_are_rejected(tmp_path):
    d = Data.pile(seed=1, n_boxes=3, n_spheres=3)
    good = tmp_path / "good.seevr"
    d.save(good)
    raw = good.read_bytes()
    for name, data in (("magic", b"NOTASCN1" + raw[8:]), ("truncated", raw[: len(raw) // 2]),
                       ("empty", b"")):
        bad = tmp_path / f"{name}.seevr"
        bad.write_bytes(data)
        with pytest.raises(OSError):
            Data.load(bad)
    with pytest.raises(OSError):
        Data.load(tmp_path / "missing.seevr")
