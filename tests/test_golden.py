"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py):
the seeded scene generator and the FP32 oracle must reproduce them bit for
bit, so a change to either that alters any result is caught here."""
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden  # noqa: E402


def load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
def test_oracle_reproduces_golden(name):
    ref = load(name)
    assert int(ref["num_contacts"]) > 0  # the fixture pins contacts, not free flight only
    _, _, out = make_golden.run_case(name)
    assert str(out["scene_sha256"]) == str(ref["scene_sha256"]), "scene generator changed"
    for k in make_golden.KEYS + ("num_pairs", "num_contacts"):
        assert out[k].dtype == ref[k].dtype and out[k].shape == ref[k].shape, k
        assert np.array_equal(np.atleast_1d(out[k]).view(np.uint8),
                              np.atleast_1d(ref[k]).view(np.uint8)), k
