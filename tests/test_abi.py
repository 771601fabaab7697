"""C ABI checks that need no GPU: every symbol declared in include/*.h is
exported by the built library, defaults equal the reference constants, and
argument errors come back as status codes."""
import ctypes as C
import re
from pathlib import Path

import pytest

from conftest import ROOT, cuda_available
from seevr_b200 import _lib as L


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names.update(re.findall(r"\b(seevr_\w+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(str(L.LIB_PATH))
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_default_params_are_reference_constants():
    p = L.default_params()
    assert p.pgs_iterations == 4                     # physics.comp:68
    assert p.baumgarte == pytest.approx(0.2)         # physics.comp:66
    assert p.slop == pytest.approx(0.005)            # physics.comp:67
    assert p.linear_damping == pytest.approx(0.999)  # physics.comp:422
    assert p.angular_damping == pytest.approx(0.998) # physics.comp:425
    assert p.mpr_eps == pytest.approx(1e-6)          # physics.comp:174
    assert p.mpr_tolerance == pytest.approx(1e-6)    # physics.comp:175
    assert p.mpr_iterations == 50                    # physics.comp:176
    assert p.mpr_discover_trials == 15               # physics.comp:290


def test_create_argument_errors():
    h = C.c_void_p()
    caps = L.Caps(16, 16, 16, 16, 16, 1)
    st = L.lib.seevr_physics_create(None, C.byref(caps), None, C.byref(h))
    assert st == L.ERR_INVALID_ARGUMENT
    b = L.Bindings()
    st = L.lib.seevr_physics_create(C.byref(b), C.byref(caps), None, C.byref(h))
    if cuda_available():
        assert st == L.ERR_INVALID_ARGUMENT  # NULL buffers
    else:
        assert st == L.ERR_NO_DEVICE
    assert not h.value
    assert L.lib.seevr_last_error()


def test_status_strings():
    for s in range(8):
        assert L.lib.seevr_status_string(s)
    assert L.lib.seevr_abi_version() == 2


def test_null_handle_calls_fail_cleanly():
    out = (C.c_uint32 * 2)()
    assert L.lib.seevr_physics_read_counters(None, out) == L.ERR_INVALID_ARGUMENT
    g = L.fptr((0, -9.81, 0), 3)
    assert L.lib.seevr_physics_step(None, 1, 0, 0, 1, 0.1, g, None) == L.ERR_INVALID_ARGUMENT
    io = L.HostState()
    assert L.lib.seevr_physics_step_io(None, 1, 0, 0, 1, 0.1, g, C.byref(io), None) == \
        L.ERR_INVALID_ARGUMENT
    assert b"io is NULL" in L.lib.seevr_last_error()
    L.lib.seevr_physics_destroy(None)
