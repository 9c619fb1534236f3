"""CPU checks of the C-ABI library: it loads without a GPU and exports every
entry point include/pdp3g.h declares; host-side argument checks answer with
status codes (no compute call is made here)."""
import ctypes
import os
import re

import pytest

from pdp3_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if not hdr.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(pdp3g_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    L = api.load()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_binding_covers_declared_symbols():
    bound = {name for name, _, _ in api.EXPORTS}
    assert set(declared_symbols()) <= bound


def test_status_strings_and_null_arguments():
    L = api.load()
    assert L.pdp3g_status_string(0) == b"ok"
    assert L.pdp3g_status_string(5) == b"particle outside the grid"
    # null config / output pointer -> INVALID_ARG, no device touched
    assert L.pdp3g_create(None, None) == 1
    assert L.pdp3g_step(None, 1) == 1
    assert L.pdp3g_sync(None) == 1
    assert L.pdp3g_species_size(None, 0) == -1
    assert L.pdp3g_adjoint_set_mode(None, 0) == 1
    assert L.pdp3g_adjoint_set_jump_terms(None, 1) == 1


def test_invalid_config_rejected_before_device_use():
    L = api.load()
    cfg = api.Config(0.1, 0.8, 2, 2049, 1e-13, 0.0, 0, 0, 0, 0, 0, 0, 0, 0, 0)  # n_grid_r < 3
    h = ctypes.c_void_p()
    assert L.pdp3g_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    cfg = api.Config(0.1, 0.8, 65, 257, -1.0, 0.0, 0, 0, 0, 0, 0, 0, 0, 0, 0)  # dt < 0
    assert L.pdp3g_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    cfg = api.Config(0.1, 0.8, 65, 257, 1e-13, 0.0, 0, 0, 0, 0, 0, 7, 0, 0, 0)  # bad pusher
    assert L.pdp3g_create(ctypes.byref(cfg), ctypes.byref(h)) == 1


def test_no_device_is_reported_not_faked():
    L = api.load()
    if L.pdp3g_device_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError):
        api.Simulation(0.05, 0.2, 65, 257, 1e-12)
