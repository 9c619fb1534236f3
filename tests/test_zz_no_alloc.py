"""The allocation-free diagnostics entry point, through the C ABI.

pdp3g_field_diagnostics_noalloc serves callers that may not allocate device
memory (code inside CUDA graph capture, hosts whose allocator owns every
device byte, embedders that forbid cudaMalloc after start-up): they hand it
device pointers they already own, and its scratch is a static device array.
Its results must equal those of pdp3g_diagnostics (the allocating, context-
based entry point) within the tolerance the parity tests use (1e-12
relative), on two calls in a row, since the calls share the static scratch.

This file is named to be collected last: device buffers for the test itself
come from torch (the test may allocate; the entry point may not).
"""
import ctypes

import numpy as np
import pytest

from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).reshape(-1)).cuda()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_diagnostics_match_context_diagnostics_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    wl = W.thermal_config(steps=6, ppc=4)
    sim = api.from_workload(wl)
    rho0_host = sim.charge_density()
    sim.mark_initial_charge()
    # put non-trivial fields on the grid, then advance the plasma
    rng = np.random.default_rng(21)
    sim.set_field("E_z", rng.normal(0.0, 1e3, (wl.n_grid_r, wl.n_grid_z)))
    sim.step(6)
    sim.sync()
    ref = sim.diagnostics()

    names = ["E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z"]
    grids = [_dev(torch, sim.field(n)) for n in names]
    rho_host = sim.charge_density()
    rho = _dev(torch, rho_host)
    rho0 = _dev(torch, rho0_host)
    sigma = _dev(torch, sim.field("sigma"))
    L = api.load()
    stream = torch.cuda.current_stream()
    results = []
    for call in range(2):
        out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
        st = L.pdp3g_field_diagnostics_noalloc(
            *[_ptr(g) for g in grids], _ptr(rho), _ptr(rho0), _ptr(sigma), wl.n_grid_r,
            wl.n_grid_z, wl.r_size, wl.z_size, _ptr(out), ctypes.c_void_p(stream.cuda_stream))
        assert st == 0, "call %d returned status %d" % (call, st)
        torch.cuda.synchronize()
        results.append(out.cpu().numpy().copy())
    # the net charge of a neutral plasma is a cancellation residue: compare it
    # on the scale of one species' charge, sum |rho_electrons| dV
    i = np.arange(wl.n_grid_r, dtype=np.float64)[:, None]
    vol = np.where(i == 0, np.pi * wl.dz * wl.dr ** 2 / 4.0, 2.0 * np.pi * wl.dz * wl.dr ** 2 * i)
    charge_scale = float((np.abs(sim.charge_density(1)) * vol).sum())
    for got in results:
        assert abs(got[0] - ref["field_energy"]) <= TOL * abs(ref["field_energy"])
        assert abs(got[1] - ref["gauss_residual"]) <= TOL * ref["gauss_residual"]
        assert abs(got[2] - ref["charge_total"]) <= TOL * charge_scale
    assert np.array_equal(results[0], results[1])
    assert ref["field_energy"] > 0
    sim.close()


def test_noalloc_rejects_oversized_grid():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = api.load()
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = _ptr(dummy)
    # 4097 x 4097 nodes is above the 16,777,216-node limit: rejected before any launch
    st = L.pdp3g_field_diagnostics_noalloc(p, p, p, p, p, p, p, None, p, 4097, 4097, 0.1, 0.8,
                                           p, None)
    assert st == 1
