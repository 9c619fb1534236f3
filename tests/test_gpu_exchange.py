"""pdp3g_exchange_species: the state out and the next state in, with the two
copy directions pipelined by chunks of 2^20 particles on two streams.

* out receives exactly what pdp3g_get_species returns; the species then
  holds in (bit for bit in the FP64 form; in the FP32 form as
  pdp3g_set_species would store it).
* in == out (a round trip through pinned host memory, several chunks): the
  state is unchanged and the next step equals the step of a context that
  made no round trip (to 1e-12 in the FP64 form: its grid currents are
  summed by atomics in a varying order).
* pdp3g_exchange_all (every species in one pipeline): out receives the
  state as pdp3g_exchange_species's out does, and the state loaded from the
  same input arrays equals what one pdp3g_exchange_species call per species
  loads, in any item order; a repeated species or a null array is refused.
"""
import numpy as np
import pytest
import torch

from helpers import rel_inf
from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu

KEYS = ("r", "z", "vr", "vphi", "vz")


def pinned(a):
    t = torch.empty(a.size, dtype=torch.from_numpy(a[:1]).dtype, pin_memory=True).numpy()
    t[:] = a
    return t


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_exchange_out_and_in(precision):
    wl = W.small_config(beam=True, steps=3)
    sim = api.from_workload(wl, precision=precision)
    sim.step(3)
    sim.sync()
    for sid in range(3):
        state = sim.species(sid)
        n = state["r"].size
        out = {k: np.zeros(n) for k in KEYS}
        out["alive"] = np.zeros(n, dtype=np.uint8)
        inp = {k: state[k].copy() for k in KEYS}
        inp["vz"] = inp["vz"] * 0.5
        inp["alive"] = state["alive"].copy()
        sim.exchange_species(sid, out, inp)
        for k in KEYS + ("alive",):
            assert np.array_equal(out[k], state[k]), (sid, k)
        now = sim.species(sid)
        m = state["alive"].astype(bool)
        if precision == "fp64":
            for k in KEYS:
                assert np.array_equal(now[k], inp[k]), (sid, k)
        else:
            assert np.abs(now["r"][m] - inp["r"][m]).max() <= 1e-6 * wl.r_size
            assert np.abs(now["z"][m] - inp["z"][m]).max() <= 1e-6 * wl.z_size
            for k in ("vr", "vphi", "vz"):
                scale = max(float(np.abs(inp[k][m]).max()), 1.0)
                assert np.abs(now[k][m] - inp[k][m]).max() <= 1e-6 * scale, (sid, k)
    sim.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_round_trip_in_place_several_chunks(precision):
    wl = W.wake_config(ppc=3)          # 1.57M particles per plasma species: 2 chunks
    a = api.from_workload(wl, precision=precision)
    b = api.from_workload(wl, precision=precision)
    for s_ in (a, b):
        s_.step(2)
        s_.sync()
    before = [a.species(sid) for sid in range(2)]
    for sid in range(2):
        buf = {k: pinned(before[sid][k]) for k in KEYS}
        buf["alive"] = pinned(before[sid]["alive"])
        a.exchange_species(sid, buf, buf)
        for k in KEYS:
            assert np.array_equal(buf[k], before[sid][k]), (sid, k)
        after = a.species(sid)
        for k in KEYS:
            if precision == "fp64":
                assert np.array_equal(after[k], before[sid][k]), (sid, k)
            else:
                scale = max(float(np.abs(before[sid][k]).max()), 1e-300)
                assert np.abs(after[k] - before[sid][k]).max() <= 1e-6 * scale, (sid, k)
    a.step(1)
    b.step(1)
    a.sync()
    b.sync()
    # the FP64 grid currents sum by atomics, whose order varies run to run
    tol = 1e-12 if precision == "fp64" else 1e-5
    for c in ("E_r", "E_z", "H_phi", "J_r", "J_z"):
        assert rel_inf(a.field(c), b.field(c)) <= tol, c
    a.close()
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_exchange_all_equals_one_call_per_species(precision):
    wl = W.wake_config(ppc=3)          # 2 chunks per plasma species, and the bunch
    a = api.from_workload(wl, precision=precision)
    b = api.from_workload(wl, precision=precision)
    for s_ in (a, b):
        s_.step(3)
        s_.sync()
    n_sp = 3
    # each context's own state (two runs differ by the atomics' summation order)
    states = [a.species(sid) for sid in range(n_sp)]
    states_b = [b.species(sid) for sid in range(n_sp)]
    outs_a, outs_b, inps = [], [], []
    for sid in range(n_sp):
        n = states[sid]["r"].size
        inp = {k: pinned(states[sid][k]) for k in KEYS}
        inp["vz"] = pinned(states[sid]["vz"] * 0.5)
        inp["alive"] = pinned(states[sid]["alive"])
        inps.append(inp)
        for outs in (outs_a, outs_b):
            o = {k: pinned(np.zeros(n)) for k in KEYS}
            o["alive"] = pinned(np.zeros(n, dtype=np.uint8))
            outs.append(o)
    # items in reverse species order: the order of the items is free
    a.exchange_all([(sid, outs_a[sid], inps[sid]) for sid in reversed(range(n_sp))])
    for sid in range(n_sp):
        b.exchange_species(sid, outs_b[sid], inps[sid])
    for sid in range(n_sp):
        for k in KEYS + ("alive",):
            assert np.array_equal(outs_a[sid][k], states[sid][k]), (sid, k)
            assert np.array_equal(outs_b[sid][k], states_b[sid][k]), (sid, k)
        # the state loaded from the same input arrays is the same
        sa, sb = a.species(sid), b.species(sid)
        for k in KEYS + ("alive",):
            assert np.array_equal(sa[k], sb[k]), (sid, k)
    # in place, all species at once
    bufs = [{k: pinned(a.species(sid)[k]) for k in KEYS + ("alive",)} for sid in range(n_sp)]
    keep = [{k: v.copy() for k, v in bf.items()} for bf in bufs]
    a.exchange_all([(sid, bufs[sid], bufs[sid]) for sid in range(n_sp)])
    for sid in range(n_sp):
        now = a.species(sid)
        for k in KEYS:
            assert np.array_equal(bufs[sid][k], keep[sid][k]), (sid, k)
            if precision == "fp64":
                assert np.array_equal(now[k], keep[sid][k]), (sid, k)
    with pytest.raises(api.Pdp3gError):
        a.exchange_all([(0, bufs[0], bufs[0]), (0, bufs[0], bufs[0])])
    arr = (api.ExchangeItem * 1)()
    arr[0].id = 0
    with pytest.raises(api.Pdp3gError):
        a._check(a.L.pdp3g_exchange_all(a.h, arr, 1), "exchange_all")
    a.close()
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_exchange_all_with_one_host_block_per_species(precision):
    """The five host arrays of a species in one block (equally spaced): the
    exchange moves them with 2-D copies; same result as separate arrays."""
    wl = W.wake_config(ppc=3)
    a = api.from_workload(wl, precision=precision)
    a.step(2)
    a.sync()
    n_sp = 3
    before = [a.species(sid) for sid in range(n_sp)]
    blocks, bufs = [], []
    for sid in range(n_sp):
        n = before[sid]["r"].size
        blk = pinned(np.zeros(5 * n))
        d = {k: blk[j * n:(j + 1) * n] for j, k in enumerate(KEYS)}
        for k in KEYS:
            d[k][:] = before[sid][k]
        d["alive"] = pinned(before[sid]["alive"])
        blocks.append(blk)
        bufs.append(d)
    inp = [{k: (pinned(before[sid][k] * (0.5 if k == "vz" else 1.0)) if k != "alive"
                else pinned(before[sid]["alive"])) for k in KEYS + ("alive",)}
           for sid in range(n_sp)]
    # out into the blocks, in from separate arrays
    a.exchange_all([(sid, bufs[sid], inp[sid]) for sid in range(n_sp)])
    for sid in range(n_sp):
        for k in KEYS:
            assert np.array_equal(bufs[sid][k], before[sid][k]), (sid, k)
    loaded = [a.species(sid) for sid in range(n_sp)]
    # in from the blocks (now holding the previous state), out to separate arrays
    outs = [{k: pinned(np.zeros(before[sid]["r"].size)) for k in KEYS} for sid in range(n_sp)]
    a.exchange_all([(sid, outs[sid], bufs[sid]) for sid in range(n_sp)])
    for sid in range(n_sp):
        for k in KEYS:
            assert np.array_equal(outs[sid][k], loaded[sid][k]), (sid, k)
        now = a.species(sid)
        if precision == "fp64":
            for k in KEYS:
                assert np.array_equal(now[k], before[sid][k]), (sid, k)
    a.close()

