"""Device selection through the C ABI: a context lives on the device its
config names (pdp3g_config.device, the rank's local GPU in bench.py), every
visible device steps, and an ordinal past the last device is refused with
PDP3G_INVALID_ARG (no CUDA error left pending) instead of falling back to
device 0."""
import pytest

from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_each_visible_device_steps_and_a_missing_one_is_refused():
    torch = pytest.importorskip("torch")
    n = torch.cuda.device_count()
    assert n >= 1
    wl = W.small_config(beam=True, steps=2)
    for d in range(n):
        sim = api.from_workload(wl, device=d)
        sim.step(2)
        sim.sync()
        assert sim.status() == 0
        # an event recorded on the context's stream, as device d's, completes
        stream = torch.cuda.ExternalStream(sim.stream_ptr, device=torch.device("cuda", d))
        ev = torch.cuda.Event()
        ev.record(stream)
        ev.synchronize()
        sim.close()
    for bad in (n, -1):
        with pytest.raises(api.Pdp3gError) as err:
            api.from_workload(wl, device=bad)
        assert err.value.status == 1  # PDP3G_INVALID_ARG
    # nothing pending: the next context on device 0 steps normally
    sim = api.from_workload(wl, device=0)
    sim.step(1)
    sim.sync()
    assert sim.status() == 0
    sim.close()
