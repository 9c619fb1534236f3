"""ctypes binding of libpdp3g.so (the C ABI declared in include/pdp3g.h).

This module never falls back to a CPU path: if the CUDA library is missing
or no device is usable, constructing a Simulation raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpdp3g.so")

E_R, E_PHI, E_Z, H_R, H_PHI, H_Z, H_R_HALF, H_PHI_HALF, H_Z_HALF, J_R, J_PHI, J_Z, SIGMA = \
    range(13)
COMP = {"E_r": E_R, "E_phi": E_PHI, "E_z": E_Z, "H_r": H_R, "H_phi": H_PHI, "H_z": H_Z,
        "H_r_half": H_R_HALF, "H_phi_half": H_PHI_HALF, "H_z_half": H_Z_HALF,
        "J_r": J_R, "J_phi": J_PHI, "J_z": J_Z, "sigma": SIGMA}
PUSHERS = {"boris": 0, "vay": 1, "boris_classic": 2}
PROBE_RHO_BEAM = 100
PROBE_T = 101
PROBE_DENSITY = 102
PRECISIONS = {"fp64": 0, "fp32": 1}
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "NaN position",
          4: "velocity >= c", 5: "particle outside the grid", 6: "timeout",
          7: "not supported", 8: "out of device memory"}


class Pdp3gError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("pdp3g status %d (%s): %s" % (status, STATUS.get(status, "?"), msg))
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [("r_size", ctypes.c_double), ("z_size", ctypes.c_double),
                ("n_grid_r", ctypes.c_int32), ("n_grid_z", ctypes.c_int32),
                ("dt", ctypes.c_double), ("current_time", ctypes.c_double),
                ("pml_l1", ctypes.c_double), ("pml_l2", ctypes.c_double),
                ("pml_l3", ctypes.c_double), ("pml_sigma1", ctypes.c_double),
                ("pml_sigma2", ctypes.c_double),
                ("pusher", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("device", ctypes.c_int32), ("sort_interval", ctypes.c_int32)]


class Diag(ctypes.Structure):
    _fields_ = [("field_energy", ctypes.c_double), ("kinetic_energy", ctypes.c_double),
                ("gauss_residual", ctypes.c_double), ("gauss_norm", ctypes.c_double),
                ("charge_total", ctypes.c_double), ("alive", ctypes.c_int64)]


class EnsembleInfo(ctypes.Structure):
    _fields_ = [("runs", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("blocks", ctypes.c_int32), ("used_graph", ctypes.c_int32),
                ("last_ms", ctypes.c_double), ("last_steps_done", ctypes.c_int64),
                ("particles", ctypes.c_int64), ("mode", ctypes.c_int32),
                ("graph_blocks_per_sm", ctypes.c_int32)]


class ExchangeItem(ctypes.Structure):
    _fields_ = ([("id", ctypes.c_int32)] +
                [("out_" + k, ctypes.POINTER(ctypes.c_double))
                 for k in ("r", "z", "vr", "vphi", "vz")] +
                [("out_alive", ctypes.POINTER(ctypes.c_uint8))] +
                [("in_" + k, ctypes.POINTER(ctypes.c_double))
                 for k in ("r", "z", "vr", "vphi", "vz")] +
                [("in_alive", ctypes.POINTER(ctypes.c_uint8))])


class Timing(ctypes.Structure):
    _fields_ = [("ms_step_total", ctypes.c_double), ("ms_particles", ctypes.c_double),
                ("ms_fields", ctypes.c_double), ("ms_sort", ctypes.c_double),
                ("ms_other", ctypes.c_double), ("launches", ctypes.c_int64),
                ("particle_launches", ctypes.c_int64), ("steps", ctypes.c_int64),
                ("particle_steps", ctypes.c_int64)]


_D = ctypes.POINTER(ctypes.c_double)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_VP = ctypes.c_void_p
_I32 = ctypes.c_int32
_lib = None

EXPORTS = [
    ("pdp3g_create", _I32, [ctypes.POINTER(Config), ctypes.POINTER(_VP)]),
    ("pdp3g_destroy", None, [_VP]),
    ("pdp3g_add_species", _I32, [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int64] +
     [_D] * 6 + [_U8, ctypes.POINTER(_I32)]),
    ("pdp3g_add_species_device", _I32, [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int64] +
     [_VP] * 6 + [ctypes.POINTER(_I32)]),
    ("pdp3g_add_bunch", _I32, [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                               ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, _I32, ctypes.c_double, ctypes.POINTER(_I32)]),
    ("pdp3g_step", _I32, [_VP, _I32]),
    ("pdp3g_sync", _I32, [_VP]),
    ("pdp3g_sort", _I32, [_VP]),
    ("pdp3g_inject", _I32, [_VP]),
    ("pdp3g_calc_h", _I32, [_VP]),
    ("pdp3g_reset_j", _I32, [_VP]),
    ("pdp3g_push_deposit", _I32, [_VP]),
    ("pdp3g_calc_e", _I32, [_VP]),
    ("pdp3g_advance_time", _I32, [_VP]),
    ("pdp3g_set_time", _I32, [_VP, ctypes.c_double]),
    ("pdp3g_get_field", _I32, [_VP, _I32, _D]),
    ("pdp3g_set_field", _I32, [_VP, _I32, _D]),
    ("pdp3g_get_species", _I32, [_VP, _I32] + [_D] * 6 + [_U8]),
    ("pdp3g_set_species", _I32, [_VP, _I32] + [_D] * 5 + [_U8]),
    ("pdp3g_species_size", ctypes.c_int64, [_VP, _I32]),
    ("pdp3g_charge_density", _I32, [_VP, ctypes.c_uint32, _D]),
    ("pdp3g_mark_initial_charge", _I32, [_VP]),
    ("pdp3g_diagnostics", _I32, [_VP, ctypes.POINTER(Diag)]),
    ("pdp3g_set_timing", _I32, [_VP, _I32]),
    ("pdp3g_get_timing", _I32, [_VP, ctypes.POINTER(Timing)]),
    ("pdp3g_reset_timing", _I32, [_VP]),
    ("pdp3g_current_time", ctypes.c_double, [_VP]),
    ("pdp3g_stream", _VP, [_VP]),
    ("pdp3g_device_bytes", ctypes.c_int64, [_VP]),
    ("pdp3g_status_string", ctypes.c_char_p, [_I32]),
    ("pdp3g_last_error", ctypes.c_char_p, [_VP]),
    ("pdp3g_device_available", _I32, []),
    ("pdp3g_ensemble_create", _I32, [ctypes.POINTER(_VP), _I32, ctypes.POINTER(_VP)]),
    ("pdp3g_ensemble_run", _I32, [_VP, _I32]),
    ("pdp3g_ensemble_autotune", _I32, [_VP, _I32, ctypes.POINTER(_I32)]),
    ("pdp3g_ensemble_set_mode", _I32, [_VP, _I32]),
    ("pdp3g_ensemble_set_budget", _I32, [_VP, ctypes.c_double]),
    ("pdp3g_ensemble_set_sort_interval", _I32, [_VP, _I32]),
    ("pdp3g_ensemble_cancel", _I32, [_VP, _I32]),
    ("pdp3g_ensemble_info", _I32, [_VP, ctypes.POINTER(EnsembleInfo)]),
    ("pdp3g_ensemble_last_error", ctypes.c_char_p, [_VP]),
    ("pdp3g_ensemble_destroy", None, [_VP]),
    ("pdp3g_field_diagnostics_noalloc", _I32, [_VP] * 9 + [_I32, _I32, ctypes.c_double,
                                                          ctypes.c_double, _VP, _VP]),
    ("pdp3g_probe_read", _I32, [_VP] + [_I32] * 6 + [_D, ctypes.c_int64,
                                                      ctypes.POINTER(ctypes.c_int64)]),
    ("pdp3g_add_species_upstream", _I32, [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int64]
     + [ctypes.c_double] * 4 + [ctypes.POINTER(_I32)]),
    ("pdp3g_probe_read_species", _I32, [_VP] + [_I32] * 7 + [_D, ctypes.c_int64,
                                                              ctypes.POINTER(ctypes.c_int64)]),
    ("pdp3g_temperature", _I32, [_VP, _I32, _D]),
    ("pdp3g_density", _I32, [_VP, _I32, _D]),
    ("pdp3g_exchange_species", _I32, [_VP, _I32] + [_D] * 5 + [_U8] + [_D] * 5 + [_U8]),
    ("pdp3g_exchange_all", _I32, [_VP, ctypes.POINTER(ExchangeItem), _I32]),
    ("pdp3g_poisson_solve", _I32, [_VP, _D, _D]),
    ("pdp3g_probe_particles", _I32, [_VP] + [_I32] * 5 + [_D] * 5 +
     [ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    ("pdp3g_adjoint_create", _I32, [_VP] + [_I32] * 6 + [ctypes.POINTER(_VP)]),
    ("pdp3g_forward_window", _I32, [_VP, _D]),
    ("pdp3g_backward_window", _I32, [_VP]),
    ("pdp3g_adjoint_species", _I32, [_VP, _I32] + [_D] * 6),
    ("pdp3g_adjoint_field", _I32, [_VP, _I32, _D]),
    ("pdp3g_adjoint_bunch_velocity", _I32, [_VP, _I32, _D]),
    ("pdp3g_adjoint_timing", _I32, [_VP, _D, _D]),
    ("pdp3g_adjoint_set_mode", _I32, [_VP, _I32]),
    ("pdp3g_adjoint_set_jump_terms", _I32, [_VP, ctypes.c_uint32]),
    ("pdp3g_adjoint_set_face_width", _I32, [_VP, ctypes.c_double]),
    ("pdp3g_adjoint_bytes", ctypes.c_int64, [_VP]),
    ("pdp3g_adjoint_destroy", None, [_VP]),
]


def load(path=LIB_PATH):
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError("%s is missing: build it with `python -m pdp3_b200.build` "
                                "(there is no CPU fallback)" % path)
    L = ctypes.CDLL(path)
    for name, res, args in EXPORTS:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(_D)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Simulation:
    """One device-resident PDP3 simulation (grids + species) on a CUDA device."""

    def __init__(self, r_size, z_size, n_grid_r, n_grid_z, dt, current_time=0.0, pml=None,
                 pusher="boris", precision="fp64", device=0, sort_interval=0):
        self.L = load()
        if not self.L.pdp3g_device_available():
            raise RuntimeError("no CUDA device available to pdp3g")
        pml = [0.0] * 5 if pml is None else list(pml)
        cfg = Config(r_size, z_size, n_grid_r, n_grid_z, dt, current_time, pml[0], pml[1],
                     pml[2], pml[3], pml[4], PUSHERS[pusher], PRECISIONS[precision], device,
                     sort_interval)
        h = _VP()
        st = self.L.pdp3g_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            raise Pdp3gError(st, "pdp3g_create")
        self.h = h
        self.nr, self.nz = n_grid_r, n_grid_z

    def _check(self, st, what):
        if st != 0:
            msg = self.L.pdp3g_last_error(self.h)
            raise Pdp3gError(st, "%s: %s" % (what, msg.decode() if msg else ""))

    def add_species(self, charge_e, mass_me, r, z, vr, vphi, vz, w, alive=None):
        arrs = [_f64(a) for a in (r, z, vr, vphi, vz, w)]
        al = None if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
        sid = _I32()
        self._check(self.L.pdp3g_add_species(self.h, charge_e, mass_me, len(arrs[0]),
                                             *[_p(a) for a in arrs],
                                             al.ctypes.data_as(_U8) if al is not None else None,
                                             ctypes.byref(sid)), "add_species")
        return sid.value

    def add_species_device(self, charge_e, mass_me, r, z, vr, vphi, vz, w):
        """Adds a species from six FP64 device arrays (torch tensors on this
        simulation's device, contiguous, equal length)."""
        arrs = [r, z, vr, vphi, vz, w]
        n = int(arrs[0].numel())
        for a in arrs:
            assert a.is_cuda and a.is_contiguous() and a.numel() == n and str(a.dtype) == "torch.float64"
        sid = _I32()
        self._check(self.L.pdp3g_add_species_device(self.h, float(charge_e), float(mass_me), n,
                                                    *[a.data_ptr() for a in arrs],
                                                    ctypes.byref(sid)), "add_species_device")
        return sid.value

    def add_species_upstream(self, charge_e, mass_me, n, left_density, right_density,
                             temperature, left_plasma_boundary=0.0):
        """The upstream's own initial state of a plasma species (cylindrical
        load with a linear density ramp, Maxwell-Juttner velocities, TESTMODE
        sequences) generated on the device."""
        sid = _I32()
        self._check(self.L.pdp3g_add_species_upstream(
            self.h, float(charge_e), float(mass_me), int(n), float(left_density),
            float(right_density), float(left_plasma_boundary), float(temperature),
            ctypes.byref(sid)), "add_species_upstream")
        return sid.value

    def add_bunch(self, charge_e, mass_me, n, duration, radius, density, velocity,
                  bunch_number=0, hole_duration=0.0):
        sid = _I32()
        self._check(self.L.pdp3g_add_bunch(self.h, charge_e, mass_me, int(n), duration, radius,
                                           density, velocity, int(bunch_number), hole_duration,
                                           ctypes.byref(sid)), "add_bunch")
        return sid.value

    def step(self, n=1):
        self._check(self.L.pdp3g_step(self.h, int(n)), "step")

    def sort(self):
        self._check(self.L.pdp3g_sort(self.h), "sort")

    def sync(self):
        self._check(self.L.pdp3g_sync(self.h), "sync")

    def status(self):
        """Status of pdp3g_sync without raising."""
        return self.L.pdp3g_sync(self.h)

    def field(self, name):
        out = np.empty(self.nr * self.nz)
        self._check(self.L.pdp3g_get_field(self.h, COMP[name], _p(out)), "get_field")
        return out.reshape(self.nr, self.nz)

    def set_field(self, name, arr):
        a = _f64(arr).reshape(-1)
        assert a.size == self.nr * self.nz
        self._check(self.L.pdp3g_set_field(self.h, COMP[name], _p(a)), "set_field")

    def species_size(self, sid):
        return int(self.L.pdp3g_species_size(self.h, sid))

    def species(self, sid):
        n = self.species_size(sid)
        out = {k: np.empty(n) for k in ("r", "z", "vr", "vphi", "vz", "w")}
        alive = np.empty(n, dtype=np.uint8)
        self._check(self.L.pdp3g_get_species(self.h, sid, *[_p(out[k]) for k in
                                                            ("r", "z", "vr", "vphi", "vz", "w")],
                                             alive.ctypes.data_as(_U8)), "get_species")
        out["alive"] = alive
        return out

    def exchange_species(self, sid, out, inp):
        """pdp3g_exchange_species: fills out (dict of float64 r, z, vr, vphi,
        vz and uint8 alive arrays, each of the species' size; pinned memory
        for the copy overlap) with the state and loads inp (same layout; may
        be out itself) as the new state."""
        keys = ("r", "z", "vr", "vphi", "vz")
        n = self.species_size(sid)
        for d in (out, inp):
            for k in keys:
                a = d[k]
                assert a.dtype == np.float64 and a.flags.c_contiguous and a.size == n, k
        oa, ia = out.get("alive"), inp.get("alive")
        self._check(self.L.pdp3g_exchange_species(
            self.h, sid, *[_p(out[k]) for k in keys],
            oa.ctypes.data_as(_U8) if oa is not None else None,
            *[_p(inp[k]) for k in keys],
            ia.ctypes.data_as(_U8) if ia is not None else None), "exchange_species")

    def exchange_all(self, items):
        """pdp3g_exchange_all: items is a list of (sid, out, inp) with out and
        inp as in exchange_species; one pipeline over all of them."""
        keys = ("r", "z", "vr", "vphi", "vz")
        arr = (ExchangeItem * len(items))()
        for j, (sid, out, inp) in enumerate(items):
            n = self.species_size(sid)
            for d in (out, inp):
                for k in keys:
                    a = d[k]
                    assert a.dtype == np.float64 and a.flags.c_contiguous and a.size == n, k
                for k in ("alive",):
                    a = d.get(k)
                    assert a is None or (a.dtype == np.uint8 and a.size == n), k
            it = arr[j]
            it.id = sid
            for k in keys:
                setattr(it, "out_" + k, _p(out[k]))
                setattr(it, "in_" + k, _p(inp[k]))
            oa, ia = out.get("alive"), inp.get("alive")
            it.out_alive = oa.ctypes.data_as(_U8) if oa is not None else None
            it.in_alive = ia.ctypes.data_as(_U8) if ia is not None else None
        self._check(self.L.pdp3g_exchange_all(self.h, arr, len(items)), "exchange_all")

    def set_species(self, sid, r=None, z=None, vr=None, vphi=None, vz=None, alive=None):
        keep = [None if a is None else _f64(a) for a in (r, z, vr, vphi, vz)]
        al = None if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
        self._check(self.L.pdp3g_set_species(
            self.h, sid, *[(_p(a) if a is not None else None) for a in keep],
            al.ctypes.data_as(_U8) if al is not None else None), "set_species")

    def charge_density(self, mask=0xFFFFFFFF):
        out = np.empty(self.nr * self.nz)
        self._check(self.L.pdp3g_charge_density(self.h, mask, _p(out)), "charge_density")
        return out.reshape(self.nr, self.nz)

    def probe(self, name, kind, start_r, start_z, end_r=0, end_z=0):
        """ProbePlain's values of component `name` ("E_r" .. "J_z", "rho_beam")
        for a probe of `kind` ("frame", "col", "row", "dot"), in write order."""
        t = {"frame": 0, "col": 1, "row": 2, "dot": 3}[kind]
        comp = PROBE_RHO_BEAM if name == "rho_beam" else COMP[name]
        cap = max(1, (end_r - start_r) * max(end_z - start_z, 1)) if t == 0 else \
            max(1, end_r - start_r, end_z - start_z)
        out = np.empty(cap)
        n = ctypes.c_int64()
        self._check(self.L.pdp3g_probe_read(self.h, comp, t, start_r, start_z, end_r, end_z,
                                            _p(out), cap, ctypes.byref(n)), "probe_read")
        return out[:n.value]

    def temperature(self, sid):
        """TemperatureClassic of species sid (eV, NaN in empty cells)."""
        out = np.empty(self.nr * self.nz)
        self._check(self.L.pdp3g_temperature(self.h, sid, _p(out)), "temperature")
        return out.reshape(self.nr, self.nz)

    def poisson_solve(self, rho=None):
        """PoissonDirichlet::poisson_solve: writes E_r and E_z from rho (a
        [n_grid_r, n_grid_z] array, or None for the charge density of every
        species) and returns phi."""
        fi = np.empty(self.nr * self.nz)
        rp = None
        if rho is not None:
            rho = np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)
            assert rho.size == self.nr * self.nz
            rp = _p(rho)
        self._check(self.L.pdp3g_poisson_solve(self.h, rp, _p(fi)), "poisson_solve")
        return fi.reshape(self.nr, self.nz)

    def density(self, sid):
        """ParticlesDensity of species sid: [n_grid_r, n_grid_z]."""
        out = np.empty(self.nr * self.nz)
        self._check(self.L.pdp3g_density(self.h, sid, _p(out)), "density")
        return out.reshape(self.nr, self.nz)

    def probe_species(self, name, sid, kind, start_r, start_z, end_r=0, end_z=0):
        """A per-species probe ("T" or "density") of species sid, in write
        order."""
        t = {"frame": 0, "col": 1, "row": 2, "dot": 3}[kind]
        comp = {"T": PROBE_T, "density": PROBE_DENSITY}[name]
        cap = max(1, (end_r - start_r) * max(end_z - start_z, 1)) if t == 0 else \
            max(1, end_r - start_r, end_z - start_z)
        out = np.empty(cap)
        n = ctypes.c_int64()
        self._check(self.L.pdp3g_probe_read_species(self.h, comp, sid, t, start_r, start_z,
                                                    end_r, end_z, _p(out), cap, ctypes.byref(n)),
                    "probe_read_species")
        return out[:n.value]

    def probe_particles(self, sid, start_r, start_z, end_r, end_z):
        """ProbePlain::mpwrite's selection: dict r, z, vr, vphi, vz."""
        cap = self.species_size(sid)
        out = {k: np.empty(max(cap, 1)) for k in ("r", "z", "vr", "vphi", "vz")}
        n = ctypes.c_int64()
        self._check(self.L.pdp3g_probe_particles(
            self.h, sid, start_r, start_z, end_r, end_z,
            *[_p(out[k]) for k in ("r", "z", "vr", "vphi", "vz")], cap, ctypes.byref(n)),
            "probe_particles")
        return {k: v[:n.value] for k, v in out.items()}

    def mark_initial_charge(self):
        self._check(self.L.pdp3g_mark_initial_charge(self.h), "mark_initial_charge")

    def diagnostics(self):
        d = Diag()
        self._check(self.L.pdp3g_diagnostics(self.h, ctypes.byref(d)), "diagnostics")
        return {f: getattr(d, f) for f, _ in Diag._fields_}

    def set_timing(self, on=True):
        self._check(self.L.pdp3g_set_timing(self.h, 1 if on else 0), "set_timing")

    def reset_timing(self):
        self._check(self.L.pdp3g_reset_timing(self.h), "reset_timing")

    def timing(self):
        t = Timing()
        self._check(self.L.pdp3g_get_timing(self.h, ctypes.byref(t)), "get_timing")
        return {f: getattr(t, f) for f, _ in Timing._fields_}

    @property
    def time(self):
        return self.L.pdp3g_current_time(self.h)

    @property
    def stream_ptr(self):
        return int(self.L.pdp3g_stream(self.h) or 0)

    @property
    def device_bytes(self):
        return int(self.L.pdp3g_device_bytes(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.L.pdp3g_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def from_workload(wl, precision="fp64", device=0, pusher=None, sort_interval=None):
    """Builds a Simulation holding a pdp3_b200.workloads.Workload (sort
    interval: the workload's unless given)."""
    if sort_interval is None:
        sort_interval = getattr(wl, "sort_interval", 0)
    sim = Simulation(wl.r_size, wl.z_size, wl.n_grid_r, wl.n_grid_z, wl.dt, pml=wl.pml,
                     pusher=pusher or wl.pusher, precision=precision, device=device,
                     sort_interval=sort_interval)
    for s in wl.species:
        sim.add_species(s.charge_e, s.mass_me, s.r, s.z, s.vr, s.vphi, s.vz, s.w)
    if getattr(wl, "device_plasma", None) is not None:
        wl.device_plasma.add_to(sim, device)
    if wl.beam is not None:
        b = wl.beam
        for nb in range(b.number_bunches):
            sim.add_bunch(b.charge_e, b.mass_me, b.number_macro, b.bunch_length / b.velocity,
                          b.radius, b.density, b.velocity, nb, b.bunches_distance / b.velocity)
    return sim


class Ensemble:
    """Independent FP32 runs advanced together by one persistent kernel."""

    def __init__(self, sims):
        self.L = load()
        self.sims = list(sims)
        arr = (_VP * len(self.sims))(*[s.h for s in self.sims])
        h = _VP()
        st = self.L.pdp3g_ensemble_create(arr, len(self.sims), ctypes.byref(h))
        if st != 0:
            msg = self.L.pdp3g_last_error(self.sims[0].h)
            raise Pdp3gError(st, "ensemble_create: %s" % (msg.decode() if msg else ""))
        self.h = h

    def _check(self, st, what):
        if st != 0:
            msg = self.L.pdp3g_ensemble_last_error(self.h)
            raise Pdp3gError(st, "%s: %s" % (what, msg.decode() if msg else ""))

    def run(self, nsteps):
        self._check(self.L.pdp3g_ensemble_run(self.h, int(nsteps)), "ensemble_run")

    def run_status(self, nsteps):
        return self.L.pdp3g_ensemble_run(self.h, int(nsteps))

    def autotune(self, steps_per_trial=2):
        b = _I32()
        self._check(self.L.pdp3g_ensemble_autotune(self.h, int(steps_per_trial), ctypes.byref(b)),
                    "ensemble_autotune")
        return b.value

    MODES = {"persistent": 0, "step_graph": 1}

    def set_mode(self, mode):
        """"persistent" (one cooperative kernel per call) or "step_graph" (one
        captured graph per step with every run's own kernels)."""
        self._check(self.L.pdp3g_ensemble_set_mode(self.h, self.MODES[mode]), "set_mode")

    def set_budget(self, max_ms):
        self._check(self.L.pdp3g_ensemble_set_budget(self.h, float(max_ms)), "set_budget")

    def set_sort_interval(self, steps):
        self._check(self.L.pdp3g_ensemble_set_sort_interval(self.h, int(steps)),
                    "set_sort_interval")

    def cancel(self, on=True):
        self._check(self.L.pdp3g_ensemble_cancel(self.h, 1 if on else 0), "cancel")

    def info(self):
        i = EnsembleInfo()
        self._check(self.L.pdp3g_ensemble_info(self.h, ctypes.byref(i)), "ensemble_info")
        return {f: getattr(i, f) for f, _ in EnsembleInfo._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.L.pdp3g_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Adjoint:
    """Forward/backward (vector-Jacobian) pair over a window of FP32 steps of
    one Simulation (precision "fp32", relativistic Boris).  loss = sum over
    the probe nodes [r0, r1) x [z0, z1) of E_z^2 times the node ring volume,
    after the window.  backward() returns nothing; the gradients with respect
    to the state at the start of the window are read with species(), field()
    and bunch_velocity()."""

    def __init__(self, sim, window_steps, checkpoint_interval, probe):
        self.L = load()
        self.sim = sim
        r0, r1, z0, z1 = (int(x) for x in probe)
        h = _VP()
        st = self.L.pdp3g_adjoint_create(sim.h, int(window_steps), int(checkpoint_interval),
                                         r0, r1, z0, z1, ctypes.byref(h))
        sim._check(st, "adjoint_create")
        self.h = h

    def forward(self):
        loss = ctypes.c_double()
        self.sim._check(self.L.pdp3g_forward_window(self.h, ctypes.byref(loss)), "forward_window")
        return loss.value

    def backward(self):
        self.sim._check(self.L.pdp3g_backward_window(self.h), "backward_window")

    def species(self, sid):
        """dL/d(initial state) of species sid: r, z (per metre), ur, uphi, uz
        (u = gamma v / c) and w (weight)."""
        n = self.sim.species_size(sid)
        out = {k: np.empty(n) for k in ("r", "z", "ur", "uphi", "uz", "w")}
        self.sim._check(self.L.pdp3g_adjoint_species(
            self.h, sid, *[_p(out[k]) for k in ("r", "z", "ur", "uphi", "uz", "w")]),
            "adjoint_species")
        return out

    def field(self, name):
        out = np.empty(self.sim.nr * self.sim.nz)
        self.sim._check(self.L.pdp3g_adjoint_field(self.h, COMP[name], _p(out)), "adjoint_field")
        return out.reshape(self.sim.nr, self.sim.nz)

    def bunch_velocity(self, sid):
        v = ctypes.c_double()
        self.sim._check(self.L.pdp3g_adjoint_bunch_velocity(self.h, sid, ctypes.byref(v)),
                        "adjoint_bunch_velocity")
        return v.value

    def set_mode(self, mode):
        """"mean_field" (default: adds the expected jump terms) or
        "pathwise" (the exact derivative of each particle's trajectory)."""
        self.sim._check(self.L.pdp3g_adjoint_set_mode(
            self.h, {"mean_field": 0, "pathwise": 1}[mode]), "adjoint_set_mode")

    def set_jump_terms(self, *terms):
        """The mean-field terms one by one: any of "gather" (the gather
        weights' jumps), "walls" (the momentum jumps of wall reflections),
        "wall_cells" (the axis and last radial cells hold their particles in
        the half the walls leave them; with the uniform jump density only,
        face width 0); none = pathwise."""
        bits = {"gather": 1, "walls": 2, "wall_cells": 4}
        self.sim._check(self.L.pdp3g_adjoint_set_jump_terms(
            self.h, sum(bits[t] for t in set(terms))), "adjoint_set_jump_terms")

    def set_face_width(self, half_width):
        """0: gather jump terms for a density uniform in each cell; h in
        (0, 0.5]: a box-kernel density estimate of half-width h cells."""
        self.sim._check(self.L.pdp3g_adjoint_set_face_width(self.h, float(half_width)),
                        "adjoint_set_face_width")

    def timing(self):
        f, b = ctypes.c_double(), ctypes.c_double()
        self.sim._check(self.L.pdp3g_adjoint_timing(self.h, ctypes.byref(f), ctypes.byref(b)),
                        "adjoint_timing")
        return {"forward_ms": f.value, "backward_ms": b.value}

    def device_bytes(self):
        return self.L.pdp3g_adjoint_bytes(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.pdp3g_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
