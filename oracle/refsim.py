"""ctypes wrapper around oracle/_ref/libpdp3ref_<pusher>.so.

ORACLE ONLY (test infrastructure): the library is the unmodified upstream
PDP3 hot-path sources plus oracle/ref_driver.cpp.  Only tests/, the smoke
check and bench.py's CPU-baseline leg may load it, as a checker or as the
timed CPU reference; the GPU product never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

# Component ids understood by ref_get_field (see oracle/ref_driver.cpp).
COMP = {"E_r": 0, "E_phi": 1, "E_z": 2, "H_r": 3, "H_phi": 4, "H_z": 5,
        "H_r_half": 6, "H_phi_half": 7, "H_z_half": 8,
        "J_r": 9, "J_phi": 10, "J_z": 11, "rho_bunch": 12, "rho_beam": 13}

_D = ctypes.POINTER(ctypes.c_double)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_libs = {}


def lib_path(pusher="boris"):
    return os.path.join(REF_DIR, "libpdp3ref_%s.so" % pusher)


def available(pusher="boris"):
    return os.path.exists(lib_path(pusher))


def load(pusher="boris"):
    if pusher in _libs:
        return _libs[pusher]
    path = lib_path(pusher)
    if not os.path.exists(path):
        raise FileNotFoundError(
            "%s is not built (it is compiled from the upstream sources by "
            "oracle/Makefile)" % path)
    L = ctypes.CDLL(path)
    L.ref_create.restype = ctypes.c_void_p
    L.ref_create.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                             ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]
    L.ref_add_species.restype = ctypes.c_int
    L.ref_add_species.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int] + [_D] * 6
    L.ref_add_species_upstream_init.restype = ctypes.c_int
    L.ref_add_species_upstream_init.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                                ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.ref_set_beam.restype = None
    L.ref_set_beam.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                               ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, ctypes.c_int, ctypes.c_double]
    L.ref_step.restype = ctypes.c_int
    L.ref_step.argtypes = [ctypes.c_void_p]
    L.ref_run.restype = ctypes.c_double
    L.ref_run.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.ref_current_time.restype = ctypes.c_double
    L.ref_current_time.argtypes = [ctypes.c_void_p]
    L.ref_species_count.restype = ctypes.c_int
    L.ref_species_count.argtypes = [ctypes.c_void_p]
    L.ref_species_number.restype = ctypes.c_int
    L.ref_species_number.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.ref_get_field.restype = ctypes.c_int
    L.ref_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
    L.ref_set_field.restype = ctypes.c_int
    L.ref_set_field.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
    L.ref_get_species.restype = ctypes.c_int
    L.ref_get_species.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_D] * 7 + [_U8]
    L.ref_charge_density.restype = None
    L.ref_charge_density.argtypes = [ctypes.c_void_p, _D]
    for f in (L.ref_temperature, L.ref_density):
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
    L.ref_poisson_dirichlet.restype = ctypes.c_int
    L.ref_poisson_dirichlet.argtypes = [ctypes.c_void_p] + [_D] * 4
    L.ref_sigma.restype = ctypes.c_double
    L.ref_sigma.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.ref_destroy.restype = None
    L.ref_destroy.argtypes = [ctypes.c_void_p]
    L.ref_set_threads.restype = None
    L.ref_set_threads.argtypes = [ctypes.c_int]
    L.ref_max_threads.restype = ctypes.c_int
    L.ref_max_threads.argtypes = []
    _libs[pusher] = L
    return L


def _p(a):
    return a.ctypes.data_as(_D)


class RefSim:
    """One upstream simulation (Geometry/Time/fields/species) behind ref_driver."""

    def __init__(self, r_size, z_size, n_grid_r, n_grid_z, dt, end_time=1.0,
                 current_time=0.0, pml=None, pusher="boris"):
        self.L = load(pusher)
        self.nr, self.nz = n_grid_r, n_grid_z
        pml_arr = np.zeros(5) if pml is None else np.asarray(pml, dtype=np.float64)
        self.h = self.L.ref_create(r_size, z_size, n_grid_r, n_grid_z, dt, current_time,
                                   end_time, _p(pml_arr))

    def add_species(self, name, charge_e, mass_me, r, z, vr, vphi, vz, w):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (r, z, vr, vphi, vz, w)]
        return self.L.ref_add_species(self.h, name.encode(), charge_e, mass_me, len(arrs[0]),
                                      *[_p(a) for a in arrs])

    def add_species_upstream_init(self, name, charge_e, mass_me, n, left_density,
                                  right_density, temperature):
        return self.L.ref_add_species_upstream_init(self.h, name.encode(), charge_e, mass_me,
                                                    int(n), left_density, right_density,
                                                    temperature)

    def set_beam(self, charge_e, mass_me, number_macro, bunch_length, radius, density,
                 velocity, number_bunches=1, bunches_distance=0.0):
        self.L.ref_set_beam(self.h, charge_e, mass_me, int(number_macro), bunch_length,
                            radius, density, velocity, int(number_bunches), bunches_distance)

    def step(self):
        return self.L.ref_step(self.h)

    def run(self, n):
        return self.L.ref_run(self.h, int(n))

    @property
    def time(self):
        return self.L.ref_current_time(self.h)

    def field(self, name):
        out = np.zeros(self.nr * self.nz)
        rc = self.L.ref_get_field(self.h, COMP[name], _p(out))
        assert rc == 0
        return out.reshape(self.nr, self.nz)

    def set_field(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        assert self.L.ref_set_field(self.h, COMP[name], _p(a)) == 0

    def n_species(self):
        return self.L.ref_species_count(self.h)

    def species(self, idx):
        n = self.L.ref_species_number(self.h, idx)
        out = {k: np.zeros(n) for k in ("r", "z", "vr", "vphi", "vz", "q", "m")}
        alive = np.zeros(n, dtype=np.uint8)
        rc = self.L.ref_get_species(self.h, idx, *[_p(out[k]) for k in
                                                   ("r", "z", "vr", "vphi", "vz", "q", "m")],
                                    alive.ctypes.data_as(_U8))
        assert rc == 0
        out["alive"] = alive
        return out

    def charge_density(self):
        out = np.zeros(self.nr * self.nz)
        self.L.ref_charge_density(self.h, _p(out))
        return out.reshape(self.nr, self.nz)

    def temperature(self, idx):
        """TemperatureClassic of list entry idx: [n_grid_r-1, n_grid_z-1]."""
        out = np.zeros((self.nr - 1) * (self.nz - 1))
        rc = self.L.ref_temperature(self.h, idx, _p(out))
        assert rc == 0, rc
        return out.reshape(self.nr - 1, self.nz - 1)

    def density(self, idx):
        """ParticlesDensity of list entry idx: [n_grid_r, n_grid_z]."""
        out = np.zeros(self.nr * self.nz)
        rc = self.L.ref_density(self.h, idx, _p(out))
        assert rc == 0, rc
        return out.reshape(self.nr, self.nz)

    def poisson_dirichlet(self, rho):
        """PoissonDirichlet::poisson_solve on rho: (phi, E_r, E_z)."""
        rho = np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)
        outs = [np.zeros(self.nr * self.nz) for _ in range(3)]
        assert self.L.ref_poisson_dirichlet(self.h, _p(rho), *[_p(o) for o in outs]) == 0
        return tuple(o.reshape(self.nr, self.nz) for o in outs)

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
