"""ctypes wrapper around oracle/liboracle_pic.so (the C restatement).

ORACLE ONLY (test infrastructure): tests/, the smoke check and bench.py's
CPU-baseline leg use it as the checker for the GPU path.  The product never
imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_pic.so")

COMP = {"E_r": 0, "E_phi": 1, "E_z": 2, "H_r": 3, "H_phi": 4, "H_z": 5,
        "H_r_half": 6, "H_phi_half": 7, "H_z_half": 8,
        "J_r": 9, "J_phi": 10, "J_z": 11, "sigma": 12}
PUSHERS = {"boris": 0, "vay": 1, "boris_classic": 2}

_D = ctypes.POINTER(ctypes.c_double)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_lib = None


def build():
    """Compiles the restatement (make -C oracle oracle)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = ctypes.CDLL(LIB_PATH)
    L.orc_create.restype = ctypes.c_void_p
    L.orc_create.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                             ctypes.c_double, ctypes.c_double, _D, ctypes.c_int]
    L.orc_destroy.argtypes = [ctypes.c_void_p]
    L.orc_add_species.restype = ctypes.c_int
    L.orc_add_species.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int] + [_D] * 6
    L.orc_add_bunch.restype = ctypes.c_int
    L.orc_add_bunch.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, ctypes.c_int, ctypes.c_double]
    L.orc_step.restype = ctypes.c_int
    L.orc_step.argtypes = [ctypes.c_void_p]
    L.orc_errors.restype = ctypes.c_int
    L.orc_errors.argtypes = [ctypes.c_void_p]
    L.orc_time.restype = ctypes.c_double
    L.orc_time.argtypes = [ctypes.c_void_p]
    L.orc_species_n.restype = ctypes.c_int
    L.orc_species_n.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.orc_get_grid.restype = ctypes.c_int
    L.orc_get_grid.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
    L.orc_set_grid.restype = ctypes.c_int
    L.orc_set_grid.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
    L.orc_get_species.restype = ctypes.c_int
    L.orc_get_species.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_D] * 6 + [_U8]
    L.orc_set_species.restype = ctypes.c_int
    L.orc_set_species.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_D] * 5 + [_U8]
    L.orc_charge_density.restype = None
    L.orc_charge_density.argtypes = [ctypes.c_void_p, ctypes.c_uint32, _D]
    L.orc_field_h.argtypes = [ctypes.c_void_p]
    L.orc_field_e.argtypes = [ctypes.c_void_p]
    L.orc_gather.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _D, _D]
    L.orc_random_reverse.restype = ctypes.c_double
    L.orc_random_reverse.argtypes = [ctypes.c_double, ctypes.c_int]
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(_D)


class OracleSim:
    """The C restatement of one PDP3 simulation (grids + species)."""

    def __init__(self, r_size, z_size, n_grid_r, n_grid_z, dt, current_time=0.0, pml=None,
                 pusher="boris"):
        self.L = load()
        self.nr, self.nz = n_grid_r, n_grid_z
        pml_arr = np.zeros(5) if pml is None else np.asarray(pml, dtype=np.float64)
        self.h = self.L.orc_create(r_size, z_size, n_grid_r, n_grid_z, dt, current_time,
                                   _p(pml_arr), PUSHERS[pusher])

    def add_species(self, charge_e, mass_me, r, z, vr, vphi, vz, w):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (r, z, vr, vphi, vz, w)]
        return self.L.orc_add_species(self.h, charge_e, mass_me, len(arrs[0]),
                                      *[_p(a) for a in arrs])

    def add_bunch(self, charge_e, mass_me, n, duration, radius, density, velocity,
                  bunch_number=0, hole_duration=0.0):
        return self.L.orc_add_bunch(self.h, charge_e, mass_me, int(n), duration, radius,
                                    density, velocity, int(bunch_number), hole_duration)

    def step(self):
        return self.L.orc_step(self.h)

    def run(self, n):
        for _ in range(n):
            self.step()

    @property
    def errors(self):
        return self.L.orc_errors(self.h)

    @property
    def time(self):
        return self.L.orc_time(self.h)

    def field(self, name):
        out = np.zeros(self.nr * self.nz)
        assert self.L.orc_get_grid(self.h, COMP[name], _p(out)) == 0
        return out.reshape(self.nr, self.nz)

    def set_field(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        assert self.L.orc_set_grid(self.h, COMP[name], _p(a)) == 0

    def species(self, idx):
        n = self.L.orc_species_n(self.h, idx)
        out = {k: np.zeros(n) for k in ("r", "z", "vr", "vphi", "vz", "w")}
        alive = np.zeros(n, dtype=np.uint8)
        assert self.L.orc_get_species(self.h, idx, *[_p(out[k]) for k in
                                                      ("r", "z", "vr", "vphi", "vz", "w")],
                                      alive.ctypes.data_as(_U8)) == 0
        out["alive"] = alive
        return out

    def set_species(self, idx, r=None, z=None, vr=None, vphi=None, vz=None, alive=None):
        def p(a):
            if a is None:
                return None
            return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_D)
        keep = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in (r, z, vr, vphi, vz)]
        al = None if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
        assert self.L.orc_set_species(
            self.h, idx, *[(_p(a) if a is not None else None) for a in keep],
            al.ctypes.data_as(_U8) if al is not None else None) == 0

    def charge_density(self, mask=0xFFFFFFFF):
        out = np.zeros(self.nr * self.nz)
        self.L.orc_charge_density(self.h, mask, _p(out))
        return out.reshape(self.nr, self.nz)

    def field_h(self):
        self.L.orc_field_h(self.h)

    def field_e(self):
        self.L.orc_field_e(self.h)

    def gather(self, r, z):
        e = np.zeros(3)
        b = np.zeros(3)
        self.L.orc_gather(self.h, r, z, _p(e), _p(b))
        return e, b

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def random_reverse(x, power):
    return load().orc_random_reverse(float(x), int(power))
