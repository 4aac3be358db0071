"""ctypes backend over the CPU oracle (oracle/samos_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg.  It offers the same method surface as
samos_b200.engine.Engine so one scenario can be driven through both.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsamos_oracle.so")
_lib = None

DOUBLE_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "tau_x", "tau_y", "tau_z",
                 "nx", "ny", "nz", "Nx", "Ny", "Nz", "omega", "age", "radius", "mass")
INT_FIELDS = ("type", "ix", "iy", "iz")


def build() -> str:
    subprocess.run([os.path.join(HERE, "build.sh")], check=True)
    return LIB_PATH


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    P, I, D = C.c_void_p, C.c_int, C.c_double
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    sig = {
        "or_create": (P, [I, I]), "or_destroy": (None, [P]), "or_size": (I, [P]),
        "or_field": (dp, [P, C.c_char_p]), "or_ifield": (ip, [P, C.c_char_p]),
        "or_set_box": (None, [P, D, D, D, I]), "or_set_timestep": (None, [P, D]),
        "or_set_nlist": (I, [P, D, D]), "or_build_nlist": (I, [P]),
        "or_nlist_uses_cells": (I, [P]), "or_nlist_builds": (I, [P]),
        "or_get_pairs": (I, [P, ip, ip, I]),
        "or_add_pair": (I, [P, I, dp, dp, I, I, I, I, dp]),
        "or_add_align": (I, [P, I, D, D, dp, I]),
        "or_add_external": (I, [P, I, D, dp, I]),
        "or_add_constraint": (I, [P, I, dp]),
        "or_define_group": (I, [P, I, C.c_void_p]),
        "or_set_integrator_group": (I, [P, I, I]),
        "or_add_integrator": (I, [P, I, dp, dp]),
        "or_integrator_state": (I, [P, I, dp]),
        "or_compute": (None, [P, D]), "or_enforce_all": (None, [P]),
        "or_run": (I, [P, I]), "or_run_until_converged": (I, [P, I]),
        "or_pair_energy": (D, [P, I]), "or_align_energy": (D, [P, I]),
        "or_total_potential_energy": (D, [P]),
        "or_noise_gauss": (D, [C.c_uint32, C.c_uint64]),
        "or_noise_uniform": (D, [C.c_uint32, C.c_uint64]),
        "or_noise_log": (D, [D]),
        "or_noise_cos2pi": (D, [D]),
        "or_philox4x32_10": (None, [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class OracleSystem:
    """One system on the CPU oracle; mirrors samos_b200.engine.Engine."""

    def __init__(self, n: int, ntypes: int = 1):
        self.lib = load()
        self.n = [int(n)]
        self.ntypes = ntypes
        self.h = self.lib.or_create(int(n), int(ntypes))
        self._aligns = 0

    def close(self):
        if self.h:
            self.lib.or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_box(self, lx, ly, lz, periodic=True, replica=None):
        self.lib.or_set_box(self.h, lx, ly, lz, int(bool(periodic)))

    def set_timestep(self, dt):
        self.lib.or_set_timestep(self.h, float(dt))

    def _view(self, field):
        if field in INT_FIELDS:
            ptr = self.lib.or_ifield(self.h, field.encode())
            return np.ctypeslib.as_array(ptr, shape=(self.n[0],))
        ptr = self.lib.or_field(self.h, field.encode())
        if not ptr:
            raise KeyError(field)
        return np.ctypeslib.as_array(ptr, shape=(self.n[0],))

    def upload(self, field, values, replica=0):
        self._view(field)[:] = values

    def download(self, field, replica=0):
        return self._view(field).copy()

    def set_nlist(self, rcut, pad):
        self.lib.or_set_nlist(self.h, float(rcut), float(pad))

    def build_nlist(self):
        self.lib.or_build_nlist(self.h)

    def uses_cells(self) -> bool:
        return bool(self.lib.or_nlist_uses_cells(self.h))

    def nlist_builds(self) -> int:
        return int(self.lib.or_nlist_builds(self.h))

    def pairs(self, replica=0):
        n = -self.lib.or_get_pairs(self.h, None, None, 0)
        n = max(n, 1)
        i = np.empty(n, np.int32)
        j = np.empty(n, np.int32)
        m = self.lib.or_get_pairs(self.h, i.ctypes.data_as(C.POINTER(C.c_int)),
                                  j.ctypes.data_as(C.POINTER(C.c_int)), n)
        return i[:m], j[:m]

    def add_pair(self, kind, global_params, table=None, use_radii=False, phase_in=False,
                 shifted=False, has_pair_params=False, phase_value=None):
        g = np.zeros(8)
        g[:len(global_params)] = global_params
        t, pv = _d(table), _d(phase_value)
        self.lib.or_add_pair(self.h, int(kind), _p(g), _p(t), int(use_radii), int(phase_in),
                             int(shifted), int(has_pair_params), _p(pv))

    def add_align(self, kind, J, rcut, table=None, has_pair_params=False):
        t = _d(table)
        self.lib.or_add_align(self.h, int(kind), float(J), float(rcut), _p(t), int(has_pair_params))

    def add_external(self, kind, alpha, type_alpha=None, has_params=False):
        t = _d(type_alpha)
        self.lib.or_add_external(self.h, int(kind), float(alpha), _p(t), int(has_params))

    def add_constraint(self, kind, params):
        p = np.zeros(9)
        p[:len(params)] = params
        if self.lib.or_add_constraint(self.h, int(kind), _p(p)) != 0:
            raise ValueError("constraint parameters rejected (as the reference constructor rejects them)")
        self.lib.or_enforce_all(self.h)  # samos.cpp:518-522

    def add_integrator(self, kind, params, temperature=None):
        p = np.zeros(16)
        p[:len(params)] = params
        t = _d(temperature)
        self.lib.or_add_integrator(self.h, int(kind), _p(p), _p(t))

    def define_group(self, group, member, replica=0):
        m = np.ascontiguousarray(member, dtype=np.uint8)
        if self.lib.or_define_group(self.h, int(group), m.ctypes.data) != 0:
            raise ValueError("bad group index")

    def set_integrator_group(self, index, group):
        if self.lib.or_set_integrator_group(self.h, int(index), int(group)) != 0:
            raise ValueError("bad integrator or group index")

    def compute(self, dt):
        self.lib.or_compute(self.h, float(dt))

    def enforce(self):
        self.lib.or_enforce_all(self.h)

    def run(self, steps):
        self.lib.or_run(self.h, int(steps))

    def minimize(self, max_steps):
        return np.array([self.lib.or_run_until_converged(self.h, int(max_steps))]), None

    def energy(self, cls, comp, replica=0):
        if cls == 0:
            return float(self.lib.or_pair_energy(self.h, comp))
        return float(self.lib.or_align_energy(self.h, comp))

    def fire_state(self, replica=0, idx=0):
        out = np.zeros(8)
        self.lib.or_integrator_state(self.h, idx, _p(out))
        return np.array([out[0], out[1], out[2], out[3], out[4]])


def noise_gauss(seed: int, counter: int) -> float:
    return float(load().or_noise_gauss(seed & 0xffffffff, counter))


def noise_uniform(seed: int, counter: int) -> float:
    return float(load().or_noise_uniform(seed & 0xffffffff, counter))


def noise_log(x: float) -> float:
    return float(load().or_noise_log(x))


def noise_cos2pi(u: float) -> float:
    return float(load().or_noise_cos2pi(u))


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    load().or_philox4x32_10(c, k, o)
    return list(o)
