"""ctypes backend over the reference-source oracle (oracle/_ref, built by
oracle/build_ref.sh from SAMoS's own hot-path sources).

TEST INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's reference arm
and CPU-baseline leg.  :class:`RefSimulation` takes the conf-level commands
that :class:`samos_b200.plugins.Simulation` takes (box, input, nlist,
constraint, pair_potential, pair_param, pair_align, align_param, external,
external_param, timestep, integrator, disable, run) and hands their parameter
blocks, as text, to the reference's own classes, so one scenario drives the
reference, the C oracle and the GPU engine alike.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_STRICT = os.path.join(REF_DIR, "libsamos_ref.so")
LIB_FAST = os.path.join(REF_DIR, "libsamos_ref_fast.so")
_libs: dict[str, C.CDLL] = {}

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "tau_x", "tau_y", "tau_z", "nx", "ny", "nz",
          "Nx", "Ny", "Nz", "omega", "age", "radius", "mass", "ix", "iy", "iz", "type")
# columns the reference's particle reader takes under `keys:` (system.cpp:170-330)
INPUT_KEYS = ("type", "radius", "x", "y", "z", "vx", "vy", "vz", "nx", "ny", "nz", "omega", "ix", "iy", "iz",
              "mass")


def available(fast: bool = False) -> bool:
    return os.path.exists(LIB_FAST if fast else LIB_STRICT)


def build(src: str = "/root/reference/src") -> None:
    subprocess.run([os.path.join(HERE, "build_ref.sh"), src], check=True)


def load(fast: bool = False) -> C.CDLL:
    path = LIB_FAST if fast else LIB_STRICT
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (oracle/build_ref.sh)")
    lib = C.CDLL(path)
    P, I, D, S = C.c_void_p, C.c_int, C.c_double, C.c_char_p
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    sig = {
        "rs_create": (P, [S]), "rs_destroy": (None, [P]), "rs_error": (S, [P]),
        "rs_box": (I, [P, D, D, D, I]), "rs_input": (I, [P, S]), "rs_size": (I, [P]),
        "rs_nlist": (I, [P, S]), "rs_constraint": (I, [P, S, S]), "rs_group": (I, [P, S, S]),
        "rs_pair_potential": (I, [P, S, S]), "rs_pair_param": (I, [P, S, S]),
        "rs_external": (I, [P, S, S]), "rs_external_param": (I, [P, S, S]),
        "rs_pair_align": (I, [P, S, S]), "rs_align_param": (I, [P, S, S]),
        "rs_timestep": (I, [P, D]), "rs_integrator": (I, [P, S, S]), "rs_disable": (I, [P, S, S]),
        "rs_compute": (I, [P]), "rs_run": (I, [P, I]), "rs_nlist_builds": (I, [P]),
        "rs_build_nlist": (I, [P]), "rs_get": (I, [P, S, dp]), "rs_pairs": (I, [P, ip, ip, I]),
        "rs_energy": (I, [P, I, S, dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _libs[path] = lib
    return lib


class RefError(RuntimeError):
    """The reference logged Messenger::ERROR and threw."""


def _block(params: dict | None) -> bytes:
    """{"k": "10", "use_particle_radii": ""} -> b"k=10;use_particle_radii"."""
    items = []
    for k, v in (params or {}).items():
        items.append(k if v in ("", None) else f"{k}={v}")
    return ";".join(items).encode()


def _num(v) -> str:
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v))  # shortest round-trip text: strtod reads the same double back


class RefSimulation:
    """The hot-path subset of the `samos` command loop over the reference's
    own objects.  Method names and argument meaning follow
    samos_b200.plugins.Simulation."""

    def __init__(self, fast: bool = False, ntypes: int = 1):
        self.lib = load(fast)
        self.h = self.lib.rs_create(b"/dev/null")
        self.ntypes = ntypes
        self.n = 0
        self._tmp = tempfile.TemporaryDirectory(prefix="samos_ref_")
        self._box = None

    def close(self):
        if self.h:
            self.lib.rs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, rc):
        if rc != 0:
            raise RefError(self.lib.rs_error(self.h).decode())

    # conf commands ---------------------------------------------------------
    def box(self, lx, ly, lz, periodic=True):
        self._ok(self.lib.rs_box(self.h, float(lx), float(ly), float(lz), int(bool(periodic))))

    def input(self, **arrays):
        """Writes the arrays as a `keys:` particle file (17 significant
        digits, read back exactly by the reference's reader) and reads it
        with System's constructor."""
        n = len(next(iter(arrays.values())))
        cols = [k for k in INPUT_KEYS if k in arrays]
        path = os.path.join(self._tmp.name, "particles.dat")
        with open(path, "w") as f:
            f.write("keys: id " + " ".join(cols) + "\n")
            data = [np.asarray(arrays[k]) for k in cols]
            for i in range(n):
                f.write(str(i) + " " + " ".join(_num(a[i]) for a in data) + "\n")
        self._ok(self.lib.rs_input(self.h, path.encode()))
        self.n = int(self.lib.rs_size(self.h))

    def input_file(self, path):
        """input <file>: a particle file as the reference reads it."""
        self._ok(self.lib.rs_input(self.h, os.fspath(path).encode()))
        self.n = int(self.lib.rs_size(self.h))

    def nlist(self, rcut=3.0, pad=0.5):
        self._ok(self.lib.rs_nlist(self.h, _block({"rcut": _num(rcut), "pad": _num(pad)})))

    def group(self, name, params=None):
        self._ok(self.lib.rs_group(self.h, name.encode(), _block(params)))

    def constraint(self, name, params=None):
        self._ok(self.lib.rs_constraint(self.h, name.encode(), _block(params)))

    def pair_potential(self, name, params=None):
        self._ok(self.lib.rs_pair_potential(self.h, name.encode(), _block(params)))

    def pair_param(self, name, params):
        self._ok(self.lib.rs_pair_param(self.h, name.encode(), _block(params)))

    def pair_align(self, name, params=None):
        self._ok(self.lib.rs_pair_align(self.h, name.encode(), _block(params)))

    def align_param(self, name, params):
        self._ok(self.lib.rs_align_param(self.h, name.encode(), _block(params)))

    def external(self, name, params=None):
        self._ok(self.lib.rs_external(self.h, name.encode(), _block(params)))

    def external_param(self, name, params):
        self._ok(self.lib.rs_external_param(self.h, name.encode(), _block(params)))

    def timestep(self, dt):
        self._ok(self.lib.rs_timestep(self.h, float(dt)))

    def integrator(self, name, params=None):
        self._ok(self.lib.rs_integrator(self.h, name.encode(), _block(params)))

    def disable(self, name, group="all"):
        self._ok(self.lib.rs_disable(self.h, name.encode(), group.encode()))

    def commit(self):
        pass

    def run(self, steps):
        self._ok(self.lib.rs_run(self.h, int(steps)))

    # state -----------------------------------------------------------------
    def compute(self):
        """One top-of-step force and torque evaluation."""
        self._ok(self.lib.rs_compute(self.h))

    def build_nlist(self):
        self._ok(self.lib.rs_build_nlist(self.h))

    def nlist_builds(self) -> int:
        return int(self.lib.rs_nlist_builds(self.h))

    def download(self, field):
        out = np.empty(self.n, np.float64)
        self._ok(self.lib.rs_get(self.h, field.encode(), out.ctypes.data_as(C.POINTER(C.c_double))))
        if field in ("ix", "iy", "iz", "type"):
            return out.astype(np.int32)
        return out

    def pairs(self):
        """The half neighbour list in the reference's storage order."""
        m = -self.lib.rs_pairs(self.h, None, None, 0)
        i = np.empty(max(m, 1), np.int32)
        j = np.empty(max(m, 1), np.int32)
        got = self.lib.rs_pairs(self.h, i.ctypes.data_as(C.POINTER(C.c_int)), j.ctypes.data_as(C.POINTER(C.c_int)),
                                max(m, 1))
        return i[:got], j[:got]

    def energy(self, cls, name):
        out = C.c_double()
        self._ok(self.lib.rs_energy(self.h, int(cls), name.encode(), C.byref(out)))
        return float(out.value)


def drive_ref(parts, box, periodic=True, nlist=(2.4, 0.3), constraint=("plane", {}), pairs=(), aligns=(),
              externals=(), dt=1e-3, integrators=(), pair_params=(), align_params=(), fast=False):
    """The command sequence of tests/scenarios.drive, on the reference."""
    sim = RefSimulation(fast=fast)
    sim.box(*box, periodic)
    sim.input(**parts)
    if nlist is not None:
        sim.nlist(*nlist)
    if constraint is not None:
        sim.constraint(*constraint)
    for name, p in pairs:
        sim.pair_potential(name, dict(p))
    for name, p in pair_params:
        sim.pair_param(name, dict(p))
    for name, p in aligns:
        sim.pair_align(name, dict(p))
    for name, p in align_params:
        sim.align_param(name, dict(p))
    for name, p in externals:
        sim.external(name, dict(p))
    sim.timestep(dt)
    for name, p in integrators:
        sim.integrator(name, dict(p))
    return sim
