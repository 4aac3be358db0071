"""ctypes binding of the C ABI in include/samos_gpu.h.

The binding is deliberately thin: every method forwards to one ``sg_*``
entry point and turns a negative status into :class:`EngineError` carrying
``sg_last_error``.  Loading fails loudly when the CUDA library has not been
built -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import weakref

import numpy as np

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsamos_gpu.so")
_lib = None

PAIR = {"soft": 0, "lj": 1, "morse": 2, "gaussian": 3}
ALIGN = {"polar": 0, "nematic": 1, "vicsek": 2}
EXTERNAL = {"self_propulsion": 0}
CONSTRAINT = {"none": 0, "plane": 1, "sphere": 2, "cylinder": 3, "torus": 4, "ellipsoid": 5, "peanut": 6,
              "gyroid": 7, "hourglass": 8, "gaussian_bump": 9, "slab": 10, "walls": 11,
              "tetrahedron": 12}
INTEGRATOR = {"brownian": 0, "brownian_pos": 1, "brownian_align": 2, "langevin": 3, "fire": 4, "nve": 5, "vicsek": 6}
PAIR_NPARAM = 8
INT_NPARAM = 16

DOUBLE_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "tau_x", "tau_y", "tau_z",
                 "nx", "ny", "nz", "Nx", "Ny", "Nz", "omega", "age", "radius", "mass")
INT_FIELDS = ("type", "ix", "iy", "iz")


class EngineError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"samos_gpu error {code}: {msg}")
        self.code = code


class View(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ("x", "y", "z", "nx", "ny", "nz", "vx", "vy", "vz", "fx", "fy", "fz",
                                           "radius", "id", "nb", "nb_cnt", "ix", "iy")] + \
               [("nb_stride", C.c_int32), ("slots", C.c_int32)]


class RunStats(C.Structure):
    _fields_ = [("steps_done", C.c_int64), ("nlist_builds", C.c_int64),
                ("kernel_launches", C.c_int64), ("max_neighbours", C.c_int32),
                ("status", C.c_int32), ("device_ms", C.c_double), ("step_kernel_ms", C.c_double),
                ("step_kernels", C.c_int64), ("rebuild_ms", C.c_double)]


def library_path() -> str:
    return _LIB_PATH


def load() -> C.CDLL:
    """Load libsamos_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} is missing: build it with "
                          "`python -m samos_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(_LIB_PATH)
    P, I, D, I64 = C.c_void_p, C.c_int, C.c_double, C.c_int64
    dp = C.POINTER(C.c_double)
    sig = {
        "sg_create": (I, [I, C.POINTER(C.c_int32), I, C.POINTER(P)]),
        "sg_destroy": (I, [P]),
        "sg_error_string": (C.c_char_p, [I]),
        "sg_last_error": (C.c_char_p, [P]),
        "sg_set_box": (I, [P, I, D, D, D, I]),
        "sg_set_timestep": (I, [P, D]),
        "sg_upload": (I, [P, I, C.c_char_p, P]),
        "sg_download": (I, [P, I, C.c_char_p, P]),
        "sg_set_nlist": (I, [P, D, D]),
        "sg_build_nlist": (I, [P]),
        "sg_get_pairs": (I, [P, I, C.POINTER(C.c_int32), C.POINTER(C.c_int32), I64, C.POINTER(I64)]),
        "sg_add_pair": (I, [P, I, dp, dp, I, I, I, I, dp]),
        "sg_add_align": (I, [P, I, D, D, dp, I]),
        "sg_add_external": (I, [P, I, D, dp, I]),
        "sg_add_constraint": (I, [P, I, dp]),
        "sg_add_constraint_per_replica": (I, [P, I, dp, dp]),
        "sg_add_integrator": (I, [P, I, dp, dp]),
        "sg_set_replica_param": (I, [P, I, I, I, I, D]),
        "sg_compute": (I, [P, D]),
        "sg_enforce": (I, [P]),
        "sg_run": (I, [P, I64, C.POINTER(RunStats)]),
        "sg_run_continue": (I, [P, I64, C.POINTER(RunStats)]),
        "sg_begin_step": (I, [P]),
        "sg_insert_integrator": (I, [P, I, I, dp, dp]),
        "sg_disable_integrator": (I, [P, I]),
        "sg_clear_forces": (I, [P]),
        "sg_minimize": (I, [P, I64, C.POINTER(I64), C.POINTER(RunStats)]),
        "sg_energy": (I, [P, I, I, I, dp]),
        "sg_fire_state": (I, [P, I, dp]),
        "sg_kernel_launches": (I64, [P]),
        "sg_set_profiling": (I, [P, I]),
        "sg_set_device": (I, [I]),
        "sg_set_path": (I, [P, I]),
        "sg_get_view": (I, [P, C.POINTER(View)]),
        "sg_replica_slots": (I, [P, I, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "sg_positions_changed": (I, [P]),
        "sg_memcpy": (I, [P, P, I64]),
        "sg_host_alloc": (I, [I64, C.POINTER(P)]),
        "sg_coordination": (I, [P, I, C.POINTER(C.c_int32)]),
        "sg_define_group": (I, [P, I, I, P]),
        "sg_set_integrator_group": (I, [P, I, I]),
        "sg_host_free": (I, [P]),
        "sg_set_variant": (I, [P, I]),
        "sg_set_build": (I, [P, I]),
        "sg_set_fire_order": (I, [P, I]),
        "sg_upload_fields": (I, [P, I, I, C.POINTER(C.c_char_p), C.POINTER(C.c_void_p)]),
        "sg_download_fields": (I, [P, I, I, C.POINTER(C.c_char_p), C.POINTER(C.c_void_p)]),
        "sg_set_generic_occupancy": (I, [P, I]), "sg_get_generic_occupancy": (I, [P]),
        "sg_get_variant": (I, [P]),
        "sg_compute_static": (I, [I, D, D, D, I, D, D] + [P] * 7 + [D, D, I, I, D, D] + [P] * 6 + [P]),
        "sg_compute_static_scratch_bytes": (I64, []),
        "sg_compute_static_overflow": (I, [C.POINTER(C.c_int), P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def pinned_empty(n: int, dtype=np.float64) -> np.ndarray:
    """A numpy array of n elements in page-locked host memory (sg_host_alloc),
    freed when the array is garbage-collected.  Uploads from and downloads into
    such arrays run at the link's speed."""
    lib = load()
    dt = np.dtype(dtype)
    nbytes = max(1, int(n) * dt.itemsize)
    p = C.c_void_p()
    rc = lib.sg_host_alloc(nbytes, C.byref(p))
    if rc != 0 or not p.value:
        raise EngineError(rc or -3, "page-locked host allocation failed")
    buf = (C.c_char * nbytes).from_address(p.value)
    a = np.frombuffer(buf, dtype=dt, count=int(n))
    weakref.finalize(buf, lib.sg_host_free, C.c_void_p(p.value))
    return a


def pinned_copy(values, dtype=np.float64) -> np.ndarray:
    """Page-locked copy of an array (see pinned_empty)."""
    v = np.ascontiguousarray(values, dtype=dtype)
    a = pinned_empty(v.size, dtype)
    a[:] = v.ravel()
    return a


def _arr(a):
    """float64 contiguous copy (or None); the caller keeps it alive across the call."""
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _dptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class Engine:
    """One device ensemble of ``len(n_particles)`` replicas."""

    def __init__(self, n_particles, ntypes: int = 1, device: int | None = None):
        self.lib = load()
        if device is not None and self.lib.sg_set_device(int(device)) != 0:
            raise EngineError(-2, f"cannot select CUDA device {device}")
        if np.isscalar(n_particles):
            n_particles = [int(n_particles)]
        self.n = [int(v) for v in n_particles]
        self.ntypes = int(ntypes)
        arr = (C.c_int32 * len(self.n))(*self.n)
        h = C.c_void_p()
        rc = self.lib.sg_create(len(self.n), arr, self.ntypes, C.byref(h))
        if rc != 0:
            raise EngineError(rc, self.lib.sg_error_string(rc).decode())
        self.h = h

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise EngineError(rc, self.lib.sg_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.sg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- configuration -----------------------------------------------------
    def set_box(self, lx, ly, lz, periodic=True, replica=None):
        if not hasattr(self, "boxes"):
            self.boxes = [None] * len(self.n)
        for r in (range(len(self.n)) if replica is None else [replica]):
            self._check(self.lib.sg_set_box(self.h, r, lx, ly, lz, int(bool(periodic))))
            self.boxes[r] = (float(lx), float(ly), float(lz), bool(periodic))

    def set_timestep(self, dt):
        self._check(self.lib.sg_set_timestep(self.h, float(dt)))

    def upload(self, field: str, values, replica: int = 0):
        dtype = np.int32 if field in INT_FIELDS else np.float64
        a = np.ascontiguousarray(values, dtype=dtype)
        if a.shape != (self.n[replica],):
            raise ValueError(f"{field}: expected {self.n[replica]} values, got {a.shape}")
        self._check(self.lib.sg_upload(self.h, replica, field.encode(), a.ctypes.data_as(C.c_void_p)))

    def upload_fields(self, arrays: dict, replica: int = 0) -> None:
        """Several fields at once ({name: values}): copies enqueued back to back, one wait."""
        names, bufs = [], []
        for field, values in arrays.items():
            dtype = np.int32 if field in INT_FIELDS else np.float64
            a = values if (isinstance(values, np.ndarray) and values.dtype == dtype and values.flags.c_contiguous) \
                else np.ascontiguousarray(values, dtype=dtype)
            if a.shape != (self.n[replica],):
                raise ValueError(f"{field}: expected {self.n[replica]} values, got {a.shape}")
            names.append(field.encode())
            bufs.append(a)
        cn = (C.c_char_p * len(names))(*names)
        cp = (C.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
        self._check(self.lib.sg_upload_fields(self.h, replica, len(names), cn, cp))

    def download_fields(self, fields, replica: int = 0, out: dict | None = None) -> dict:
        """Several fields at once; written into `out[field]` arrays when given."""
        res = {}
        for f in fields:
            dtype = np.int32 if f in INT_FIELDS else np.float64
            a = out[f] if out is not None and f in out else np.empty(self.n[replica], dtype=dtype)
            if a.dtype != dtype or a.shape != (self.n[replica],) or not a.flags.c_contiguous or not a.flags.writeable:
                raise ValueError(f"{f}: out must be a writeable contiguous {dtype} array of {self.n[replica]}")
            res[f] = a
        cn = (C.c_char_p * len(res))(*[f.encode() for f in res])
        cp = (C.c_void_p * len(res))(*[a.ctypes.data for a in res.values()])
        self._check(self.lib.sg_download_fields(self.h, replica, len(res), cn, cp))
        return res

    def download(self, field: str, replica: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """The field in particle-id order; written into `out` when given
        (contiguous, the field's dtype and length), e.g. a pinned_empty array."""
        dtype = np.int32 if field in INT_FIELDS else np.float64
        if out is None:
            a = np.empty(self.n[replica], dtype=dtype)
        else:
            a = out
            if a.dtype != dtype or a.shape != (self.n[replica],) or not a.flags.c_contiguous or not a.flags.writeable:
                raise ValueError(f"{field}: out must be a writeable contiguous {dtype} array of {self.n[replica]}")
        self._check(self.lib.sg_download(self.h, replica, field.encode(), a.ctypes.data_as(C.c_void_p)))
        return a

    def define_group(self, group: int, member, replica: int = 0) -> None:
        """Group `group` (1..7) of a replica: the particles with member[id] != 0."""
        m = np.ascontiguousarray(member, dtype=np.uint8)
        if m.shape != (self.n[replica],):
            raise ValueError("one membership flag per particle expected")
        self._check(self.lib.sg_define_group(self.h, replica, int(group), m.ctypes.data_as(C.c_void_p)))

    def set_integrator_group(self, index: int, group: int) -> None:
        """The integrator at map position `index` moves only group `group` (0 = all)."""
        self._check(self.lib.sg_set_integrator_group(self.h, int(index), int(group)))

    def coordination(self, replica: int = 0) -> np.ndarray:
        """Contacts per particle at the last list build (Particle::coordination)."""
        out = np.empty(self.n[replica], np.int32)
        self._check(self.lib.sg_coordination(self.h, replica, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    def set_nlist(self, rcut, pad):
        self._check(self.lib.sg_set_nlist(self.h, float(rcut), float(pad)))

    def build_nlist(self):
        self._check(self.lib.sg_build_nlist(self.h))

    def pairs(self, replica: int = 0):
        n = C.c_int64()
        self.lib.sg_get_pairs(self.h, replica, None, None, 0, C.byref(n))
        cap = max(1, n.value)
        i = np.empty(cap, np.int32)
        j = np.empty(cap, np.int32)
        self._check(self.lib.sg_get_pairs(self.h, replica, i.ctypes.data_as(C.POINTER(C.c_int32)),
                                          j.ctypes.data_as(C.POINTER(C.c_int32)), cap, C.byref(n)))
        return i[:n.value], j[:n.value]

    def add_pair(self, kind, global_params, table=None, use_radii=False, phase_in=False,
                 shifted=False, has_pair_params=False, phase_value=None):
        g = np.zeros(PAIR_NPARAM)
        g[:len(global_params)] = global_params
        t, pv = _arr(table), _arr(phase_value)
        self._check(self.lib.sg_add_pair(self.h, int(kind), _dptr(g), _dptr(t), int(use_radii),
                                         int(phase_in), int(shifted), int(has_pair_params), _dptr(pv)))

    def add_align(self, kind, J, rcut, table=None, has_pair_params=False):
        t = _arr(table)
        self._check(self.lib.sg_add_align(self.h, int(kind), float(J), float(rcut), _dptr(t),
                                          int(has_pair_params)))

    def add_external(self, kind, alpha, type_alpha=None, has_params=False):
        t = _arr(type_alpha)
        self._check(self.lib.sg_add_external(self.h, int(kind), float(alpha), _dptr(t), int(has_params)))

    def add_constraint(self, kind, params):
        p = np.zeros(9)
        p[:len(params)] = params
        self._check(self.lib.sg_add_constraint(self.h, int(kind), _dptr(p)))

    def add_constraint_per_replica(self, kind, params, value0):
        p = np.zeros(9)
        p[:len(params)] = params
        v = np.ascontiguousarray(value0, dtype=np.float64)
        if v.shape != (len(self.n),):
            raise ValueError("one value per replica expected")
        self._check(self.lib.sg_add_constraint_per_replica(self.h, int(kind), _dptr(p), _dptr(v)))

    def add_integrator(self, kind, params, temperature=None):
        p = np.zeros(INT_NPARAM)
        p[:len(params)] = params
        t = _arr(temperature)
        self._check(self.lib.sg_add_integrator(self.h, int(kind), _dptr(p), _dptr(t)))

    def insert_integrator(self, pos, kind, params, temperature=None):
        p = np.zeros(INT_NPARAM)
        p[:len(params)] = params
        t = _arr(temperature)
        self._check(self.lib.sg_insert_integrator(self.h, int(pos), int(kind), _dptr(p), _dptr(t)))

    def disable_integrator(self, index):
        self._check(self.lib.sg_disable_integrator(self.h, int(index)))

    def clear_forces(self):
        self._check(self.lib.sg_clear_forces(self.h))

    def run_continue(self, steps: int) -> "RunStats":
        st = RunStats()
        self._check(self.lib.sg_run_continue(self.h, int(steps), C.byref(st)))
        return st

    def begin_step(self):
        self._check(self.lib.sg_begin_step(self.h))

    def set_replica_param(self, replica, cls, comp, slot, value):
        self._check(self.lib.sg_set_replica_param(self.h, replica, cls, comp, slot, float(value)))

    # -- execution ---------------------------------------------------------
    def compute(self, dt):
        self._check(self.lib.sg_compute(self.h, float(dt)))

    def enforce(self):
        self._check(self.lib.sg_enforce(self.h))

    def run(self, steps: int) -> RunStats:
        st = RunStats()
        self._check(self.lib.sg_run(self.h, int(steps), C.byref(st)))
        return st

    def minimize(self, max_steps: int):
        st = RunStats()
        conv = np.full(len(self.n), -1, np.int64)
        self._check(self.lib.sg_minimize(self.h, int(max_steps),
                                         conv.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(st)))
        return conv, st

    def energy(self, cls: int, comp: int, replica: int = 0) -> float:
        out = C.c_double()
        self._check(self.lib.sg_energy(self.h, replica, cls, comp, C.byref(out)))
        return out.value

    def fire_state(self, replica: int = 0):
        out = np.zeros(5)
        self._check(self.lib.sg_fire_state(self.h, replica, _dptr(out)))
        return out

    def set_profiling(self, on: bool) -> None:
        self._check(self.lib.sg_set_profiling(self.h, int(bool(on))))

    def set_generic_path(self, on: bool) -> None:
        """Force the generic structure-of-arrays kernels (for comparisons)."""
        self._check(self.lib.sg_set_path(self.h, int(bool(on))))

    def set_path(self, path: int) -> None:
        """0 automatic, 1 generic SoA kernels, 2 packed kernels unspecialised."""
        self._check(self.lib.sg_set_path(self.h, int(path)))

    def view(self) -> View:
        """Device pointers into the current state and neighbour lists (see sg_view)."""
        v = View()
        self._check(self.lib.sg_get_view(self.h, C.byref(v)))
        return v

    def replica_slots(self, replica: int):
        off, n = C.c_int32(), C.c_int32()
        self._check(self.lib.sg_replica_slots(self.h, replica, C.byref(off), C.byref(n)))
        return off.value, n.value

    def positions_changed(self) -> None:
        self._check(self.lib.sg_positions_changed(self.h))

    def set_variant(self, v: int) -> None:
        """Pin a step-kernel variant (0..31) or re-enable autotuning (-1)."""
        self._check(self.lib.sg_set_variant(self.h, int(v)))

    def set_generic_occupancy(self, blocks_per_sm: int) -> None:
        """Generic fused kernel: 6 or 8 blocks per SM, or 0 to time both and keep the faster."""
        self._check(self.lib.sg_set_generic_occupancy(self.h, int(blocks_per_sm)))

    def generic_occupancy(self) -> int:
        return int(self.lib.sg_get_generic_occupancy(self.h))

    def set_fire_order(self, ordered: bool) -> None:
        """FIRE's sums in the reference's particle order (True) or a fixed tree (False)."""
        self._check(self.lib.sg_set_fire_order(self.h, int(bool(ordered))))

    def set_build(self, mode: int) -> None:
        """Neighbour-list build kernel: 0 automatic, 1 one thread per particle, 2 teams,
        3 cell tiles staged in shared memory (quasi-2-D replicas on the cell path)."""
        self._check(self.lib.sg_set_build(self.h, int(mode)))

    def variant(self) -> int:
        return int(self.lib.sg_get_variant(self.h))

    def kernel_launches(self) -> int:
        return int(self.lib.sg_kernel_launches(self.h))
