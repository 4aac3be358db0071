"""The allocation-free entry point sg_compute_static, through the C ABI.

Some callers cannot call cudaMalloc (code living inside another framework's
memory pool or under a no-allocation policy, plugins handed device pointers by
their host application).  For them sg_compute_static evaluates the soft
pair forces and polar/nematic torques from caller-owned device arrays, keeping
its cell lists in one fixed device array compiled into the library.  This
file checks it against the engine's own evaluation (sg_compute) on two
different systems called one after the other -- so a second call cannot lean
on what the first left in the shared scratch -- bit for bit, the tolerance
the other force tests use, and on the other paths the call takes: a box too
small for the cell path (the N^2 list), a box without periodic wrap, the
fixed contact distance `a` without an aligner, and a clump with more
neighbours than the call stages (NaN outputs, counted by
sg_compute_static_overflow).  It is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from samos_b200 import Engine, engine as E
from scenarios import drive, plane_disks

pytestmark = pytest.mark.gpu

IN_FIELDS = ("x", "y", "z", "nx", "ny", "nz", "radius")
OUT_FIELDS = ("fx", "fy", "fz", "tau_x", "tau_y", "tau_z")


def engine_forces(parts, box, nlist, k, aligner, J, periodic=True, radii=True, a=2.0, backend=Engine):
    n = len(parts["x"])
    e = backend(n)
    soft = {"k": repr(k), "use_particle_radii": ""} if radii else {"k": repr(k), "a": repr(a)}
    sim = drive(e, parts, box, periodic=periodic, nlist=nlist, constraint=None, pairs=[("soft", soft)],
                aligns=[(aligner, {"J": repr(J)})] if aligner else [])
    sim.commit()
    e.compute(1e-3)
    out = {f: e.download(f) for f in OUT_FIELDS}
    e.close()
    return out


def static_forces(lib, parts, box, nlist, k, align_kind, J, periodic=True, radii=True, a=2.0):
    import torch
    dev = torch.device("cuda:0")
    n = len(parts["x"])
    ins = {f: torch.tensor(np.ascontiguousarray(parts[f]), dtype=torch.float64, device=dev) for f in IN_FIELDS}
    outs = {f: torch.full((n,), float("nan"), dtype=torch.float64, device=dev) for f in OUT_FIELDS}
    torch.cuda.synchronize()
    ptr = lambda t: C.c_void_p(t.data_ptr())
    rc = lib.sg_compute_static(n, box[0], box[1], box[2], int(periodic), nlist[0], nlist[1],
                               *[ptr(ins[f]) for f in IN_FIELDS], k, a, int(radii), align_kind, J, nlist[0],
                               *[ptr(outs[f]) for f in OUT_FIELDS], None)
    torch.cuda.synchronize()
    assert rc == 0, lib.sg_error_string(rc)
    return {f: outs[f].cpu().numpy() for f in OUT_FIELDS}


def test_static_entry_point_matches_engine_on_two_calls_in_a_row():
    lib = E.load()
    assert 0 < lib.sg_compute_static_scratch_bytes() <= 8 << 20
    cases = [
        (plane_disks(20000, 0.8, seed=31, bidisperse=(1.0, 1.4)), (2.8, 0.3), 10.0, "nematic", E.ALIGN["nematic"], 0.5),
        (plane_disks(6000, 0.6, seed=32), (2.4, 0.3), 7.0, "polar", E.ALIGN["polar"], 0.2),
    ]
    for (parts, L), nlist, k, aname, akind, J in cases:
        box = (L, L, 10.0)
        want = engine_forces(parts, box, nlist, k, aname, J)
        got = static_forces(lib, parts, box, nlist, k, akind, J)
        for f in OUT_FIELDS:
            assert np.isfinite(got[f]).all(), f
            np.testing.assert_array_equal(got[f], want[f], err_msg=f"{f} ({aname})")


def overflow_count(lib):
    c = C.c_int(-1)
    assert lib.sg_compute_static_overflow(C.byref(c), None) == 0
    return c.value


def test_static_entry_point_on_its_other_paths():
    from oracle.oracle import OracleSystem
    lib = E.load()
    rng = np.random.default_rng(33)
    # (1) N^2 list: one side shorter than 2 (rcut + pad); (2) no periodic
    # wrap; (3) fixed contact distance a, no aligner
    n1 = 300
    th = rng.uniform(0, 2 * np.pi, n1)
    small = dict(x=rng.uniform(-2.6, 2.6, n1), y=rng.uniform(-60.0, 60.0, n1), z=np.zeros(n1), nx=np.cos(th),
                 ny=np.sin(th), nz=np.zeros(n1), radius=rng.uniform(0.9, 1.1, n1))
    parts2, L2 = plane_disks(3000, 0.6, seed=34)
    parts2["x"] *= 0.98  # strictly inside the box: nothing to wrap
    parts2["y"] *= 0.98
    parts3, L3 = plane_disks(4000, 0.5, seed=35)
    cases = [
        ("nsq", small, (5.4, 120.0, 10.0), dict(periodic=True, radii=True), "polar", E.ALIGN["polar"], 0.3),
        ("fixed_box", parts2, (L2, L2, 10.0), dict(periodic=False, radii=True), "nematic", E.ALIGN["nematic"], 0.4),
        ("no_aligner", parts3, (L3, L3, 10.0), dict(periodic=True, radii=False, a=2.2), None, -1, 0.0),
    ]
    for name, parts, box, kw, aname, akind, J in cases:
        want = engine_forces(parts, box, (2.4, 0.3), 10.0, aname, J, **kw)
        oracle = engine_forces(parts, box, (2.4, 0.3), 10.0, aname, J, backend=OracleSystem, **kw)
        got = static_forces(lib, parts, box, (2.4, 0.3), 10.0, akind, J, **kw)
        assert overflow_count(lib) == 0
        for f in OUT_FIELDS:
            np.testing.assert_array_equal(got[f], want[f], err_msg=f"{f} ({name})")
            np.testing.assert_array_equal(got[f], oracle[f], err_msg=f"{f} ({name}, oracle)")


def test_static_entry_point_flags_a_clump_it_cannot_stage():
    # 150 particles inside a disk of radius 1 among sparse ones: each of them
    # has more than 64 neighbours on one side of its id within rcut + pad
    lib = E.load()
    parts, L = plane_disks(2000, 0.3, seed=36)
    rng = np.random.default_rng(36)
    ang, rad = rng.uniform(0, 2 * np.pi, 150), np.sqrt(rng.uniform(0, 1, 150))
    parts["x"][:150], parts["y"][:150] = rad * np.cos(ang), rad * np.sin(ang)
    got = static_forces(lib, parts, (L, L, 10.0), (2.4, 0.3), 10.0, E.ALIGN["polar"], 0.1)
    bad = ~np.isfinite(got["fx"])
    assert bad.sum() > 0 and bad[150:].sum() <= bad.sum()
    assert overflow_count(lib) == int(bad.sum())
    # the next call starts its count afresh
    parts2, L2 = plane_disks(1000, 0.5, seed=37)
    static_forces(lib, parts2, (L2, L2, 10.0), (2.4, 0.3), 10.0, E.ALIGN["polar"], 0.1)
    assert overflow_count(lib) == 0


def test_static_entry_point_rejects_sizes_beyond_its_scratch():
    lib = E.load()
    null = C.c_void_p(0)
    too_many = 65536 + 1
    rc = lib.sg_compute_static(too_many, 100.0, 100.0, 10.0, 1, 2.4, 0.3, *([null] * 7), 10.0, 2.0, 1, 0, 0.1,
                               2.4, *([null] * 6), None)
    assert rc == -1  # SG_ERR_ARG, nothing launched
    # a box whose cell grid exceeds the scratch's cell capacity
    rc = lib.sg_compute_static(10, 5000.0, 5000.0, 10.0, 1, 2.4, 0.3, *([null] * 7), 10.0, 2.0, 1, 0, 0.1,
                               2.4, *([null] * 6), None)
    assert rc == -1
    # a side so long that its cell count does not fit an int, and a NaN side
    for lx in (1e300, float("nan"), float("inf")):
        rc = lib.sg_compute_static(10, lx, 100.0, 10.0, 1, 2.4, 0.3, *([null] * 7), 10.0, 2.0, 1, 0, 0.1,
                                   2.4, *([null] * 6), None)
        assert rc == -1
