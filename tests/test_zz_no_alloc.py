"""The allocation-free entry point sg_compute_static, through the C ABI.

Some callers cannot call cudaMalloc (code living inside another framework's
memory pool or under a no-allocation policy, plugins handed device pointers by
their host application).  For them sg_compute_static evaluates the soft
pair forces and polar/nematic torques from caller-owned device arrays, keeping
its cell lists in one fixed device array compiled into the library.  This
file checks it against the engine's own evaluation (sg_compute) on two
different systems called one after the other -- so a second call cannot lean
on what the first left in the shared scratch -- bit for bit, the tolerance
the other force tests use.  It is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from samos_b200 import Engine, engine as E
from scenarios import drive, plane_disks

pytestmark = pytest.mark.gpu

IN_FIELDS = ("x", "y", "z", "nx", "ny", "nz", "radius")
OUT_FIELDS = ("fx", "fy", "fz", "tau_x", "tau_y", "tau_z")


def engine_forces(parts, box, nlist, k, aligner, J):
    n = len(parts["x"])
    e = Engine(n)
    sim = drive(e, parts, box, nlist=nlist, constraint=None,
                pairs=[("soft", {"k": repr(k), "use_particle_radii": ""})],
                aligns=[(aligner, {"J": repr(J)})])
    sim.commit()
    e.compute(1e-3)
    out = {f: e.download(f) for f in OUT_FIELDS}
    e.close()
    return out


def static_forces(lib, parts, box, nlist, k, align_kind, J):
    import torch
    dev = torch.device("cuda:0")
    n = len(parts["x"])
    ins = {f: torch.tensor(np.ascontiguousarray(parts[f]), dtype=torch.float64, device=dev) for f in IN_FIELDS}
    outs = {f: torch.full((n,), float("nan"), dtype=torch.float64, device=dev) for f in OUT_FIELDS}
    torch.cuda.synchronize()
    ptr = lambda t: C.c_void_p(t.data_ptr())
    rc = lib.sg_compute_static(n, box[0], box[1], box[2], 1, nlist[0], nlist[1],
                               *[ptr(ins[f]) for f in IN_FIELDS], k, 2.0, 1, align_kind, J, nlist[0],
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
