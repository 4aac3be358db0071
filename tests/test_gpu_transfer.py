"""Host transfers through the C ABI: page-locked arrays (sg_host_alloc) and
ordinary numpy arrays give the same values, in particle-id order, after the
particle arrays have been re-sorted into cell order by list rebuilds."""
import numpy as np
import pytest

from samos_b200 import Engine
from samos_b200.engine import pinned_copy, pinned_empty
from scenarios import drive, plane_disks

pytestmark = pytest.mark.gpu


def test_pinned_and_pageable_transfers_agree():
    n = 3000
    parts, L = plane_disks(n, 0.6, seed=5)
    e = Engine(n)
    sim = drive(e, parts, (L, L, 10.0), nlist=(2.4, 0.3), pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
                integrators=[("brownian", {"v0": "0.5", "nu": "0.1", "mu": "1", "mur": "1", "seed": "4"})])
    sim.run(200)  # several rebuilds: slots are no longer in id order
    for f in ("x", "y", "nx", "ny", "vx", "vy", "radius", "fx"):
        plain = e.download(f)
        pinned = pinned_empty(n)
        got = e.download(f, out=pinned)
        assert got is pinned
        np.testing.assert_array_equal(plain, pinned)
    # upload from page-locked memory, read back through both paths
    rng = np.random.default_rng(1)
    x_new = e.download("x") + rng.uniform(-0.01, 0.01, n)
    e.upload("x", pinned_copy(x_new))
    np.testing.assert_array_equal(e.download("x"), x_new)
    out = pinned_empty(n)
    np.testing.assert_array_equal(e.download("x", out=out), x_new)
    ix = pinned_empty(n, np.int32)
    np.testing.assert_array_equal(e.download("ix", out=ix), e.download("ix"))
    with pytest.raises(ValueError):
        e.download("x", out=np.empty(n - 1))
    with pytest.raises(ValueError):
        e.download("x", out=np.empty(n, np.float32))


def test_multi_field_transfers_equal_one_field_transfers():
    # sg_upload_fields / sg_download_fields against one call per field, on a
    # run whose slots have been re-sorted by rebuilds, ints and the host-side
    # surface normals included
    n = 3000
    parts, L = plane_disks(n, 0.6, seed=6)
    kw = dict(nlist=(2.4, 0.3), pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
              integrators=[("brownian", {"v0": "0.5", "nu": "0.1", "mu": "1", "mur": "1", "seed": "4"})])
    a, b = Engine(n), Engine(n)
    sa, sb = drive(a, parts, (L, L, 10.0), **kw), drive(b, parts, (L, L, 10.0), **kw)
    sa.run(200)
    sb.run(200)
    fields = ("x", "y", "z", "nx", "ny", "vx", "vy", "radius", "age", "ix", "iy", "type", "Nz")
    one = {f: a.download(f) for f in fields}
    many = a.download_fields(fields, out={"x": pinned_empty(n)})
    for f in fields:
        np.testing.assert_array_equal(one[f], many[f], err_msg=f)
    rng = np.random.default_rng(2)
    new = {"x": pinned_copy(one["x"] + rng.uniform(-0.01, 0.01, n)), "y": one["y"] + rng.uniform(-0.01, 0.01, n),
           "ix": one["ix"] + 1, "nx": pinned_copy(one["nx"])}
    for f, v in new.items():
        b.upload(f, v)
    a.upload_fields(new)
    for e in (a, b):
        e.positions_changed()
    sa.run(50)
    sb.run(50)
    for f in ("x", "y", "nx", "ny", "ix", "iy"):
        np.testing.assert_array_equal(a.download(f), b.download(f), err_msg=f)
