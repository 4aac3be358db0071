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
