"""The engine's failure paths, made on the host: the reference stops with
Messenger::ERROR and an exception (src/samos.cpp:200,253); the engine returns
a status code through the C ABI and leaves the handle usable.

* a non-finite position (NaN uploaded into one particle): the step kernels
  flag it in the device status word and sg_run returns SG_ERR_NONFINITE; a
  clean upload and a list rebuild make the handle run again (the packed ABP
  path and the generic fused path);
* a clump with more neighbours than the list build stages (more than 48
  lower-id neighbours within rcut + pad): the rebuild returns
  SG_ERR_OVERFLOW, and a spread-out configuration builds and runs again.

Neither case faults the device: the cell index of a NaN position is clamped
into the grid, and the list build never writes past its staging arrays or
the list's capacity; it counts and reports instead.
"""
import numpy as np
import pytest

from samos_b200 import Engine, EngineError
from scenarios import drive, plane_disks

pytestmark = pytest.mark.gpu

STATE = ("x", "y", "z", "nx", "ny", "nz", "vx", "vy", "vz")


def program(b, parts, L, aligner):
    return drive(b, parts, (L, L, 10.0), nlist=(2.4, 0.3), pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
                 aligns=[aligner], dt=1e-3, integrators=[("brownian", {"v0": "0.5", "nu": "0.1", "seed": "3"})])


@pytest.mark.parametrize("aligner", [("polar", {"J": "0.1"}), ("vicsek", {"rcut": "2.0"})])
def test_nonfinite_position_is_reported_and_the_handle_recovers(aligner):
    n = 3000
    parts, L = plane_disks(n, 0.6, seed=61)
    e = Engine(n)
    sim = program(e, parts, L, aligner)
    sim.run(20)
    good = {f: e.download(f) for f in STATE}
    bad_x = good["x"].copy()
    bad_x[1234] = np.nan
    e.upload("x", bad_x)
    with pytest.raises(EngineError) as err:
        sim.run(10)
    assert err.value.code == -6  # SG_ERR_NONFINITE
    for f in STATE:
        e.upload(f, good[f])
    e.positions_changed()
    st = sim.run(30)
    assert st.steps_done == 31
    for f in STATE:
        assert np.isfinite(e.download(f)).all(), f


def test_neighbour_overflow_is_reported_and_the_handle_recovers():
    n = 3000
    parts, L = plane_disks(n, 0.5, seed=62)
    e = Engine(n)
    sim = program(e, parts, L, ("polar", {"J": "0.1"}))
    sim.run(5)
    good = {f: e.download(f) for f in STATE}
    clump_x, clump_y = good["x"].copy(), good["y"].copy()
    rng = np.random.default_rng(62)
    ang, rad = rng.uniform(0, 2 * np.pi, 120), np.sqrt(rng.uniform(0, 1, 120))
    clump_x[:120], clump_y[:120] = rad * np.cos(ang), rad * np.sin(ang)  # 120 particles within radius 1
    e.upload("x", clump_x)
    e.upload("y", clump_y)
    with pytest.raises(EngineError) as err:
        e.positions_changed()  # the list rebuild
    assert err.value.code == -5  # SG_ERR_OVERFLOW
    for f in STATE:
        e.upload(f, good[f])
    e.positions_changed()
    st = sim.run(20)
    assert st.steps_done == 21
    assert np.isfinite(e.download("x")).all()
