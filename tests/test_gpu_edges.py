"""Edge cases of the GPU path against the oracle and the engine's own error
behaviour: systems of one and two particles, a ragged ensemble whose
replicas straddle the 128-slot block boundary (one particle, 127, 128, 129),
neighbour counts that outgrow the list's first capacity (regrowth), and the
errors the reference raises for a run before its components exist."""
import numpy as np
import pytest

from oracle.oracle import OracleSystem
from samos_b200 import Engine, EngineError
from samos_b200.ensemble import SphereReplica, sphere_ensemble
from scenarios import drive, plane_disks, sphere_disks

pytestmark = pytest.mark.gpu

BROWNIAN = [("brownian", {"v0": "0.5", "nu": "0.1", "seed": "3"})]


def both(parts, box, steps, **kw):
    n = len(parts["x"])
    out = []
    for b in (Engine(n), OracleSystem(n)):
        sim = drive(b, parts, box, **kw)
        sim.run(steps)
        out.append(b)
    return out


def same(e, o, fields=("x", "y", "nx", "ny"), tol=1e-12):
    for f in fields:
        err = float(np.max(np.abs(e.download(f) - o.download(f))))
        assert err <= tol, (f, err)


def tiny(xs, ys):
    n = len(xs)
    th = np.linspace(0.3, 2.0, n)
    return dict(x=np.array(xs, float), y=np.array(ys, float), z=np.zeros(n), vx=np.zeros(n), vy=np.zeros(n),
                vz=np.zeros(n), nx=np.cos(th), ny=np.sin(th), nz=np.zeros(n), radius=np.ones(n))


def test_one_particle_has_no_neighbours_and_moves_like_the_oracle():
    e, o = both(tiny([0.3], [-1.2]), (20.0, 20.0, 10.0), 200, pairs=[("soft", {"k": "10"})],
                aligns=[("polar", {"J": "1"})], integrators=BROWNIAN)
    assert len(e.pairs()[0]) == 0
    same(e, o)


def test_two_overlapping_particles_across_the_periodic_edge():
    # the pair straddles x = +-L/2: the minimum image carries the contact
    e, o = both(tiny([9.6, -9.7], [0.0, 0.2]), (20.0, 20.0, 10.0), 100, pairs=[("soft", {"k": "10"})],
                aligns=[("nematic", {"J": "0.5"})], integrators=BROWNIAN)
    i, j = o.pairs()
    assert len(i) == 1
    np.testing.assert_array_equal(e.pairs()[0], i)
    same(e, o, tol=1e-9)


def test_ragged_ensemble_across_block_boundaries():
    sizes = [1, 127, 128, 129, 300]
    rng = np.random.default_rng(50)
    reps = []
    for k, n in enumerate(sizes):
        if n == 1:
            parts = dict(x=np.array([4.0]), y=np.zeros(1), z=np.zeros(1), vx=np.zeros(1), vy=np.zeros(1),
                         vz=np.zeros(1), nx=np.zeros(1), ny=np.ones(1), nz=np.zeros(1), radius=np.ones(1))
            R = 4.0
        else:
            parts, R = sphere_disks(n, seed=60 + k)
        reps.append(SphereReplica(parts=parts, R=R, v0=float(rng.uniform(0.1, 1.0)), J=float(rng.uniform(0, 1)),
                                  nu=0.05, seed=int(rng.integers(1, 10**6))))
    batched = sphere_ensemble(reps)
    batched.run(200)
    for i, r in enumerate(reps):
        single = sphere_ensemble([r])
        single.run(200)
        for f in ("x", "y", "z", "nx", "ny", "nz"):
            np.testing.assert_array_equal(batched.download(f, replica=i), single.download(f), err_msg=f"{i} {f}")
        single.close()


def test_dense_lists_outgrow_their_first_capacity():
    # up to ~40 neighbours within rcut + pad per disk (the list starts with
    # room for 32): the list is regrown and its pairs are still the oracle's,
    # in the oracle's order
    parts, L = plane_disks(1500, 1.0, seed=51, rmin=0.5, rmax=0.6)
    e, o = both(parts, (L, L, 10.0), 20, nlist=(2.4, 0.3), pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
                integrators=BROWNIAN)
    i, j = o.pairs()
    assert np.bincount(np.concatenate([i, j])).max() > 32
    ei, ej = e.pairs()
    np.testing.assert_array_equal(ei, i)
    np.testing.assert_array_equal(ej, j)
    same(e, o, tol=1e-9)


def test_runs_before_their_components_exist_are_refused():
    parts, L = plane_disks(200, 0.5, seed=52)
    e = Engine(200)
    e.set_box(L, L, 10.0, True)
    for f in ("x", "y", "z", "nx", "ny", "nz", "radius"):
        e.upload(f, parts[f])
    with pytest.raises(EngineError):
        e.run(5)  # no constraint (samos.cpp: "Constraint has not been defined")
    with pytest.raises(ValueError):
        e.upload("x", parts["x"][:-1])
    with pytest.raises(EngineError):
        e.upload("type", np.full(200, 3, np.int32))  # types outside 1..ntypes
