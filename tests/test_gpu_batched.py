"""Batched replicas: R independent sphere systems with different sizes,
radii, activities, couplings, noise strengths and seeds in one engine handle
must give exactly the trajectories of the same systems run one at a time
(they share launches, never data), and one of them must match the oracle."""
import numpy as np
import pytest

from oracle.oracle import OracleSystem
from samos_b200 import Engine
from samos_b200.ensemble import SphereReplica, sphere_ensemble
from scenarios import drive, sphere_disks

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "nx", "ny", "nz", "vx", "vy", "vz", "age")


def make_reps(count, seed):
    rng = np.random.default_rng(seed)
    reps = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(300), np.log(4000)))))
        parts, R = sphere_disks(n, seed=100 + i)
        reps.append(SphereReplica(parts=parts, R=R, v0=float(rng.uniform(0.01, 1.0)), J=float(rng.uniform(0, 1)),
                                  nu=float(np.exp(rng.uniform(np.log(1e-3), 0.0))), seed=int(rng.integers(1, 10**6))))
    return reps


def test_batched_equals_serial_bitwise():
    reps = make_reps(7, 1)
    batched = sphere_ensemble(reps)
    batched.run(300)
    for i, r in enumerate(reps):
        single = sphere_ensemble([r])
        single.run(300)
        for f in FIELDS:
            np.testing.assert_array_equal(batched.download(f, replica=i), single.download(f), err_msg=f"rep {i} {f}")
        single.close()


@pytest.mark.parametrize("byval,twin", [(22, 17), (24, 11)])
def test_by_value_variant_pinned_on_an_ensemble_runs_its_twin(byval, twin):
    # a variant that takes one replica's parameters by value cannot serve
    # several replicas: the engine runs its shared-memory twin, same bits
    reps = make_reps(4, 3)
    runs = []
    for v in (byval, twin):
        e = sphere_ensemble(reps)
        e.set_variant(v)
        e.run(150)
        runs.append(e)
    for i in range(len(reps)):
        for f in FIELDS:
            np.testing.assert_array_equal(runs[0].download(f, replica=i), runs[1].download(f, replica=i),
                                          err_msg=f"rep {i} {f}")
    single = sphere_ensemble([reps[2]])
    single.set_variant(byval)
    single.run(150)
    for f in FIELDS:
        np.testing.assert_array_equal(single.download(f), runs[0].download(f, replica=2), err_msg=f)


def test_batched_replica_matches_oracle():
    reps = make_reps(3, 2)
    batched = sphere_ensemble(reps)
    batched.run(200)
    r = reps[1]
    n = len(r.parts["x"])
    o = OracleSystem(n)
    side = 2 * r.R + 6.0
    sim = drive(o, r.parts, (side, side, side), periodic=False, nlist=(2.4, 0.3),
                constraint=("sphere", {"r": repr(r.R)}),
                pairs=[("soft", {"k": "10.0", "use_particle_radii": ""})], aligns=[("polar", {"J": repr(r.J)})],
                dt=1e-3, integrators=[("brownian", {"v0": repr(r.v0), "nu": repr(r.nu), "seed": str(r.seed)})])
    sim.run(200)
    for f in ("x", "y", "z", "nx", "ny", "nz"):
        err = np.max(np.abs(batched.download(f, replica=1) - o.download(f)))
        assert err <= 1e-9, (f, err)


def test_batched_fire_matches_one_at_a_time():
    # replicas converge at different iterations; the minimiser then launches
    # only the blocks of the replicas still running: results must be those of
    # each replica minimised alone
    from samos_b200.ensemble import plane_fire_ensemble, quench_disks
    insts = [quench_disks(n, phi, seed) for n, phi, seed in ((300, 0.85, 1), (520, 0.88, 2), (800, 0.86, 3),
                                                            (256, 0.90, 4))]
    eng = plane_fire_ensemble(insts, fmax=1e-10)
    eng.build_nlist()
    conv, _ = eng.minimize(400000)
    assert (conv > 0).all() and len(set(conv.tolist())) > 1
    for r, inst in enumerate(insts):
        one = plane_fire_ensemble([inst], fmax=1e-10)
        one.build_nlist()
        c1, _ = one.minimize(400000)
        assert c1[0] == conv[r]
        for f in ("x", "y", "vx", "vy"):
            np.testing.assert_array_equal(one.download(f), eng.download(f, replica=r), err_msg=f"{f} replica {r}")
        one.close()
    eng.close()
