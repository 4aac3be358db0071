"""GPU parity: the CUDA path through the C ABI against the CPU oracle on the
same seeded inputs.

Bars (FP64): neighbour pair lists identical (same pairs, same order); forces,
torques of soft / polar / nematic / vicsek / self-propulsion identical bit for
bit (same operation order, no FMA); exp-based potentials (LJ uses none, but
Morse and Gaussian do) within 1e-12 relative; energies within 1e-12 relative;
trajectories within 1e-9 after 1000 steps with the shared noise stream.
"""
import numpy as np
import pytest

from oracle.oracle import OracleSystem
from samos_b200 import Engine
from scenarios import drive, plane_disks, sphere_disks, surface_disks, tetra_value

pytestmark = pytest.mark.gpu

REL = 1e-12      # per-step forces / torques / energies
TRAJ = 1e-9      # positions after 1000 steps


def pair_lists(parts, box, periodic=True, nlist=(2.4, 0.3), constraint=("plane", {})):
    n = len(parts["x"])
    e, o = Engine(n), OracleSystem(n)
    for b in (e, o):
        drive(b, parts, box, periodic=periodic, nlist=nlist, constraint=constraint)
    return e.pairs(), o.pairs(), o


def test_pairs_cell_path_identical():
    parts, L = plane_disks(2000, 0.6, seed=1)
    (ei, ej), (oi, oj), o = pair_lists(parts, (L, L, 10.0))
    assert o.uses_cells()
    assert len(oi) > 4000
    np.testing.assert_array_equal(ei, oi)
    np.testing.assert_array_equal(ej, oj)


def test_pairs_nsq_path_identical():
    parts, L = plane_disks(500, 0.6, seed=2)
    (ei, ej), (oi, oj), o = pair_lists(parts, (L, L, 4.0))
    assert not o.uses_cells()
    np.testing.assert_array_equal(ei, oi)
    np.testing.assert_array_equal(ej, oj)


def test_pairs_two_cell_dimension_duplicates_like_reference():
    # lz = 6 > 2 (rcut+pad) = 5.4 gives nz = 2: the reference's stencil
    # visits that layer twice and lists such pairs twice
    parts, L = plane_disks(800, 0.6, seed=3)
    (ei, ej), (oi, oj), o = pair_lists(parts, (L, L, 6.0))
    assert o.uses_cells()
    np.testing.assert_array_equal(ei, oi)
    np.testing.assert_array_equal(ej, oj)


def test_pairs_sphere_identical():
    parts, R = sphere_disks(3000, seed=4)
    box = 2 * R + 6.0
    (ei, ej), (oi, oj), _ = pair_lists(parts, (box, box, box), periodic=False,
                                       constraint=("sphere", {"r": repr(R)}))
    np.testing.assert_array_equal(ei, oi)
    np.testing.assert_array_equal(ej, oj)


def full_lists(e):
    """Every slot's whole neighbour list (lower-id part, then upper part) in
    particle ids, keyed by the particle id, read through the device view."""
    v = e.view()
    n = v.slots
    cnt = np.empty(n, np.int32)
    ids = np.empty(n, np.int32)
    e._check(e.lib.sg_memcpy(cnt.ctypes.data, v.nb_cnt, cnt.nbytes))
    e._check(e.lib.sg_memcpy(ids.ctypes.data, v.id, ids.nbytes))
    rows = int(cnt.max())
    nb = np.empty((rows, v.nb_stride), np.int32)
    for q in range(rows):
        e._check(e.lib.sg_memcpy(nb[q].ctypes.data, v.nb + 4 * q * v.nb_stride, 4 * v.nb_stride))
    out = {}
    for k in range(n):
        out[int(ids[k])] = [int(ids[nb[q, k]]) for q in range(cnt[k])]
    return out


def clustered_disks(per=24, grid=12, spacing=4.0, seed=9):
    """Tight clumps of `per` disks on a square grid: every disk has all its
    clump in its own cell, more finds than one lane of a team build stages."""
    rng = np.random.default_rng(seed)
    cx, cy = np.meshgrid(np.arange(grid) * spacing, np.arange(grid) * spacing)
    L = grid * spacing
    c = np.stack([cx.ravel(), cy.ravel()], 1) - L / 2 + spacing / 2
    a = rng.uniform(0.0, 2.0 * np.pi, (len(c), per))
    rr = 0.4 * np.sqrt(rng.uniform(0.0, 1.0, (len(c), per)))
    x = (c[:, 0:1] + rr * np.cos(a)).ravel()
    y = (c[:, 1:2] + rr * np.sin(a)).ravel()
    n = len(x)
    order = rng.permutation(n)
    th = rng.uniform(0.0, 2.0 * np.pi, n)
    parts = dict(x=x[order], y=y[order], z=np.zeros(n), vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n),
                 nx=np.cos(th), ny=np.sin(th), nz=np.zeros(n), radius=np.full(n, 0.1))
    return parts, L


BUILD_CASES = {
    "plane_cells": lambda: (plane_disks(2000, 0.6, seed=1), 10.0, True, ("plane", {})),
    "plane_two_cell_z": lambda: (plane_disks(800, 0.6, seed=3), 6.0, True, ("plane", {})),
    "plane_nsq": lambda: (plane_disks(500, 0.6, seed=2), 4.0, True, ("plane", {})),
    "plane_clumps": lambda: (clustered_disks(), 10.0, True, ("plane", {})),
}


@pytest.mark.parametrize("case", list(BUILD_CASES) + ["sphere"])
def test_team_and_thread_list_builds_identical(case):
    if case == "sphere":
        parts, R = sphere_disks(3000, seed=4)
        box, periodic, cons = (2 * R + 6.0,) * 3, False, ("sphere", {"r": repr(R)})
    else:
        (parts, L), lz, periodic, cons = BUILD_CASES[case]()
        box = (L, L, lz)
    n = len(parts["x"])
    lists, pairs = [], []
    for mode in (1, 2, 3):  # one thread per particle, teams, cell tiles (where eligible)
        e = Engine(n)
        e.set_build(mode)
        drive(e, parts, box, periodic=periodic, nlist=(2.4, 0.3), constraint=cons)
        lists.append(full_lists(e))
        pairs.append(e.pairs())
    o = OracleSystem(n)
    drive(o, parts, box, periodic=periodic, nlist=(2.4, 0.3), constraint=cons)
    assert lists[0] == lists[1] == lists[2]
    oi, oj = o.pairs()
    for ei, ej in pairs:
        np.testing.assert_array_equal(ei, oi)
        np.testing.assert_array_equal(ej, oj)
    if case == "plane_clumps":  # some disks have more finds on one side than a lane stages (16)
        assert max(max(sum(j < i for j in v), sum(j > i for j in v)) for i, v in lists[0].items()) > 16


def test_tile_build_through_list_only_rebuilds_and_resorts():
    # the cell-tile build (mode 3) against the one-thread build (mode 1) over
    # a run with many rebuilds: list-only rebuilds through the cell-ordered
    # slot index and every 8th one a full re-sort; every field bit for bit
    n = 20000
    parts, L = plane_disks(n, 0.7, seed=71, bidisperse=(1.0, 1.4))
    out = []
    for mode in (1, 3):
        e = Engine(n)
        e.set_build(mode)
        sim = drive(e, parts, (L, L, 10.0), nlist=(2.8, 0.1), pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
                    aligns=[("nematic", {"J": "0.5"})], dt=1e-3,
                    integrators=[("brownian", {"v0": "2.0", "nu": "0.1", "seed": "9"})])
        st = sim.run(299)
        out.append((e, st.nlist_builds))
    (a, ba), (b, bb) = out
    assert ba == bb >= 10
    for f in ("x", "y", "nx", "ny", "vx", "vy", "fx", "fy", "tau_z", "ix", "iy"):
        np.testing.assert_array_equal(a.download(f), b.download(f), err_msg=f)
    assert full_lists(a) == full_lists(b)


def compute_both(parts, box, pairs=(), aligns=(), externals=(), nlist=(2.4, 0.3), periodic=True,
                 constraint=("plane", {}), ntypes=1, pair_params=(), align_params=()):
    n = len(parts["x"])
    out = []
    for b in (Engine(n, ntypes), OracleSystem(n, ntypes)):
        sim = drive(b, parts, box, periodic=periodic, nlist=nlist, constraint=constraint, pairs=pairs,
                    aligns=aligns, externals=externals, ntypes=ntypes, pair_params=pair_params,
                    align_params=align_params)
        sim.commit()
        b.compute(1e-3)
        out.append(b)
    return out


FIELDS = ("fx", "fy", "fz", "tau_x", "tau_y", "tau_z")


@pytest.mark.parametrize("align", ["polar", "nematic", "vicsek"])
def test_soft_plus_aligner_bitexact(align):
    parts, L = plane_disks(2000, 0.8, seed=5, bidisperse=(1.0, 1.4))
    rng = np.random.default_rng(5)
    parts["vx"], parts["vy"] = rng.normal(size=2000), rng.normal(size=2000)
    e, o = compute_both(parts, (L, L, 10.0), nlist=(2.8, 0.3),
                        pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
                        aligns=[(align, {"J": "0.5"})],
                        externals=[("self_propulsion", {"alpha": "0.3"})])
    for f in FIELDS:
        np.testing.assert_array_equal(e.download(f), o.download(f), err_msg=f)
    assert e.energy(0, 0) == pytest.approx(o.energy(0, 0), rel=REL)
    if align != "vicsek":
        assert e.energy(1, 0) == pytest.approx(o.energy(1, 0), rel=REL)


@pytest.mark.parametrize("name,params", [
    ("lj", {"epsilon": "1", "sigma": "1", "rcut": "2.5", "use_particle_radii": "", "shifted": ""}),
    ("morse", {"D": "1", "a": "2", "re": "2", "rcut": "2.5", "shifted": ""}),
    ("gaussian", {"A": "2", "B": "-1", "alpha": "1", "beta": "3", "rA": "0", "rB": "1.5", "rcut": "2.5"}),
])
def test_other_pair_potentials(name, params):
    parts, L = plane_disks(1500, 0.4, seed=6)
    e, o = compute_both(parts, (L, L, 10.0), nlist=(2.5, 0.3), pairs=[(name, params)])
    for f in ("fx", "fy"):
        a, b = e.download(f), o.download(f)
        scale = np.max(np.abs(b))
        assert np.max(np.abs(a - b)) <= REL * scale, f
    assert e.energy(0, 0) == pytest.approx(o.energy(0, 0), rel=REL)


def test_type_tables_and_pair_params():
    parts, L = plane_disks(1500, 0.7, seed=7)
    rng = np.random.default_rng(7)
    parts["type"] = rng.integers(1, 3, 1500).astype(np.int32)
    e, o = compute_both(parts, (L, L, 10.0), ntypes=2,
                        pairs=[("soft", {"k": "10", "a": "2.0"})],
                        pair_params=[("soft", {"type_1": "1", "type_2": "2", "k": "3", "a": "1.8"})],
                        aligns=[("polar", {"J": "0.2"})],
                        align_params=[("polar", {"type_1": "2", "type_2": "2", "J": "1.5", "rcut": "2.0"})])
    for f in FIELDS:
        np.testing.assert_array_equal(e.download(f), o.download(f), err_msg=f)


def test_sphere_forces_bitexact():
    parts, R = sphere_disks(3000, seed=8)
    box = 2 * R + 6.0
    e, o = compute_both(parts, (box, box, box), periodic=False, constraint=("sphere", {"r": repr(R)}),
                        pairs=[("soft", {"k": "10", "use_particle_radii": ""})], aligns=[("polar", {"J": "0.2"})])
    for f in FIELDS:
        np.testing.assert_array_equal(e.download(f), o.download(f), err_msg=f)


def run_both(n, parts, box, steps, **kw):
    out = []
    for b in (Engine(n, kw.get("ntypes", 1)), OracleSystem(n, kw.get("ntypes", 1))):
        sim = drive(b, parts, box, **kw)
        sim.run(steps)
        out.append(b)
    return out


def assert_traj(e, o, fields=("x", "y", "z", "nx", "ny", "nz"), tol=TRAJ):
    for f in fields:
        a, b = e.download(f), o.download(f)
        err = np.max(np.abs(a - b))
        assert err <= tol, f"{f}: max |gpu - oracle| = {err}"


def test_trajectory_brownian_plane_1000_steps():
    n = 2000
    parts, L = plane_disks(n, 0.6, seed=1)
    e, o = run_both(n, parts, (L, L, 10.0), 999, nlist=(2.4, 0.3),
                    pairs=[("soft", {"k": "10", "use_particle_radii": ""})], aligns=[("polar", {"J": "0.1"})],
                    dt=1e-3, integrators=[("brownian", {"v0": "0.5", "nu": "0.1", "mu": "1", "mur": "1",
                                                         "seed": "1"})])
    assert_traj(e, o)
    np.testing.assert_array_equal(e.download("ix"), o.download("ix"))
    np.testing.assert_array_equal(e.download("iy"), o.download("iy"))
    assert e.download("age") == pytest.approx(o.download("age"), rel=1e-15)


def test_trajectory_brownian_sphere_1000_steps():
    n = 3000
    parts, R = sphere_disks(n, seed=2)
    box = 2 * R + 6.0
    e, o = run_both(n, parts, (box, box, box), 999, periodic=False, nlist=(2.4, 0.3),
                    constraint=("sphere", {"r": repr(R)}),
                    pairs=[("soft", {"k": "10", "use_particle_radii": ""})], aligns=[("polar", {"J": "0.2"})],
                    dt=1e-3, integrators=[("brownian", {"v0": "1.0", "nu": "0.05", "seed": "2"})])
    assert_traj(e, o)


def test_trajectory_pos_align_selfprop_temperature():
    n = 1500
    parts, L = plane_disks(n, 0.6, seed=3)
    e, o = run_both(n, parts, (L, L, 10.0), 499, nlist=(2.4, 0.3),
                    pairs=[("soft", {"k": "10", "use_particle_radii": ""})], aligns=[("nematic", {"J": "0.5"})],
                    externals=[("self_propulsion", {"alpha": "0.5"})], dt=1e-3,
                    integrators=[("brownian_pos", {"mu": "1", "seed": "4", "min_val": "0.01"}),
                                 ("brownian_align", {"nu": "0.1", "mur": "1", "seed": "5", "nematic": "",
                                                     "tau": "0.5"})])
    assert_traj(e, o)


@pytest.mark.parametrize("method", ["baoab", "spv", "bbk"])
def test_trajectory_langevin(method):
    n = 1000
    parts, L = plane_disks(n, 0.5, seed=9)
    e, o = run_both(n, parts, (L, L, 10.0), 299, nlist=(2.5, 0.3),
                    pairs=[("lj", {"epsilon": "1", "sigma": "1", "rcut": "2.5", "shifted": ""})], dt=1e-3,
                    integrators=[("langevin", {"gamma": "1", "seed": "7", "method": method, "min_val": "0.5"})])
    assert_traj(e, o, ("x", "y", "vx", "vy"))


@pytest.mark.parametrize("limits", [{"limit": "0.0001"}, {}, {"limit": "0.001", "angle_limit": "0.0005"}])
def test_trajectory_nve(limits):
    # the relaxation stage of the example configurations: nve with a
    # displacement limit over overlapping soft disks with a polar aligner
    n = 1000
    parts, L = plane_disks(n, 0.6, seed=10)
    e, o = run_both(n, parts, (L, L, 10.0), 299, nlist=(2.4, 0.3),
                    pairs=[("soft", {"k": "1.0"})], aligns=[("polar", {"J": "1.0"})], dt=1e-3,
                    integrators=[("nve", dict(limits))])
    assert_traj(e, o, ("x", "y", "vx", "vy", "nx", "ny", "omega"))


@pytest.mark.parametrize("integ", [
    ("langevin", {"gamma": "1", "seed": "7", "method": "baoab", "min_val": "0.5"}),
    ("langevin", {"gamma": "1", "seed": "7", "method": "bbk", "min_val": "0.5"}),
    ("nve", {"limit": "0.0001"}),
])
def test_reused_start_of_step_forces_are_the_recomputed_ones(integ):
    # within a run, Langevin (BAOAB, BBK) and NVE on a periodic plane take the
    # start-of-step forces from the previous step's own force pass; every run
    # starts by recomputing them, so 120 one-step runs recompute every time:
    # both must give the same bits
    n = 1000
    parts, L = plane_disks(n, 0.6, seed=12)
    kw = dict(nlist=(2.5, 0.3), pairs=[("soft", {"k": "1.0"})], aligns=[("polar", {"J": "1.0"})], dt=1e-3,
              integrators=[integ])
    a, b = Engine(n), Engine(n)
    sa, sb = drive(a, parts, (L, L, 10.0), **kw), drive(b, parts, (L, L, 10.0), **kw)
    sa.run(119)
    for _ in range(120):
        sb.run(0)
    for f in ("x", "y", "vx", "vy", "nx", "ny", "omega", "fx", "fy"):
        np.testing.assert_array_equal(a.download(f), b.download(f), err_msg=f)


def test_fire_matches_oracle():
    n = 600
    parts, L = plane_disks(n, 0.86, seed=11, bidisperse=(1.0, 1.4))
    out = []
    for b in (Engine(n), OracleSystem(n)):
        sim = drive(b, parts, (L, L, 10.0), nlist=(2.8, 0.3), pairs=[("soft", {"k": "1", "use_particle_radii": ""})],
                    dt=0.01, integrators=[("fire", {"dt_max": "0.1", "fmax_tolerance": "1e-10"})])
        sim.commit()
        steps, _ = b.minimize(200000)
        out.append((b, int(steps[0])))
    (e, se), (o, so) = out
    assert se > 0 and so > 0
    # both minimise to Fmax < 1e-10 and land in the same minimum
    for b in (e, o):
        f = np.hypot(b.download("fx"), b.download("fy"))
        assert f.max() < 1e-10
    assert abs(se - so) <= max(5, so // 20)
    assert_traj(e, o, ("x", "y"), tol=1e-7)


@pytest.mark.parametrize("n,phi,seed", [(600, 0.86, 11), (1500, 0.88, 12)])
def test_fire_parity_mode_takes_the_reference_iterations(n, phi, seed):
    # FIRE with its sums P, |F|^2, |v|^2 taken in particle-id order, as the
    # reference loops (integrator_fire.cpp:79-94): the dt / alpha branches
    # and the velocity mixing then see the reference's values, so the
    # quench takes the oracle's iterations exactly and lands on its bits
    parts, L = plane_disks(n, phi, seed=seed, bidisperse=(1.0, 1.4))
    out = []
    for b in (Engine(n), OracleSystem(n)):
        if isinstance(b, Engine):
            b.set_fire_order(True)
        sim = drive(b, parts, (L, L, 10.0), nlist=(2.8, 0.3), pairs=[("soft", {"k": "1", "use_particle_radii": ""})],
                    dt=0.01, integrators=[("fire", {"dt_max": "0.1", "fmax_tolerance": "1e-10"})])
        sim.commit()
        steps, _ = b.minimize(200000)
        out.append((b, int(steps[0])))
    (e, se), (o, so) = out
    assert se == so > 0
    for f in ("x", "y", "vx", "vy", "fx", "fy"):
        np.testing.assert_array_equal(e.download(f), o.download(f), err_msg=f)


@pytest.mark.parametrize("shape", ["plane", "sphere"])
def test_hot_kernels_match_generic_kernels_bitwise(shape):
    n = 2500
    if shape == "plane":
        parts, L = plane_disks(n, 0.7, seed=21)
        kw = dict(box=(L, L, 10.0), periodic=True, constraint=("plane", {}))
    else:
        parts, R = sphere_disks(n, seed=21)
        b = 2 * R + 6.0
        kw = dict(box=(b, b, b), periodic=False, constraint=("sphere", {"r": repr(R)}))
    out = []
    for path in (0, 1, 2):
        e = Engine(n)
        e.set_path(path)
        sim = drive(e, parts, kw["box"], periodic=kw["periodic"], nlist=(2.4, 0.3), constraint=kw["constraint"],
                    pairs=[("soft", {"k": "10", "use_particle_radii": ""})], aligns=[("polar", {"J": "0.3"})],
                    externals=[("self_propulsion", {"alpha": "0.2"})], dt=1e-3,
                    integrators=[("brownian", {"v0": "0.5", "nu": "0.2", "seed": "9", "min_val": "0.05"})])
        sim.run(300)
        out.append(e)
    for f in ("x", "y", "z", "nx", "ny", "nz", "vx", "vy", "vz", "fx", "fy", "tau_z", "omega", "age", "ix", "iy"):
        ref = out[1].download(f)
        np.testing.assert_array_equal(out[0].download(f), ref, err_msg=f + " (specialised vs generic)")
        np.testing.assert_array_equal(out[2].download(f), ref, err_msg=f + " (packed vs generic)")


VARIANT_CASES = {
    # the headline program, slow motion (no rebuild in 120 steps)
    "plane_nematic": dict(n=3000, phi=0.8, v0="0.3", dt=5e-4, steps=120, align=("nematic", {"J": "0.5"}), sp=False),
    # fast motion: list-only rebuilds and full re-sorts (every 8th build) inside the run
    "plane_polar_fast": dict(n=3000, phi=0.7, v0="3.0", dt=5e-3, steps=200, align=("polar", {"J": "0.2"}), sp=False),
    # sphere with polar alignment and self-propulsion
    "sphere_polar_sp": dict(n=3000, phi=None, v0="1.0", dt=1e-3, steps=120, align=("polar", {"J": "0.2"}), sp=True),
}


@pytest.mark.parametrize("case", sorted(VARIANT_CASES))
@pytest.mark.parametrize("variant", list(range(32)))
def test_every_tuning_variant_gives_identical_bits(variant, case):
    c = VARIANT_CASES[case]
    n = c["n"]
    if c["phi"] is None:
        parts, R = sphere_disks(n, seed=23)
        box, periodic, cons = (2 * R + 10,) * 3, False, ("sphere", {"r": repr(R)})
        pairs = [("soft", {"k": "10"})]
    else:
        parts, L = plane_disks(n, c["phi"], seed=22, bidisperse=(1.0, 1.4))
        box, periodic, cons = (L, L, 10.0), True, ("plane", {})
        pairs = [("soft", {"k": "10", "use_particle_radii": ""})]
    outs = []
    for v in (variant, -2):
        e = Engine(n)
        if v >= 0:
            e.set_variant(v)
        else:
            e.set_path(1)
        sim = drive(e, parts, box, periodic=periodic, nlist=(2.8, 0.3), constraint=cons, pairs=pairs,
                    aligns=[c["align"]], externals=[("self_propulsion", {"alpha": "0.5"})] if c["sp"] else [],
                    dt=c["dt"], integrators=[("brownian", {"v0": c["v0"], "nu": "0.1", "seed": "1"})])
        st = sim.run(c["steps"])
        outs.append((e, st))
    if case == "plane_polar_fast":
        assert outs[0][1].nlist_builds >= 9  # at least one full re-sort besides list-only builds
    fields = ["x", "y", "z", "nx", "ny", "nz", "vx", "vy", "vz", "fx", "fy", "fz", "tau_x", "tau_y", "tau_z", "omega",
              "age", "ix", "iy"]
    for f in fields:
        np.testing.assert_array_equal(outs[0][0].download(f), outs[1][0].download(f), err_msg=f)


@pytest.mark.parametrize("kind,shape,box,n", [
    ("cylinder", {"r": 10.0, "Lz": 60.0}, (40.0, 40.0, 60.0), 700),
    ("torus", {"c": 20.0, "a": 8.0}, (70.0, 70.0, 30.0), 1500),
    ("ellipsoid", {"a": 20.0, "b": 15.0, "c": 12.0}, (50.0, 40.0, 34.0), 800),
])
def test_trajectory_curved_constraints(kind, shape, box, n):
    # active Brownian particles on a cylinder / torus / ellipsoid (the generic
    # fused kernel), 300 steps against the oracle with the shared noise stream
    parts = surface_disks(kind, n, seed=17, **shape)
    conf = {k: repr(v) for k, v in shape.items() if k != "Lz"}
    e, o = run_both(n, parts, box, 299, periodic=(kind == "cylinder"), nlist=(2.4, 0.3), constraint=(kind, conf),
                    pairs=[("soft", {"k": "10"})], aligns=[("polar", {"J": "0.2"})], dt=1e-3,
                    integrators=[("brownian", {"v0": "1.0", "nu": "0.1", "seed": "4"})])
    assert_traj(e, o)


@pytest.mark.parametrize("kind,shape,conf,box,periodic,n", [
    ("peanut", {"a": 8.0, "b": 10.0}, {"a": "8.0", "b": "10.0"}, (60.0, 60.0, 60.0), False, 400),
    ("hourglass", {"R": 10.0, "A": 2.0, "n_nodes": 2.0, "Lz": 40.0}, {"R": "10.0", "A": "2.0", "n": "2.0"},
     (40.0, 40.0, 40.0), False, 700),
    ("gaussian_bump", {"A": 4.0, "a": 30.0, "b": 20.0, "L": 40.0}, {"A": "4.0", "a": "30.0", "b": "20.0"},
     (40.0, 40.0, 20.0), False, 400),
    ("gyroid", {"box": (30.0, 30.0, 30.0)}, {}, (30.0, 30.0, 30.0), True, 800),
    ("tetrahedron", {"scale": 10.0, "value": 0.3}, {"scale": "10.0", "value": "0.3"}, (80.0, 80.0, 80.0), False, 600),
])
def test_trajectory_implicit_surfaces(kind, shape, conf, box, periodic, n):
    # active Brownian particles on a peanut / hourglass / Gaussian bump /
    # gyroid / tetrahedral equipotential (SHAKE projection of the implicit surface, the generic fused
    # kernel), 300 steps against the oracle with the shared noise stream
    parts = surface_disks(kind, n, seed=18, **shape)
    e, o = run_both(n, parts, box, 299, periodic=periodic, nlist=(2.4, 0.3), constraint=(kind, conf),
                    pairs=[("soft", {"k": "10"})], aligns=[("polar", {"J": "0.2"})], dt=1e-3,
                    integrators=[("brownian", {"v0": "1.0", "nu": "0.1", "seed": "4"})])
    assert_traj(e, o)


def test_trajectory_slab_and_walls():
    # 3-D active particles between the slab's planes (reflections, no
    # rotation: constraint_slab.hpp:85-91) and 2-D ones between walls at
    # x = +-l (constraint_plane_walls.cpp), 300 steps against the oracle
    rng = np.random.default_rng(31)
    n, L = 1200, 40.0
    d = rng.normal(size=(3, n))
    d /= np.linalg.norm(d, axis=0)
    parts = dict(x=rng.uniform(-L / 2, L / 2, n), y=rng.uniform(-L / 2, L / 2, n), z=rng.uniform(-2.5, 2.5, n),
                 vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n), nx=d[0], ny=d[1], nz=d[2], radius=np.full(n, 1.0))
    e, o = run_both(n, parts, (L, L, 20.0), 299, periodic=True, nlist=(2.4, 0.3),
                    constraint=("slab", {"z_lo": "-2.0", "z_hi": "2.0"}), pairs=[("soft", {"k": "10"})],
                    aligns=[("polar", {"J": "0.2"})], dt=1e-3,
                    integrators=[("brownian", {"v0": "3.0", "nu": "0.1", "seed": "5"})])
    assert_traj(e, o)
    assert np.all(np.abs(e.download("z")) <= 2.0)
    parts, L = plane_disks(1500, 0.5, seed=32)
    e, o = run_both(1500, parts, (L, L, 10.0), 299, periodic=True, nlist=(2.4, 0.3),
                    constraint=("walls", {"l": repr(0.4 * L)}), pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
                    aligns=[("polar", {"J": "0.2"})], dt=1e-3,
                    integrators=[("brownian", {"v0": "3.0", "nu": "0.1", "seed": "6"})])
    assert_traj(e, o)
    assert np.all(np.abs(e.download("x")) <= 0.4 * L)


def test_trajectory_vicsek_model():
    # the Vicsek integrator with the Vicsek aligner (and a soft repulsion
    # through the mobility), on the generic fused kernel
    n = 1500
    parts, L = plane_disks(n, 0.4, seed=14)
    rng = np.random.default_rng(14)
    th = rng.uniform(0, 2 * np.pi, n)
    parts["vx"], parts["vy"] = np.cos(th), np.sin(th)
    e, o = run_both(n, parts, (L, L, 10.0), 299, nlist=(2.4, 0.3),
                    pairs=[("soft", {"k": "10", "use_particle_radii": ""})], aligns=[("vicsek", {"rcut": "2.0"})],
                    dt=1e-2, integrators=[("vicsek", {"v0": "0.5", "eta": "0.3", "mu": "0.1", "seed": "5"})])
    assert_traj(e, o, ("x", "y", "vx", "vy"))


def test_trajectory_vicsek_generic_fused_path():
    n = 1200
    parts, L = plane_disks(n, 0.5, seed=12)
    rng = np.random.default_rng(12)
    parts["vx"], parts["vy"] = rng.normal(size=n), rng.normal(size=n)
    e, o = run_both(n, parts, (L, L, 10.0), 299, nlist=(2.4, 0.3),
                    pairs=[("soft", {"k": "10", "use_particle_radii": ""})], aligns=[("vicsek", {"rcut": "2.0"})],
                    dt=1e-3, integrators=[("brownian", {"v0": "0.5", "nu": "0.1", "seed": "3"})])
    assert_traj(e, o)


def test_coordination_counts_contacts_at_the_build():
    # Particle::coordination (neighbour_list.cpp:185-206, 229-268): every
    # listed pair within the sum of the radii at the build counts for both
    parts, L = plane_disks(3000, 0.7, seed=41)
    e = Engine(3000)
    drive(e, parts, (L, L, 10.0), nlist=(2.4, 0.3))
    e.build_nlist()
    i, j = e.pairs()
    x, y, r = e.download("x"), e.download("y"), e.download("radius")
    dx, dy = x[i] - x[j], y[i] - y[j]
    dx -= L * np.round(dx / L)
    dy -= L * np.round(dy / L)
    touch = dx * dx + dy * dy < (r[i] + r[j]) ** 2
    want = np.bincount(i[touch], minlength=3000) + np.bincount(j[touch], minlength=3000)
    np.testing.assert_array_equal(e.coordination(), want)
    assert want.sum() > 3000


@pytest.mark.parametrize("integrators", [
    # the two-component example: one brownian integrator per group, the passive one at T > 0
    [("brownian", {"group": "active", "v0": "0.5", "nu": "0.01", "seed": "1"}),
     ("brownian", {"group": "passive", "v0": "0.0", "nu": "0.0", "seed": "4", "temperature_control": "constant",
                   "min_val": "0.3"})],
    # positions of one group, rotations of all (nematic flips), map order across groups
    [("brownian_pos", {"group": "passive", "seed": "2", "min_val": "0.1"}),
     ("brownian_align", {"seed": "5", "nu": "0.2", "nematic": "", "tau": "0.5"})],
])
def test_trajectory_grouped_integrators(integrators):
    n = 1800
    parts, L = plane_disks(n, 0.6, seed=45)
    parts["type"] = np.where(np.arange(n) % 3 == 0, 2, 1)
    runs = []
    for b in (Engine(n, 2), OracleSystem(n, 2)):
        sim = drive(b, parts, (L, L, 10.0), nlist=(2.4, 0.3), pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
                    aligns=[("polar", {"J": "0.2"})], dt=1e-3, ntypes=2)
        sim.group("passive", {"type": "1"})
        sim.group("active", {"type": "2"})
        for name, p in integrators:
            sim.integrator(name, dict(p))
        sim.run(299)
        runs.append(b)
    assert_traj(*runs)


def test_trajectory_sphere_rescale():
    # ConstraintSphere::rescale (constraint_sphere.cpp:87-104): every
    # rescale_freq steps below rescale_steps the radius grows by
    # rescale^(freq/steps), every particle is projected onto the new sphere and
    # the lists are rebuilt (samos.cpp:882-886)
    parts, R = sphere_disks(1500, seed=46)
    conf = {"r": repr(R), "rescale": "1.5", "rescale_steps": "1000", "rescale_freq": "10"}
    box = (4 * R + 10.0,) * 3
    e, o = run_both(1500, parts, box, 299, periodic=False, nlist=(2.4, 0.3), constraint=("sphere", conf),
                    pairs=[("soft", {"k": "10"})], aligns=[("polar", {"J": "0.2"})], dt=1e-3,
                    integrators=[("brownian", {"v0": "1.0", "nu": "0.1", "seed": "4"})])
    assert_traj(e, o)
    r_end = np.sqrt(e.download("x") ** 2 + e.download("y") ** 2 + e.download("z") ** 2)
    np.testing.assert_allclose(r_end, R * (1.5 ** (10 / 1000)) ** 30, rtol=1e-12)


def test_sphere_rescale_across_runs_and_begin_step():
    # two `run` commands continue the global step the rescale is keyed on
    # (ConstraintSphere::rescale reads System::get_step); sg_begin_step (the
    # dump/log point at the top of a step) applies a due rescale once
    parts, R = sphere_disks(1200, seed=47)
    conf = {"r": repr(R), "rescale": "0.8", "rescale_steps": "300", "rescale_freq": "7"}
    kw = dict(periodic=False, nlist=(2.4, 0.3), constraint=("sphere", conf), pairs=[("soft", {"k": "10"})],
              aligns=[("nematic", {"J": "0.3"})], dt=1e-3,
              integrators=[("brownian", {"v0": "0.8", "nu": "0.1", "seed": "5"})])
    box = (4 * R + 10.0,) * 3
    e, o = Engine(1200), OracleSystem(1200)
    se, so = drive(e, parts, box, **kw), drive(o, parts, box, **kw)
    se.run(139)
    so.run(139)
    e.begin_step()  # step 140 is a rescale step (140 % 7 == 0)
    e.begin_step()
    se.run(200)
    so.run(200)
    assert_traj(e, o)
    events = len(range(0, 300, 7))
    r_end = np.sqrt(e.download("x") ** 2 + e.download("y") ** 2 + e.download("z") ** 2)
    np.testing.assert_allclose(r_end, R * (0.8 ** (7 / 300)) ** events, rtol=1e-12)


@pytest.mark.parametrize("kind,shape,conf,box,periodic,n,a", [
    ("cylinder", {"r": 10.0, "Lz": 60.0}, {"r": "10.0"}, (40.0, 40.0, 60.0), True, 700, 1.3),
    ("tetrahedron", {"scale": 10.0, "value": 0.3}, {"scale": "10.0", "value": "0.3"}, (90.0, 90.0, 90.0), False, 600,
     0.8),
])
def test_trajectory_rescaled_cylinder_and_tetrahedron(kind, shape, conf, box, periodic, n, a):
    # ConstraintCylinder::rescale (constraint_cylinder.cpp:79-96: steps up to
    # and including rescale_steps) and ConstraintTetrahedron::rescale
    # (constraint_tetrahedron.cpp:88-109: below it, charges move with the
    # scale).  The tetrahedron shrinks: growing its charges apart at a fixed
    # level pinches the surface into lobes, where the SHAKE projection (and the
    # reference's, constraint.cpp:40-87) divides by a vanishing gradient product
    parts = surface_disks(kind, n, seed=19, **shape)
    conf = dict(conf, rescale=repr(a), rescale_steps="200", rescale_freq="10")
    e, o = run_both(n, parts, box, 299, periodic=periodic, nlist=(2.4, 0.3), constraint=(kind, conf),
                    pairs=[("soft", {"k": "10"})], aligns=[("polar", {"J": "0.2"})], dt=1e-3,
                    integrators=[("brownian", {"v0": "1.0", "nu": "0.1", "seed": "4"})])
    assert_traj(e, o)
    f = a ** (10 / 200)
    x, y, z = e.download("x"), e.download("y"), e.download("z")
    if kind == "cylinder":
        np.testing.assert_allclose(np.hypot(x, y), 10.0 * f ** 21, rtol=1e-12)
    else:
        assert np.max(np.abs(tetra_value(np.stack([x, y, z], 1), 10.0 * f ** 20, 0.3))) < 2e-6


def test_generic_kernel_occupancy_choices_give_the_same_bits():
    # the generic fused kernel bounded for 6 or 8 blocks per SM, pinned or
    # picked by timing the run's first steps: same bits
    n = 1500
    parts = surface_disks("torus", n, seed=17, c=20.0, a=8.0)
    kw = dict(periodic=False, nlist=(2.4, 0.3), constraint=("torus", {"c": "20.0", "a": "8.0"}),
              pairs=[("soft", {"k": "10"})], aligns=[("polar", {"J": "0.2"})], dt=1e-3,
              integrators=[("brownian", {"v0": "1.0", "nu": "0.1", "seed": "4"})])
    outs = []
    for occ in (6, 8, 0):
        e = Engine(n)
        e.set_generic_occupancy(occ)
        drive(e, parts, (70.0, 70.0, 30.0), **kw).run(199)
        assert e.generic_occupancy() in ((6, 8) if occ == 0 else (occ,))
        outs.append(e)
    for f in ("x", "y", "z", "nx", "ny", "nz", "vx", "vy", "vz"):
        np.testing.assert_array_equal(outs[0].download(f), outs[1].download(f), err_msg=f)
        np.testing.assert_array_equal(outs[0].download(f), outs[2].download(f), err_msg=f)


@pytest.mark.parametrize("kind", ["torus", "vicsek"])
def test_generic_batched_stepping_gives_the_stepwise_bits(kind):
    # the generic fused kernel enqueues up to 32 steps per host round trip,
    # a step that flags a rebuild halting the rest; profiling mode steps one
    # at a time: both must give the same bits, through rebuilds
    if kind == "torus":
        shape = {"c": 20.0, "a": 8.0}
        n, box = 1500, (70.0, 70.0, 30.0)
        parts = surface_disks("torus", n, seed=27, **shape)
        kw = dict(periodic=False, nlist=(2.4, 0.3), constraint=("torus", {k: repr(v) for k, v in shape.items()}),
                  pairs=[("soft", {"k": "10"})], aligns=[("polar", {"J": "0.2"})], dt=1e-3,
                  integrators=[("brownian", {"v0": "2.0", "nu": "0.1", "seed": "4"})])
    else:
        n = 2000
        parts, L = plane_disks(n, 0.5, seed=28)
        box = (L, L, 10.0)
        kw = dict(nlist=(2.4, 0.3), pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
                  aligns=[("vicsek", {"rcut": "2.0"})], dt=1e-2,
                  integrators=[("vicsek", {"v0": "0.5", "eta": "0.3", "mu": "0.1", "seed": "5"})])
    out = []
    for prof in (False, True):
        e = Engine(n)
        e.set_profiling(prof)
        sim = drive(e, parts, box, **kw)
        st = sim.run(400)
        out.append((e, st))
    assert out[0][1].nlist_builds > 2  # rebuilds inside the batches
    for f in ("x", "y", "z", "nx", "ny", "nz", "vx", "vy", "vz", "fx", "fy", "age", "ix", "iy"):
        np.testing.assert_array_equal(out[0][0].download(f), out[1][0].download(f), err_msg=f)


@pytest.mark.parametrize("integ", [
    ("langevin", {"gamma": "1", "seed": "7", "method": "baoab", "min_val": "1.0"}),
    ("langevin", {"gamma": "1", "seed": "7", "method": "bbk", "min_val": "1.0"}),
    ("nve", {}),
])
def test_unfused_batched_stepping_gives_the_stepwise_bits(integ):
    # Langevin / NVE steps with reused forces are enqueued up to 32 per host
    # round trip (halted after a step that flags a rebuild); profiling mode
    # steps one at a time: the same bits, through rebuilds
    n = 1500
    parts, L = plane_disks(n, 0.6, seed=29)
    kw = dict(nlist=(2.5, 0.3), pairs=[("soft", {"k": "1.0"})], aligns=[("polar", {"J": "1.0"})], dt=2e-3,
              integrators=[integ])
    out = []
    for prof in (False, True):
        e = Engine(n)
        e.set_profiling(prof)
        sim = drive(e, parts, (L, L, 10.0), **kw)
        st = sim.run(400)
        out.append((e, st))
    assert out[0][1].nlist_builds >= 1
    for f in ("x", "y", "vx", "vy", "nx", "ny", "omega", "fx", "fy", "age", "ix", "iy"):
        np.testing.assert_array_equal(out[0][0].download(f), out[1][0].download(f), err_msg=f)


@pytest.mark.parametrize("align", ["polar", "nematic"])
def test_run_energies_on_every_path(align):
    # the energies a run reports come from its last step's force evaluation:
    # on the specialised path that step runs the pipelined kernel, whose lanes
    # are in neighbour-count order and whose block sums are taken in slot order,
    # so they are the generic and packed paths' sums bit for bit; against the
    # oracle (a sequential sum) within the per-step bar
    parts, L = plane_disks(3000, 0.8, seed=51, bidisperse=(1.0, 1.4))
    res = []
    for backend, path in ((Engine, 0), (Engine, 1), (Engine, 2), (OracleSystem, None)):
        b = backend(3000)
        if path is not None:
            b.set_path(path)
        sim = drive(b, parts, (L, L, 10.0), nlist=(2.8, 0.3), pairs=[("soft", {"k": "10", "use_particle_radii": ""})],
                    aligns=[(align, {"J": "0.5"})], dt=5e-4,
                    integrators=[("brownian", {"v0": "0.3", "nu": "0.1", "seed": "4"})])
        sim.run(40)
        res.append((b.energy(0, 0), b.energy(1, 0)))
    specialised, generic, packed, oracle = res
    assert specialised == generic == packed
    assert specialised[0] == pytest.approx(oracle[0], rel=REL)
    assert specialised[1] == pytest.approx(oracle[1], rel=REL)
