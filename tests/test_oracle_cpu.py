"""CPU checks of the oracle against hand-derived known answers (the
reference ships no test vectors): two-particle forces/energies of each pair
potential, aligner torques, constraint projections, integrator steps, the
neighbour-list build invariants and the noise stream."""
import math

import numpy as np
import pytest

from oracle.oracle import OracleSystem, noise_gauss, noise_log, noise_uniform
from samos_b200 import engine as E
from scenarios import (drive, gyroid_gradient, gyroid_value, plane_disks, sphere_disks, surface_disks, tetra_gradient,
                       tetra_value)


def two(x2, y2=0.0, r=(1.0, 1.0), box=20.0, n1=(1.0, 0.0, 0.0), n2=(0.0, 1.0, 0.0)):
    parts = dict(x=np.array([0.0, x2]), y=np.array([0.0, y2]), z=np.zeros(2),
                 nx=np.array([n1[0], n2[0]]), ny=np.array([n1[1], n2[1]]), nz=np.array([n1[2], n2[2]]),
                 radius=np.array(r, float))
    return parts, (box, box, box)


def run_compute(parts, box, pairs=(), aligns=(), externals=(), nlist=(3.0, 0.5)):
    o = OracleSystem(len(parts["x"]))
    sim = drive(o, parts, box, nlist=nlist, constraint=None, pairs=pairs, aligns=aligns, externals=externals)
    sim.commit()
    o.compute(1e-3)
    return o


def test_soft_two_particles():
    parts, box = two(1.5, r=(1.0, 0.8))
    o = run_compute(parts, box, pairs=[("soft", {"k": "10", "use_particle_radii": ""})])
    # U = k/2 (a_i + a_j - r)^2, F_i = -k (a_i+a_j-r) * (x_j - x_i)/r
    d = 1.8 - 1.5
    assert o.energy(0, 0) == pytest.approx(0.5 * 10 * d * d, rel=1e-15)
    fx = o.download("fx")
    assert fx[0] == pytest.approx(-10 * d, rel=1e-14)
    assert fx[1] == -fx[0]


def test_soft_out_of_contact_is_zero():
    parts, box = two(2.5, r=(1.0, 1.0))
    o = run_compute(parts, box, pairs=[("soft", {"k": "10", "use_particle_radii": ""})])
    assert o.energy(0, 0) == 0.0
    assert np.all(o.download("fx") == 0.0)


def test_lj_two_particles_reference_force_factor():
    parts, box = two(1.2)
    o = run_compute(parts, box, pairs=[("lj", {"epsilon": "1.5", "sigma": "1.1", "rcut": "2.5"})])
    s2 = 1.1 ** 2 / 1.2 ** 2
    s6 = s2 ** 3
    assert o.energy(0, 0) == pytest.approx(4 * 1.5 * s6 * (s6 - 1), rel=1e-13)
    # the reference multiplies by sigma^2/r^2 (pair_lj_potential.cpp:107)
    ff = 48 * 1.5 * s6 * (s6 - 0.5) * s2
    assert o.download("fx")[0] == pytest.approx(ff * (0.0 - 1.2), rel=1e-13)


def test_morse_two_particles():
    parts, box = two(1.3)
    o = run_compute(parts, box, pairs=[("morse", {"D": "2", "a": "1.5", "re": "1.1", "rcut": "3"})])
    e = math.exp(-1.5 * (1.3 - 1.1))
    assert o.energy(0, 0) == pytest.approx(2 * (e - 1) ** 2 - 2, rel=1e-13)
    ff = 2 * 2 * 1.5 * e * (e - 1) / 1.3
    assert o.download("fx")[0] == pytest.approx(ff * (0.0 - 1.3), rel=1e-13)


def test_gaussian_shift_and_table_quirk():
    parts, box = two(1.0)
    o = run_compute(parts, box, pairs=[("gaussian", {"A": "2", "B": "-1", "alpha": "1", "beta": "3",
                                                     "rA": "0", "rB": "1.5", "rcut": "2.5", "shifted": ""})])
    u = 2 * math.exp(-1.0) - math.exp(-3 * 0.25)
    shift = 2 * math.exp(-6.25) - math.exp(-3 * 1.0)
    assert o.energy(0, 0) == pytest.approx(u - shift, rel=1e-13)


def test_polar_and_nematic_torques():
    parts, box = two(1.0, n1=(1.0, 0.0, 0.0), n2=(math.cos(0.3), math.sin(0.3), 0.0))
    o = run_compute(parts, box, aligns=[("polar", {"J": "0.7", "rcut": "2"})])
    tz = o.download("tau_z")
    assert tz[0] == pytest.approx(0.7 * math.sin(0.3), rel=1e-14)
    assert tz[1] == -tz[0]
    assert o.energy(1, 0) == pytest.approx(-2 * 0.7 * math.cos(0.3), rel=1e-14)
    o = run_compute(parts, box, aligns=[("nematic", {"J": "0.7", "rcut": "2"})])
    # J doubled by default (pair_nematic_aligner.cpp:37)
    assert o.download("tau_z")[0] == pytest.approx(1.4 * math.cos(0.3) * math.sin(0.3), rel=1e-14)


def test_vicsek_normalises():
    parts, box = two(1.0)
    parts["vx"] = np.array([1.0, 0.0])
    parts["vy"] = np.array([0.0, 2.0])
    o = run_compute(parts, box, aligns=[("vicsek", {"rcut": "2"})])
    t = np.stack([o.download("tau_x"), o.download("tau_y")], 1)
    assert np.allclose(np.linalg.norm(t, axis=1), 1.0)
    assert np.allclose(t[0], np.array([1.0, 2.0]) / math.sqrt(5))


def test_self_propulsion_adds_alpha_n():
    parts, box = two(5.0)
    o = run_compute(parts, box, externals=[("self_propulsion", {"alpha": "0.5"})])
    assert np.allclose(o.download("fx"), [0.5, 0.0])
    assert np.allclose(o.download("fy"), [0.0, 0.5])


def test_brownian_step_without_force_or_noise():
    # one step, zero force, nu = 0: x advances exactly by dt*v0*n
    parts, box = two(8.0)
    o = OracleSystem(2)
    sim = drive(o, parts, box, constraint=("plane", {}), pairs=[("soft", {"k": "1", "use_particle_radii": ""})],
                dt=0.01, integrators=[("brownian", {"v0": "0.5", "nu": "0", "seed": "1"})])
    sim.run(0)  # run 0 = one integration step
    assert o.download("x")[0] == 0.0 + 0.01 * 0.5
    assert o.download("y")[1] == 0.0 + 0.01 * 0.5


def test_sphere_projection_keeps_radius():
    parts, R = sphere_disks(300, seed=3)
    o = OracleSystem(300)
    drive(o, parts, (2 * R + 10, 2 * R + 10, 2 * R + 10), periodic=False, constraint=("sphere", {"r": str(R)}))
    r = np.sqrt(o.download("x") ** 2 + o.download("y") ** 2 + o.download("z") ** 2)
    assert np.allclose(r, R, rtol=1e-15, atol=0)
    n = np.stack([o.download("nx"), o.download("ny"), o.download("nz")], 1)
    pos = np.stack([o.download("x"), o.download("y"), o.download("z")], 1)
    assert np.allclose(np.sum(n * pos, 1) / R, 0.0, atol=1e-14)


def test_cell_and_nsq_builds_give_same_pair_set():
    parts, L = plane_disks(600, 0.6, seed=4)
    a = OracleSystem(600)
    drive(a, parts, (L, L, 10.0), nlist=(2.4, 0.3), constraint=None)
    assert a.uses_cells()
    b = OracleSystem(600)
    drive(b, parts, (L, L, 4.0), nlist=(2.4, 0.3), constraint=None)  # lz <= 2 cut -> N^2 path
    assert not b.uses_cells()
    sa = set(zip(*[x.tolist() for x in a.pairs()]))
    sb = set(zip(*[x.tolist() for x in b.pairs()]))
    assert sa == sb and len(sa) > 0
    assert all(i < j for i, j in sa)


def test_fire_relaxes_two_overlapping_disks_to_contact():
    parts, box = two(1.2, r=(1.0, 1.0))
    o = OracleSystem(2)
    sim = drive(o, parts, box, constraint=("plane", {}), pairs=[("soft", {"k": "1", "use_particle_radii": ""})],
                dt=0.01, integrators=[("fire", {"fmax_tolerance": "1e-10"})])
    sim.commit()
    steps, _ = o.minimize(100000)
    assert steps[0] > 0
    x = o.download("x")
    # soft repulsion is flat beyond contact: the minimum is any separation >= 2
    assert abs(x[1] - x[0]) > 2.0 - 1e-10
    assert np.max(np.abs(o.download("fx"))) < 1e-10


def test_noise_stream_statistics():
    g = np.array([noise_gauss(5, c) for c in range(20000)])
    assert abs(g.mean()) < 0.03 and abs(g.std() - 1.0) < 0.02
    u = np.array([noise_uniform(5, c) for c in range(20000)])
    assert u.min() >= 0.0 and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.01
    for x in (1e-300, 1e-5, 0.3, 0.7071, 0.99999999):
        assert noise_log(x) == pytest.approx(math.log(x), rel=4e-16, abs=1e-300)


def test_run_executes_steps_plus_one():
    parts, box = two(8.0)
    o = OracleSystem(2)
    sim = drive(o, parts, box, constraint=("plane", {}), pairs=[("soft", {})], dt=0.01,
                integrators=[("brownian", {"v0": "1", "nu": "0"})])
    sim.run(9)  # samos.cpp:878 runs t = 0..9
    assert o.download("x")[0] == pytest.approx(10 * 0.01, rel=1e-14)
    assert o.download("age")[0] == pytest.approx(10 * 0.01, rel=1e-14)


def test_nve_limit_clamps_displacement_and_speed():
    # free particle, v = (3, 4, 0), dt = 0.1, limit = 0.2 (integrator_nve.cpp:57-76, 96-105):
    # the drift 0.5 is cut to 0.2 along v, and |v| dt = 0.5 > 0.2 cuts v to 0.2 / dt
    parts, box = two(8.0)
    parts["vx"] = np.array([3.0, 0.0]); parts["vy"] = np.array([4.0, 0.0]); parts["vz"] = np.zeros(2)
    o = OracleSystem(2)
    sim = drive(o, parts, box, constraint=("plane", {}), dt=0.1, integrators=[("nve", {"limit": "0.2"})])
    sim.run(0)
    assert o.download("x")[0] == pytest.approx(0.12, abs=1e-15)
    assert o.download("y")[0] == pytest.approx(0.16, abs=1e-15)
    assert o.download("vx")[0] == pytest.approx(1.2, abs=1e-14)
    assert o.download("vy")[0] == pytest.approx(1.6, abs=1e-14)
    # the resting particle does not move
    assert o.download("x")[1] == 8.0 and o.download("vx")[1] == 0.0


def test_nve_without_limit_is_velocity_verlet():
    parts, box = two(1.5, r=(1.0, 1.0))  # overlapping soft disks push apart symmetrically
    o = OracleSystem(2)
    sim = drive(o, parts, box, constraint=("plane", {}), pairs=[("soft", {"k": "1", "use_particle_radii": ""})],
                dt=0.01, integrators=[("nve", {})])
    sim.run(99)
    x, vx = o.download("x"), o.download("vx")
    assert x[0] < 0.0 < 1.5 < x[1]
    assert vx[0] == -vx[1]  # momentum conserved exactly by the symmetric update


def test_vicsek_integrator_follows_the_aligned_velocity():
    # integrator_vicsek.cpp:62-80 with eta = 0: v = v0 tau, tau the normalised
    # sum of the velocities around (here the particle's own, (3, 4) -> (0.6, 0.8))
    parts, box = two(8.0)
    parts["vx"] = np.array([3.0, 0.0]); parts["vy"] = np.array([4.0, 1.0]); parts["vz"] = np.zeros(2)
    o = OracleSystem(2)
    sim = drive(o, parts, box, constraint=("plane", {}), aligns=[("vicsek", {"rcut": "1.0"})], dt=0.1,
                integrators=[("vicsek", {"v0": "0.5", "eta": "0", "seed": "3"})])
    sim.run(0)
    assert o.download("vx")[0] == pytest.approx(0.3, abs=1e-15)
    assert o.download("vy")[0] == pytest.approx(0.4, abs=1e-15)
    assert o.download("x")[0] == pytest.approx(0.03, abs=1e-15)
    assert o.download("y")[0] == pytest.approx(0.04, abs=1e-15)
    assert o.download("y")[1] == pytest.approx(0.05, abs=1e-15)  # (0, 1) -> v0 * (0, 1) * dt


@pytest.mark.parametrize("kind,shape,box", [
    ("cylinder", {"r": 10.0, "Lz": 40.0}, (40.0, 40.0, 40.0)),
    ("torus", {"c": 12.0, "a": 5.0}, (50.0, 50.0, 50.0)),
    ("ellipsoid", {"a": 12.0, "b": 9.0, "c": 7.0}, (40.0, 40.0, 40.0)),
])
def test_curved_constraints_project_onto_their_surface(kind, shape, box):
    # constraint_cylinder.cpp:38-71 (radial), Constraint::enforce SHAKE for
    # the implicit torus and ellipsoid (constraint.cpp:40-87): positions on
    # the surface, directors unit and tangent
    parts = surface_disks(kind, 300, seed=5, **shape)
    o = OracleSystem(300)
    conf = {k: repr(v) for k, v in shape.items() if k != "Lz"}
    drive(o, parts, box, periodic=(kind == "cylinder"), constraint=(kind, conf))
    x, y, z = o.download("x"), o.download("y"), o.download("z")
    n = np.stack([o.download("nx"), o.download("ny"), o.download("nz")], 1)
    if kind == "cylinder":
        assert np.allclose(np.hypot(x, y), shape["r"], rtol=1e-14)
        N = np.stack([x / shape["r"], y / shape["r"], 0 * z], 1)
    elif kind == "torus":
        g = (shape["c"] - np.hypot(x, y)) ** 2 + z ** 2 - shape["a"] ** 2
        assert np.abs(g).max() <= 1e-6
        s = np.hypot(x, y)
        N = np.stack([-2 * (shape["c"] - s) / s * x, -2 * (shape["c"] - s) / s * y, 2 * z], 1)
        N /= np.linalg.norm(N, axis=1)[:, None]
    else:
        g = x ** 2 / shape["a"] ** 2 + y ** 2 / shape["b"] ** 2 + z ** 2 / shape["c"] ** 2 - 1.0
        assert np.abs(g).max() <= 1e-6
        N = np.stack([2 * x / shape["a"] ** 2, 2 * y / shape["b"] ** 2, 2 * z / shape["c"] ** 2], 1)
        N /= np.linalg.norm(N, axis=1)[:, None]
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-14)
    assert np.abs(np.sum(n * N, 1)).max() <= 1e-6


IMPLICIT_CASES = [
    ("peanut", {"a": 8.0, "b": 10.0}, {"a": 8.0, "b": 10.0}, (60.0, 60.0, 60.0), False),
    ("hourglass", {"R": 10.0, "A": 2.0, "n_nodes": 2.0, "Lz": 40.0}, {"R": 10.0, "A": 2.0, "n": 2.0},
     (40.0, 40.0, 40.0), False),
    ("gaussian_bump", {"A": 4.0, "a": 30.0, "b": 20.0, "L": 40.0}, {"A": 4.0, "a": 30.0, "b": 20.0},
     (40.0, 40.0, 20.0), False),
    ("gyroid", {"box": (30.0, 30.0, 30.0)}, {}, (30.0, 30.0, 30.0), True),
    ("tetrahedron", {"scale": 10.0, "value": 0.3}, {"scale": 10.0, "value": 0.3}, (80.0, 80.0, 80.0), False),
]


def implicit_np(kind, conf, box, x, y, z):
    """g and its normalised gradient in numpy, from the formulas in the
    reference's constraint_<kind>.cpp."""
    if kind == "peanut":
        a, b = conf["a"], conf["b"]
        tr = x * x + y * y + z * z
        g = a ** 4 - b ** 4 - 2 * a * a * (x * x - y * y - z * z) + tr * tr
        G = np.stack([(-4 * a * a + 4 * tr) * x, (4 * a * a + 4 * tr) * y, (4 * a * a + 4 * tr) * z], 1)
    elif kind == "hourglass":
        R, A, nn, lz = conf["R"], conf["A"], conf["n"], box[2]
        zf = R + A * np.sin(2 * np.pi * nn * z / lz)
        g = x * x + y * y - zf * zf
        G = np.stack([2 * x, 2 * y, -4 * A * nn * np.pi * np.cos(2 * nn * np.pi * z / lz) * zf / lz], 1)
    elif kind == "gaussian_bump":
        # the constructor stores the widths squared (constraint_gaussian_bump.hpp)
        A, a, b = conf["A"], conf["a"] ** 2, conf["b"] ** 2
        f = np.exp(-x * x / a - y * y / b)
        g = A * f - z
        G = np.stack([-2 * A * x * f / a, -2 * A * y * f / b, -np.ones_like(z)], 1)
    elif kind == "tetrahedron":
        p = np.stack([x, y, z], 1)
        g = tetra_value(p, conf["scale"], conf["value"])
        G = tetra_gradient(p, conf["scale"])
    else:
        g = gyroid_value(x, y, z, box)
        G = gyroid_gradient(x, y, z, box)
    return g, G / np.linalg.norm(G, axis=1)[:, None]


@pytest.mark.parametrize("kind,shape,conf,box,periodic", IMPLICIT_CASES)
def test_implicit_surfaces_project_onto_their_surface(kind, shape, conf, box, periodic):
    # peanut, hourglass, Gaussian bump and gyroid have no enforce of their own:
    # Constraint::enforce's SHAKE projection (constraint.cpp:40-87) along their
    # gradients brings every particle to g = 0 within tol; directors unit and
    # tangent to the normalised gradient, which is also the stored normal
    parts = surface_disks(kind, 300, seed=6, **shape)
    o = OracleSystem(300)
    drive(o, parts, box, periodic=periodic, constraint=(kind, {k: repr(v) for k, v in conf.items()}))
    x, y, z = o.download("x"), o.download("y"), o.download("z")
    n = np.stack([o.download("nx"), o.download("ny"), o.download("nz")], 1)
    g, N = implicit_np(kind, conf, box, x, y, z)
    assert np.abs(g).max() <= 1e-6
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-14)
    assert np.abs(np.sum(n * N, 1)).max() <= 1e-6
    NN = np.stack([o.download("Nx"), o.download("Ny"), o.download("Nz")], 1)
    np.testing.assert_allclose(NN, N, atol=1e-12)


def test_implicit_surface_parameters_checked_like_the_reference():
    from samos_b200.plugins import PluginError, resolve_constraint
    with pytest.raises(PluginError):
        resolve_constraint("peanut", {})  # defaults a 10, b 8 (constraint_peanut.hpp:62-88)
    with pytest.raises(PluginError):
        resolve_constraint("peanut", {"a": "5", "b": "5"})
    with pytest.raises(PluginError):
        resolve_constraint("hourglass", {"R": "3", "A": "4"})
    kind, p = resolve_constraint("hourglass", {"R": "0.5"})  # A defaults to 1, unchecked
    assert p[0] == 0.5 and p[7] == 1.0 and p[8] == 1.0
    kind, p = resolve_constraint("gaussian_bump", {"A": "2", "a": "3", "b": "4"})
    assert (p[0], p[7], p[8]) == (2.0, 9.0, 16.0)  # widths squared (constraint_gaussian_bump.hpp)
    o = OracleSystem(4)
    with pytest.raises(ValueError):
        o.add_constraint(E.CONSTRAINT["peanut"], [5.0, 0, 100, 1e-6, 1, 1000, 10, 4.0, 0.0])


def test_slab_and_walls_reflect_like_the_reference():
    # ConstraintSlab::enforce (constraint_slab.cpp:35-61): z clamped into
    # [z_lo, z_hi] with vz and nz reversed; ConstraintPlaneWalls::enforce
    # (constraint_plane_walls.cpp:38-70): z = 0, walls at x = +-l reverse vx,
    # and l beyond the box is moved to the box edge (constraint_plane_walls.hpp:64-71)
    parts = dict(x=np.array([0.0, 1.0, 2.0]), y=np.zeros(3), z=np.array([-3.0, 0.5, 4.0]),
                 vx=np.array([1.0, 2.0, 3.0]), vy=np.zeros(3), vz=np.array([0.5, 0.5, 0.5]),
                 nx=np.array([0.6, 0.6, 0.6]), ny=np.zeros(3), nz=np.array([0.8, 0.8, 0.8]), radius=np.ones(3))
    o = OracleSystem(3)
    drive(o, parts, (20.0, 20.0, 20.0), periodic=False, constraint=("slab", {"z_lo": "-1.0", "z_hi": "2.0"}))
    np.testing.assert_array_equal(o.download("z"), [-1.0, 0.5, 2.0])
    np.testing.assert_array_equal(o.download("vz"), [-0.5, 0.5, -0.5])
    np.testing.assert_array_equal(o.download("nz"), [-0.8, 0.8, -0.8])
    parts2 = dict(parts, x=np.array([-9.0, 1.0, 9.5]))
    o = OracleSystem(3)
    drive(o, parts2, (20.0, 20.0, 20.0), periodic=False, constraint=("walls", {"l": "8.0"}))
    np.testing.assert_array_equal(o.download("x"), [-8.0, 1.0, 8.0])
    np.testing.assert_array_equal(o.download("vx"), [-1.0, 2.0, -3.0])
    np.testing.assert_array_equal(o.download("z"), [0.0, 0.0, 0.0])
    o = OracleSystem(3)
    drive(o, parts2, (16.0, 16.0, 20.0), periodic=False, constraint=("walls", {"l": "12.0"}))
    np.testing.assert_array_equal(o.download("x"), [-8.0, 1.0, 8.0])  # l = xhi = 8


def test_grouped_integrator_moves_its_group_only():
    # IntegratorBrownian over its group (integrator_brownian.cpp:50-121): the
    # other particles keep their positions when nothing else integrates them
    n = 600
    parts, L = plane_disks(n, 0.5, seed=44)
    parts["type"] = np.where(np.arange(n) % 3 == 0, 2, 1)
    o = OracleSystem(n, 2)
    sim = drive(o, parts, (L, L, 10.0), nlist=(2.4, 0.3), pairs=[("soft", {"k": "10"})], dt=1e-3, ntypes=2)
    sim.group("active", {"type": "2"})
    sim.integrator("brownian", {"group": "active", "v0": "1.0", "nu": "0.1", "seed": "3"})
    x0, y0 = o.download("x").copy(), o.download("y").copy()
    sim.run(50)
    moved = (o.download("x") != x0) | (o.download("y") != y0)
    assert np.array_equal(moved, parts["type"] == 2)
    with pytest.raises(Exception):
        sim.group("active", {"type": "1"})


@pytest.mark.parametrize("kind,shape,box,events", [
    # rescale_steps 40, freq 10, run(40) = steps 0..40: the sphere rescales at
    # 0, 10, 20, 30 (step < 40, constraint_sphere.cpp:92), the cylinder at 40
    # as well (step <= 40, constraint_cylinder.cpp:84), the torus never
    # (Constraint::rescale is a no-op, constraint.hpp:144)
    ("sphere", None, None, 4),
    ("cylinder", {"r": 10.0, "Lz": 40.0}, (40.0, 40.0, 40.0), 5),
    ("torus", {"c": 12.0, "a": 5.0}, (50.0, 50.0, 50.0), 0),
])
def test_constraint_rescale_steps_per_kind(kind, shape, box, events):
    if kind == "sphere":
        parts, R = sphere_disks(200, seed=9)
        conf, box, size = {"r": repr(R)}, (2 * R + 20,) * 3, R
    else:
        parts = surface_disks(kind, 200, seed=9, **shape)
        conf = {k: repr(v) for k, v in shape.items() if k != "Lz"}
        size = shape.get("r", shape.get("a"))
    conf.update(rescale="1.2", rescale_steps="40", rescale_freq="10")
    o = OracleSystem(200)
    sim = drive(o, parts, box, periodic=(kind == "cylinder"), constraint=(kind, conf),
                integrators=[("brownian", {"v0": "0", "nu": "0", "seed": "1"})], dt=1e-3)
    sim.run(40)
    x, y, z = o.download("x"), o.download("y"), o.download("z")
    f = 1.2 ** (10 / 40)
    if kind == "sphere":
        np.testing.assert_allclose(np.sqrt(x * x + y * y + z * z), size * f ** events, rtol=1e-13)
    elif kind == "cylinder":
        np.testing.assert_allclose(np.hypot(x, y), size * f ** events, rtol=1e-13)
    else:
        g = (shape["c"] - np.hypot(x, y)) ** 2 + z ** 2 - shape["a"] ** 2
        assert np.abs(g).max() <= 1e-6


def test_plane_rescale_scales_the_box_and_positions():
    # ConstraintPlane::rescale (constraint_plane.cpp:168-188) with Box::rescale
    # (box.hpp:72-77): at step 0 the box and every coordinate scale together
    parts, L = plane_disks(100, 0.3, seed=4)
    o = OracleSystem(100)
    sim = drive(o, parts, (L, L, 10.0), constraint=("plane", {"rescale": "2.0", "rescale_steps": "10",
                                                              "rescale_freq": "10"}),
                integrators=[("brownian", {"v0": "0", "nu": "0", "seed": "1"})], dt=1e-3)
    x0 = o.download("x").copy()
    sim.run(0)
    np.testing.assert_allclose(o.download("x"), 2.0 * x0, rtol=1e-15)
