"""The reference's own example configurations (configurations/<name>/ in the
SAMoS tree) as command sequences for the parity tests.

Each case is one example's particle file and the hot-path commands of its
.conf, shortened to a few hundred steps; dumps, logs and `messages` are left
out.  Where an example relaxes with `integrator nve { limit = ... }` before
its active run, that stage is its own case whose compared fields exclude the
directors and omega: with `limit` and no `angle_limit` the reference reads
the uninitialised m_theta_limit (integrator_nve.hpp:59-75, integrator_nve.cpp
:135-137), so its director update is undefined.  The active stage then
starts from the particle file itself.

tests/golden/make_ref_golden.py runs every case through the reference-source
build and stores the state as the reference read it and the state after the
run: tests/golden/ref_<case>.npz.
"""
from __future__ import annotations

import json

import numpy as np

P2 = ["x", "y", "vx", "vy", "nx", "ny"]
P3 = ["x", "y", "z", "vx", "vy", "vz", "nx", "ny", "nz"]

# case -> (particle file under configurations/, box (lx, ly, lz, periodic), commands, compared fields)
CASES = {
    "soft_on_plane_nve": (
        "soft_on_plane/plane.dat", (100.0, 100.0, 10.0, True),
        [("nlist", {"rcut": "2.5", "pad": "0.5"}), ("constraint", "plane", {}),
         ("pair_potential", "soft", {"k": "1.0"}), ("pair_align", "polar", {"J": "1.0"}), ("timestep", 0.001),
         ("integrator", "nve", {"limit": "0.0001"}), ("run", 300)],
        ["x", "y", "vx", "vy"]),
    "soft_on_plane_active": (
        "soft_on_plane/plane.dat", (100.0, 100.0, 10.0, True),
        [("nlist", {"rcut": "2.5", "pad": "0.5"}), ("constraint", "plane", {}),
         ("pair_potential", "soft", {"k": "1.0"}), ("pair_align", "polar", {"J": "1.0"}),
         ("external", "self_propulsion", {"alpha": "1.0"}), ("timestep", 0.01),
         ("integrator", "brownian_pos", {"seed": "1", "mu": "1.0", "group": "all"}),
         ("integrator", "brownian_align", {"seed": "1", "mur": "1.0", "nu": "0.1", "group": "all"}), ("run", 500)],
        P2),
    "soft_on_sphere_nve": (
        "soft_on_sphere/sphere.dat", (30.0, 30.0, 30.0, False),
        [("nlist", {"rcut": "2.4", "pad": "0.5"}), ("constraint", "sphere", {"r": "10"}),
         ("pair_potential", "soft", {"k": "10.0", "a": "1.0"}), ("pair_align", "polar", {"J": "1.0"}),
         ("timestep", 0.01), ("integrator", "nve", {"limit": "0.0001"}), ("run", 300)],
        ["x", "y", "z", "vx", "vy", "vz"]),
    "soft_on_sphere_active": (
        "soft_on_sphere/sphere.dat", (30.0, 30.0, 30.0, False),
        [("nlist", {"rcut": "2.4", "pad": "0.5"}), ("constraint", "sphere", {"r": "10"}),
         ("pair_potential", "soft", {"k": "10.0", "a": "1.0"}), ("pair_align", "polar", {"J": "1.0"}),
         ("external", "self_propulsion", {"alpha": "1.0"}), ("timestep", 0.01),
         ("integrator", "brownian_pos", {"seed": "0", "mu": "1.0", "temperature_control": "constant",
                                         "min_val": "0.1"}),
         ("integrator", "brownian_align", {"seed": "0", "nu": "0.01"}), ("run", 500)],
        P3),
    "lj_langevin": (
        "lj_langevin/particles.dat", (100.0, 100.0, 10.0, True),
        [("nlist", {"rcut": "3.0", "pad": "0.5"}), ("constraint", "plane", {}),
         ("pair_potential", "lj", {"epsilon": "1.0", "sigma": "1.0", "rcut": "2.5", "shifted": ""}),
         ("integrator", "langevin", {"dt": "0.001", "seed": "1", "gamma": "1.0", "min_val": "2.4",
                                     "group": "all"}), ("run", 500)],
        ["x", "y", "vx", "vy"]),
    "vicsek_on_plane": (
        "vicsek_on_plane/plane.dat", (106.0, 106.0, 10.0, True),
        [("nlist", {"rcut": "1.5", "pad": "0.5"}), ("constraint", "plane", {}),
         ("pair_align", "vicsek", {"rcut": "1.0"}),
         ("integrator", "vicsek", {"dt": "0.01", "seed": "37", "eta": "1.0", "mu": "1.0", "v0": "0.5"}),
         ("run", 500)],
        ["x", "y", "vx", "vy"]),
    "vicsek_on_sphere": (
        "vicsek_on_sphere/sphere.dat", (30.0, 30.0, 30.0, False),
        [("nlist", {"rcut": "1.0", "pad": "0.5"}), ("constraint", "sphere", {"r": "10.0"}),
         ("pair_align", "vicsek", {"rcut": "1.0"}),
         ("integrator", "vicsek", {"dt": "0.001", "seed": "1", "mu": "1.0", "eta": "0.1", "v0": "1"}),
         ("run", 500)],
        ["x", "y", "z", "vx", "vy", "vz"]),
    "soft_on_bump_active": (
        "gaussian_bump/bump.dat", (50.0, 50.0, 50.0, True),
        [("nlist", {"rcut": "2.5", "pad": "0.5"}), ("constraint", "gaussian_bump", {"A": "3.0", "a": "8.0", "b": "8.0"}),
         ("pair_potential", "soft", {"k": "0.0"}), ("pair_align", "polar", {"J": "1.0"}),
         ("external", "self_propulsion", {"alpha": "1.0"}), ("timestep", 0.01),
         ("integrator", "brownian_pos", {"seed": "0", "mu": "1.0"}),
         ("integrator", "brownian_align", {"seed": "0", "nu": "0.01"}), ("run", 500)],
        P3),
    "soft_on_hourglass_active": (
        "soft_on_hourglass/hourglass.dat", (30.0, 30.0, 30.0, True),
        [("nlist", {"rcut": "2.4", "pad": "0.5"}), ("constraint", "hourglass", {"R": "10.0", "A": "2.0"}),
         ("pair_potential", "soft", {"k": "10.0"}), ("pair_align", "polar", {"J": "1.0"}),
         ("integrator", "brownian", {"dt": "0.001", "seed": "0", "nu": "0.002", "mu": "1.0", "v0": "1.0"}),
         ("run", 500)],
        P3),
    "two_component_plane_active": (
        "two_component_plane/plane.dat", (100.0, 100.0, 10.0, True),
        [("nlist", {"rcut": "2.5", "pad": "0.5"}), ("group", "passive", {"type": "1"}),
         ("group", "active", {"type": "2"}), ("constraint", "plane", {}), ("pair_potential", "soft", {"k": "1.0"}),
         ("pair_align", "polar", {"J": "1.0"}),
         ("align_param", "polar", {"type_1": "1", "type_2": "1", "J": "0.0"}),
         ("align_param", "polar", {"type_1": "1", "type_2": "2", "J": "0.0"}),
         ("align_param", "polar", {"type_1": "2", "type_2": "2", "J": "1.0"}),
         ("integrator", "brownian", {"group": "active", "dt": "0.001", "seed": "1", "nu": "0.001", "mu": "1.0",
                                     "v0": "0.5"}),
         ("integrator", "brownian", {"group": "passive", "dt": "0.001", "seed": "4", "nu": "0.00", "mu": "1.0",
                                     "v0": "0.0", "temperature_control": "constant", "min_val": "0.3",
                                     "max_val": "0.3", "steps": "1000"}),
         ("run", 500)],
        P2),
}

# particle fields the reference's reader fills (system.cpp:170-330), in the
# order the fixtures store them
INPUT_FIELDS = ("type", "radius", "x", "y", "z", "vx", "vy", "vz", "nx", "ny", "nz", "omega", "ix", "iy", "iz",
                "mass")


def ntypes_of(types) -> int:
    return int(np.max(types)) if len(types) else 1


def apply(sim, commands):
    """Runs the command list on a RefSimulation or a plugins.Simulation."""
    for cmd in commands:
        op, args = cmd[0], cmd[1:]
        if op == "nlist":
            sim.nlist(float(args[0]["rcut"]), float(args[0]["pad"]))
        elif op == "timestep":
            sim.timestep(args[0])
        elif op == "run":
            sim.run(args[0])
        else:
            getattr(sim, op)(args[0], dict(args[1]))


def encode(commands) -> str:
    return json.dumps(commands)


def decode(text: str):
    return [tuple(c) for c in json.loads(text)]
