"""Batched ensembles: many independent systems in one engine handle.

``sphere_ensemble`` builds R active-Brownian sphere systems (soft repulsion +
polar alignment + brownian integrator on a sphere constraint) with their own
particle counts, radii, activities, couplings, noise strengths and seeds.
Every replica evolves exactly as it would as a single system: replicas share
kernel launches, never data, and each keeps its own noise counters,
neighbour-list rebuild history and reductions.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import engine as E
from .plugins import resolve_align, resolve_constraint, resolve_integrator, resolve_pair


@dataclass
class SphereReplica:
    parts: dict        # particle arrays (x, y, z, nx, ny, nz, radius, ...)
    R: float           # sphere radius
    v0: float
    J: float
    nu: float
    seed: int


def sphere_ensemble(reps: list[SphereReplica], k: float = 10.0, rcut: float = 2.4, pad: float = 0.3,
                    dt: float = 1e-3, margin: float = 6.0, engine: E.Engine | None = None) -> E.Engine:
    """One engine holding every replica; box side 2R + margin per replica (fixed box)."""
    n = [len(r.parts["x"]) for r in reps]
    eng = engine or E.Engine(n)
    for i, r in enumerate(reps):
        side = 2.0 * r.R + margin
        eng.set_box(side, side, side, periodic=False, replica=i)
        for f, v in r.parts.items():
            eng.upload(f, v, replica=i)
    eng.set_nlist(rcut, pad)
    kind, cp = resolve_constraint("sphere", {"r": repr(reps[0].R)})
    eng.add_constraint_per_replica(kind, cp, [r.R for r in reps])
    pair = resolve_pair("soft", {"k": repr(k), "use_particle_radii": ""}, 1, rcut)
    eng.add_pair(pair.kind, pair.glob, pair.table.reshape(-1), pair.use_radii, False, False, False,
                 pair.phase_value)
    al = resolve_align("polar", {"J": repr(reps[0].J)}, 1, rcut)
    eng.add_align(al.kind, al.J, al.rcut, al.table.reshape(-1), False)
    ikind, ip, temp = resolve_integrator("brownian", {"v0": repr(reps[0].v0), "nu": repr(reps[0].nu),
                                                      "seed": str(reps[0].seed)}, dt)
    eng.set_timestep(dt)
    eng.add_integrator(ikind, ip, temp)
    for i, r in enumerate(reps):
        eng.set_replica_param(i, 1, 0, 0, r.J)
        eng.set_replica_param(i, 4, 0, 1, r.v0)
        eng.set_replica_param(i, 4, 0, 2, r.nu)
        eng.set_replica_param(i, 4, 0, 5, float(r.seed))
    return eng


def quench_disks(n: int, phi: float, seed: int, radii=(1.0, 1.4)):
    """Bidisperse disks (50:50) at uniform random positions in a square periodic
    box of packing fraction phi -- the quench that FIRE relaxes."""
    rng = np.random.default_rng(seed)
    r = np.where(np.arange(n) % 2 == 0, radii[0], radii[1]).astype(np.float64)
    rng.shuffle(r)
    L = float(np.sqrt(np.sum(np.pi * r * r) / phi))
    th = rng.uniform(0.0, 2.0 * np.pi, n)
    parts = dict(x=rng.uniform(-L / 2, L / 2, n), y=rng.uniform(-L / 2, L / 2, n), z=np.zeros(n),
                 vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n),
                 nx=np.cos(th), ny=np.sin(th), nz=np.zeros(n), radius=r)
    return parts, L


def plane_fire_ensemble(insts, k: float = 1.0, rcut: float = 2.8, pad: float = 0.3, dt: float = 0.01,
                        dt_max: float = 0.2, fmax: float = 1e-10, device: int | None = None) -> E.Engine:
    """FIRE minimisation of many periodic-plane systems (soft repulsion on the
    particle radii) in one engine; insts = [(parts, L), ...]."""
    eng = E.Engine([len(p["x"]) for p, _ in insts], device=device)
    for i, (parts, L) in enumerate(insts):
        eng.set_box(L, L, 10.0, periodic=True, replica=i)
        for f, v in parts.items():
            eng.upload(f, v, replica=i)
    eng.set_nlist(rcut, pad)
    kind, cp = resolve_constraint("plane", {})
    eng.add_constraint(kind, cp)
    pair = resolve_pair("soft", {"k": repr(k), "use_particle_radii": ""}, 1, rcut)
    eng.add_pair(pair.kind, pair.glob, pair.table.reshape(-1), pair.use_radii, False, False, False,
                 pair.phase_value)
    eng.set_timestep(dt)
    ikind, ip, temp = resolve_integrator("fire", {"dt_max": repr(dt_max), "fmax_tolerance": repr(fmax)}, dt)
    eng.add_integrator(ikind, ip, temp)
    return eng
