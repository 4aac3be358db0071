"""Seeded synthetic inputs shaped like the benchmark configurations, and a
helper that drives the same conf-level command sequence through any backend
(the GPU engine or the CPU oracle)."""
from __future__ import annotations

import numpy as np

from samos_b200.plugins import Simulation


def plane_disks(n, phi, rmin=0.9, rmax=1.1, seed=1, bidisperse=None):
    """n disks uniform in a square periodic box at packing fraction phi
    (overlaps allowed), uniform random polar directions in the plane."""
    rng = np.random.default_rng(seed)
    if bidisperse is None:
        r = rng.uniform(rmin, rmax, n)
    else:
        r = np.where(np.arange(n) % 2 == 0, bidisperse[0], bidisperse[1]).astype(float)
        rng.shuffle(r)
    L = float(np.sqrt(np.sum(np.pi * r * r) / phi))
    th = rng.uniform(0.0, 2.0 * np.pi, n)
    parts = dict(x=rng.uniform(-L / 2, L / 2, n), y=rng.uniform(-L / 2, L / 2, n), z=np.zeros(n),
                 vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n),
                 nx=np.cos(th), ny=np.sin(th), nz=np.zeros(n), radius=r)
    return parts, L


def sphere_disks(n, R=None, seed=1, radius=1.0):
    """n particles uniform on a sphere (z ~ U[-R,R], phi ~ U[0,2pi)) with
    random tangent directors; R from n*pi*r^2 = 4 pi R^2 by default."""
    rng = np.random.default_rng(seed)
    if R is None:
        R = float(np.sqrt(n * radius * radius / 4.0))
    z = rng.uniform(-R, R, n)
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    s = np.sqrt(np.maximum(R * R - z * z, 0.0))
    x, y = s * np.cos(ph), s * np.sin(ph)
    pos = np.stack([x, y, z], 1)
    Nn = pos / R
    a = rng.normal(size=(n, 3))
    t = a - np.sum(a * Nn, 1)[:, None] * Nn
    t /= np.linalg.norm(t, axis=1)[:, None]
    parts = dict(x=x, y=y, z=z, vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n),
                 nx=t[:, 0], ny=t[:, 1], nz=t[:, 2], radius=np.full(n, radius))
    return parts, R


def drive(backend, parts, box, periodic=True, nlist=(2.4, 0.3), constraint=("plane", {}),
          pairs=(), aligns=(), externals=(), dt=1e-3, integrators=(), ntypes=1,
          pair_params=(), align_params=()):
    sim = Simulation(backend, ntypes=ntypes)
    sim.box(*box, periodic)
    sim.input(**parts)
    if nlist is not None:
        sim.nlist(*nlist)
    if constraint is not None:
        sim.constraint(*constraint)
    for name, p in pairs:
        sim.pair_potential(name, dict(p))
    for name, p in pair_params:
        sim.pair_param(name, dict(p))
    for name, p in aligns:
        sim.pair_align(name, dict(p))
    for name, p in align_params:
        sim.align_param(name, dict(p))
    for name, p in externals:
        sim.external(name, dict(p))
    sim.timestep(dt)
    for name, p in integrators:
        sim.integrator(name, dict(p))
    return sim


def gyroid_value(x, y, z, box):
    lx, ly, lz = box
    return (np.cos(2 * np.pi * z / lz) * np.sin(2 * np.pi * x / lx) + np.cos(2 * np.pi * x / lx) * np.sin(2 * np.pi * y / ly)
            + np.cos(2 * np.pi * y / ly) * np.sin(2 * np.pi * z / lz))


def gyroid_gradient(x, y, z, box):
    lx, ly, lz = box
    X, Y, Z = 2 * np.pi * x / lx, 2 * np.pi * y / ly, 2 * np.pi * z / lz
    return np.stack([2 * np.pi * (np.cos(X) * np.cos(Z) - np.sin(X) * np.sin(Y)) / lx,
                     2 * np.pi * (np.cos(X) * np.cos(Y) - np.sin(Y) * np.sin(Z)) / ly,
                     2 * np.pi * (np.cos(Y) * np.cos(Z) - np.sin(X) * np.sin(Z)) / lz], -1)


TETRA = np.array([[1.0, 0.0, -0.7071067811865475], [-1.0, 0.0, -0.7071067811865475],
                  [0.0, 1.0, 0.7071067811865475], [0.0, -1.0, 0.7071067811865475]])


def tetra_value(p, scale, value):
    """sum over the four scaled charges of 1/|r - a_i|, minus the level."""
    return sum(1.0 / np.linalg.norm(p - scale * a, axis=-1) for a in TETRA) - value


def tetra_gradient(p, scale):
    g = 0.0
    for a in TETRA:
        d = p - scale * a
        g = g + d / np.linalg.norm(d, axis=-1)[..., None] ** 3
    return -g


def surface_disks(kind, n, seed=1, **shape):
    """n particles scattered near a cylinder (r), torus (c, a), ellipsoid
    (a, b, c), peanut (a, b), hourglass (R, A, n_nodes, Lz), Gaussian bump
    (A, a, b, L) or gyroid (box) around the origin, with random directors; the
    constraint projects them on the surface when it is added."""
    rng = np.random.default_rng(seed)
    u, v = rng.uniform(0.0, 2.0 * np.pi, n), rng.uniform(0.0, 2.0 * np.pi, n)
    if kind == "peanut":  # rays from the origin to the surface (b > a: one root in r^2)
        a, b = shape["a"], shape["b"]
        w = rng.normal(size=(3, n))
        w /= np.linalg.norm(w, axis=0)
        c = w[0] ** 2 - w[1] ** 2 - w[2] ** 2
        r = np.sqrt(a * a * c + np.sqrt(a ** 4 * c * c - a ** 4 + b ** 4))
        x, y, z = r * w[0], r * w[1], r * w[2]
    elif kind == "hourglass":
        R, A, nn, Lz = shape["R"], shape["A"], shape["n_nodes"], shape["Lz"]
        z = rng.uniform(-0.45 * Lz, 0.45 * Lz, n)
        rho = R + A * np.sin(2 * np.pi * nn * z / Lz)
        x, y = rho * np.cos(u), rho * np.sin(u)
    elif kind == "gaussian_bump":
        A, a, b, L = shape["A"], shape["a"], shape["b"], shape["L"]
        x, y = rng.uniform(-0.45 * L, 0.45 * L, n), rng.uniform(-0.45 * L, 0.45 * L, n)
        z = A * np.exp(-x * x / (a * a) - y * y / (b * b))
    elif kind == "tetrahedron":  # rays from the origin, bisected to the level (inside it above, outside below)
        s, val = shape["scale"], shape["value"]
        w = rng.normal(size=(n, 3))
        w /= np.linalg.norm(w, axis=1)[:, None]
        lo, hi = np.zeros(n), np.full(n, 20.0 * s)
        for _ in range(80):
            mid = 0.5 * (lo + hi)
            inside = tetra_value(mid[:, None] * w, s, val) > 0.0
            lo, hi = np.where(inside, mid, lo), np.where(inside, hi, mid)
        x, y, z = (hi[:, None] * w).T
    elif kind == "gyroid":  # random points pulled onto the surface by Newton steps along the gradient
        box = shape["box"]
        p = np.stack([rng.uniform(-h / 2, h / 2, n) for h in box], -1)
        for _ in range(30):
            g = gyroid_value(p[:, 0], p[:, 1], p[:, 2], box)
            G = gyroid_gradient(p[:, 0], p[:, 1], p[:, 2], box)
            p -= (g / np.maximum(np.sum(G * G, -1), 1e-12))[:, None] * G
        x, y, z = p[:, 0], p[:, 1], p[:, 2]
    if kind in ("peanut", "hourglass", "gaussian_bump", "gyroid", "tetrahedron"):
        jitter = rng.normal(0.0, 0.02, (3, n))
        d = rng.normal(size=(3, n))
        d /= np.linalg.norm(d, axis=0)
        return dict(x=x + jitter[0], y=y + jitter[1], z=z + jitter[2], vx=np.zeros(n), vy=np.zeros(n),
                    vz=np.zeros(n), nx=d[0], ny=d[1], nz=d[2], radius=np.full(n, 1.0))
    if kind == "cylinder":
        r, Lz = shape["r"], shape["Lz"]
        x, y, z = r * np.cos(u), r * np.sin(u), rng.uniform(-Lz / 2, Lz / 2, n)
    elif kind == "torus":
        c, a = shape["c"], shape["a"]
        x, y, z = (c + a * np.cos(v)) * np.cos(u), (c + a * np.cos(v)) * np.sin(u), a * np.sin(v)
    else:
        a, b, c = shape["a"], shape["b"], shape["c"]
        w = rng.uniform(-1.0, 1.0, n)
        s = np.sqrt(1.0 - w * w)
        x, y, z = a * s * np.cos(u), b * s * np.sin(u), c * w
    jitter = rng.normal(0.0, 0.05, (3, n))
    d = rng.normal(size=(3, n))
    d /= np.linalg.norm(d, axis=0)
    return dict(x=x + jitter[0], y=y + jitter[1], z=z + jitter[2], vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n),
                nx=d[0], ny=d[1], nz=d[2], radius=np.full(n, 1.0))
