"""Conf and particle files that replay the reference's example runs
(tests/golden/ref_*.npz) through the drop-in binary `samos-gpu`.

The particle file carries the state the reference read, every double with
17 significant digits (read back exactly); the conf file carries the
example's hot-path commands followed by a `dump type=full` of the end state.
"""
from __future__ import annotations

import glob
import os

import numpy as np

from ref_fixtures import decode

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(os.path.dirname(HERE), "samos_b200", "samos-gpu")
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))
GOLDEN_IDS = [os.path.basename(p)[4:-4] for p in GOLDEN]
COLUMNS = ("type", "radius", "x", "y", "z", "vx", "vy", "vz", "nx", "ny", "nz", "omega", "ix", "iy", "iz", "mass")
INTS = ("type", "ix", "iy", "iz")


def block(params) -> str:
    items = [k if v in ("", None) else f"{k} = {v}" for k, v in params.items()]
    return "{ " + "; ".join(items) + " }"


def conf_text(z) -> str:
    lx, ly, lz = (float(v) for v in z["box"])
    kind = "periodic" if int(z["periodic"]) else "fixed"
    lines = ["messages msg.txt", f"box {kind} {{ lx = {lx!r};  ly = {ly!r};  lz = {lz!r} }}", "input p.dat"]
    for cmd in decode(str(z["commands"])):
        op, args = cmd[0], cmd[1:]
        if op == "nlist":
            lines.append(f"nlist {block(args[0])}")
        elif op == "timestep":
            lines.append(f"timestep {args[0]!r}")
        elif op == "run":
            n = int(args[0])
            # `run n` takes n + 1 steps; the state after them is dumped at the
            # top of the next run loop (samos.cpp:895-896), that of `run 0`
            lines.append(f"dump final {{ type = full; start = {n + 1}; freq = {n + 1}; multi; id; coordinate; "
                         f"velocity; director; image_flags; header }}")
            lines.append(f"run {n}")
            lines.append("run 0")
        else:
            lines.append(f"{op} {args[0]} {block(args[1])}")
    return "\n".join(lines) + "\n"


def particle_text(z) -> str:
    n = len(z["in_x"])
    data = [z["in_" + c] for c in COLUMNS]
    out = ["keys: id " + " ".join(COLUMNS)]
    for i in range(n):
        vals = [str(int(a[i])) if c in INTS else repr(float(a[i])) for c, a in zip(COLUMNS, data)]
        out.append(f"{i} " + " ".join(vals))
    return "\n".join(out) + "\n"


def write_case(directory, path):
    z = np.load(path)
    with open(os.path.join(directory, "p.dat"), "w") as f:
        f.write(particle_text(z))
    with open(os.path.join(directory, "run.conf"), "w") as f:
        f.write(conf_text(z))
    return z


def read_full_dump(path):
    """Columns id, x y z, vx vy vz, nx ny nz, ix iy iz, ordered by id."""
    rows = [l.split() for l in open(path) if l.strip() and not l.startswith("#")]
    a = np.array([[float(v) for v in r] for r in rows])
    ids = a[:, 0].astype(int)
    out = {}
    for c, f in enumerate(("x", "y", "z", "vx", "vy", "vz", "nx", "ny", "nz", "ix", "iy", "iz"), start=1):
        v = np.empty(len(ids))
        v[ids] = a[:, c]
        out[f] = v
    return out
