"""The CPU oracle pinned to the reference's own code.

oracle/build_ref.sh compiles SAMoS's unmodified hot-path sources (system,
cell and neighbour lists, the soft / LJ / Morse / Gaussian potentials, the
polar / nematic / Vicsek aligners, self-propulsion, every constraint of the
path, the brownian family, Langevin, NVE, FIRE and Vicsek integrators) into
oracle/_ref/libsamos_ref.so, with stand-ins only for Boost's string helpers,
GSL's generator (which then draws the shared noise stream) and CGAL's type
names.  Both are built strict-IEEE by gcc on the same host, so the bar is
bit-identical states:

* every scenario of tests/pin_scenarios.py, end state after its run;
* neighbour lists in the reference's storage order (cell path, N^2 path, a
  two-cell dimension with the duplicated stencil, a sphere);
* one force / torque / energy evaluation of every potential and aligner;
* the reference's example configurations, from the fixtures that
  tests/golden/make_ref_golden.py made with the reference build, which hold
  without the reference tree;
* the C++ host's particle-file reader against the reference's reader.

The live comparisons skip when oracle/_ref is not built.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

from oracle import refsrc
from oracle.oracle import OracleSystem
from pin_scenarios import NAMES, REFERENCE_UNDEFINED_RUNS, compared_fields, run_backend, run_reference
from ref_fixtures import CASES, INPUT_FIELDS, apply, decode, ntypes_of
from samos_b200.plugins import Simulation
from scenarios import drive, plane_disks, sphere_disks

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))
CONFIGURATIONS = "/root/reference/configurations"

needs_ref = pytest.mark.skipif(not refsrc.available(), reason="reference-source build (oracle/_ref) not built")


@needs_ref
@pytest.mark.parametrize("name", [n for n in NAMES if n not in REFERENCE_UNDEFINED_RUNS])
def test_oracle_reproduces_the_reference_bit_for_bit(name):
    r = run_reference(name)
    o = run_backend(OracleSystem, name)
    for f in compared_fields(name):
        a, b = r.download(f), o.download(f)
        assert np.array_equal(a, b), f"{name}: {f} differs by {np.max(np.abs(a.astype(float) - b.astype(float)))}"
    assert np.all(np.isfinite(r.download("x")))


def _lists(parts, box, periodic=True, nlist=(2.4, 0.3), constraint=("plane", {})):
    from oracle.refsrc import drive_ref
    r = drive_ref(parts, box, periodic=periodic, nlist=nlist, constraint=constraint)
    o = OracleSystem(len(parts["x"]))
    drive(o, parts, box, periodic=periodic, nlist=nlist, constraint=constraint)
    return r, o


@needs_ref
@pytest.mark.parametrize("case", ["cell", "nsq", "two_cells", "sphere"])
def test_neighbour_lists_in_the_reference_storage_order(case):
    if case == "sphere":
        parts, R = sphere_disks(1500, seed=3)
        b = 2 * R + 6.0
        r, o = _lists(parts, (b, b, b), periodic=False, constraint=("sphere", {"r": repr(R)}))
    else:
        n, phi = {"cell": (2000, 0.6), "nsq": (40, 0.5), "two_cells": (90, 0.5)}[case]
        parts, L = plane_disks(n, phi, seed=4)
        box = {"cell": (L, L, 10.0), "nsq": (L, L, 10.0), "two_cells": (5.6, 100.0, 10.0)}[case]
        if case == "two_cells":  # 5.6 / 2.7 -> exactly two cells along x (cell_list.cpp:52-63)
            parts["x"] = np.random.default_rng(5).uniform(-2.8, 2.8, n)
            parts["y"] = np.random.default_rng(6).uniform(-50.0, 50.0, n)
        r, o = _lists(parts, box)
    ri, rj = r.pairs()
    oi, oj = o.pairs()
    assert len(ri) > 0
    np.testing.assert_array_equal(ri, oi)
    np.testing.assert_array_equal(rj, oj)


@needs_ref
@pytest.mark.parametrize("pot,align", [
    (("soft", {"k": "10", "use_particle_radii": ""}), ("polar", {"J": "0.3"})),
    (("soft", {"k": "10", "a": "2.2"}), ("nematic", {"J": "0.5"})),
    (("soft", {"k": "10", "use_particle_radii": ""}), ("vicsek", {"rcut": "2.0"})),
    (("lj", {"epsilon": "1", "sigma": "1.9", "rcut": "2.5", "shifted": ""}), ("polar", {"J": "0.3"})),
    (("morse", {"D": "1", "a": "2", "re": "2", "rcut": "2.5", "use_particle_radii": ""}), ("polar", {"J": "0.3"})),
    (("gaussian", {"A": "2", "B": "-1", "alpha": "1", "beta": "3", "rA": "0", "rB": "1.5", "rcut": "2.5",
                   "shifted": ""}), ("nematic", {"J": "0.2"})),
])
def test_forces_torques_and_energies_bit_for_bit(pot, align):
    from oracle.refsrc import drive_ref
    parts, L = plane_disks(1500, 0.55, seed=9)
    rng = np.random.default_rng(9)
    parts["vx"], parts["vy"] = rng.normal(size=1500), rng.normal(size=1500)
    kw = dict(nlist=(2.5, 0.3), pairs=[pot], aligns=[align], externals=[("self_propulsion", {"alpha": "0.4"})])
    r = drive_ref(parts, (L, L, 10.0), **kw)
    r.compute()
    o = OracleSystem(1500)
    sim = drive(o, parts, (L, L, 10.0), **kw)
    sim.commit()
    o.compute(0.0)
    for f in ("fx", "fy", "fz", "tau_x", "tau_y", "tau_z"):
        np.testing.assert_array_equal(r.download(f), o.download(f), err_msg=f)
    assert r.energy(0, pot[0]) == o.energy(0, 0)
    if align[0] != "vicsek":
        assert r.energy(1, align[0]) == o.energy(1, 0)


def _golden(path):
    z = np.load(path)
    return z, decode(str(z["commands"])), str(z["fields"]).split()


def _inputs(z):
    parts = {f: z["in_" + f] for f in INPUT_FIELDS}
    parts["type"] = parts["type"].astype(np.int32)
    for f in ("ix", "iy", "iz"):
        parts[f] = parts[f].astype(np.int32)
    return parts


def run_golden_on(backend_cls, path):
    """A golden fixture's input, box and commands on the oracle or the GPU engine."""
    z, commands, fields = _golden(path)
    parts = _inputs(z)
    n, ntypes = len(parts["x"]), ntypes_of(parts["type"])
    b = backend_cls(n, ntypes)
    sim = Simulation(b, ntypes=ntypes)
    lx, ly, lz = (float(v) for v in z["box"])
    sim.box(lx, ly, lz, bool(int(z["periodic"])))
    sim.input(**parts)
    apply(sim, commands)
    return z, b, fields


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[4:-4] for p in GOLDEN])
def test_oracle_reproduces_the_reference_example_runs(path):
    z, o, fields = run_golden_on(OracleSystem, path)
    for f in fields + ["ix", "iy"]:
        np.testing.assert_array_equal(o.download(f), z["out_" + f], err_msg=f)


def test_every_example_case_has_a_fixture():
    assert sorted(os.path.basename(p)[4:-4] for p in GOLDEN) == sorted(CASES)


@pytest.mark.skipif(not os.path.isdir(CONFIGURATIONS), reason="the reference's configurations are not here")
@pytest.mark.parametrize("case", sorted(CASES))
def test_host_reader_reads_the_examples_like_the_reference(case):
    from samos_b200 import build
    binary = os.path.join(os.path.dirname(HERE), "samos_b200", "samos-gpu")
    if not os.path.exists(binary):
        build.build_all()
    path = os.path.join(CONFIGURATIONS, CASES[case][0])
    out = subprocess.run([binary, "--read-particles", path], capture_output=True, text=True, check=True).stdout
    rows = out.splitlines()
    cols = rows[0].split()
    data = np.array([[float(v) for v in r.split()] for r in rows[1:]])
    z = np.load(os.path.join(HERE, "golden", f"ref_{case}.npz"))
    for f in INPUT_FIELDS:
        np.testing.assert_array_equal(data[:, cols.index(f)], z["in_" + f], err_msg=f)
