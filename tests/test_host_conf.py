"""The C++ conf-file host (samos_b200/samos-gpu): the reference's command
syntax, plugin parameter handling and error behaviour (CPU, `--check` mode),
and on the GPU the same run through the host and through the Python
binding, bit for bit, including runs split by dumps and integrators added
and disabled between runs."""
import os
import subprocess

import numpy as np
import pytest

from samos_b200 import plugins as PL

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(os.path.dirname(HERE), "samos_b200", "samos-gpu")


def write_particles(path, parts, style="keys"):
    n = len(parts["x"])
    with open(path, "w") as f:
        if style == "keys":
            f.write("# written by the test\nkeys: id type radius x y z vx vy vz nx ny nz\n")
        elif style == "hash":
            f.write("# Total of %d particles\n# id  type radius  x   y   z   vx   vy   vz   nx   ny   nz  omega\n" % n)
        for i in range(n):
            row = [i, int(parts.get("type", np.ones(n, int))[i]), parts["radius"][i], parts["x"][i], parts["y"][i],
                   parts["z"][i], 0.0, 0.0, 0.0, parts["nx"][i], parts["ny"][i], parts["nz"][i]]
            if style != "keys":
                row.append(0.0)
            f.write(" ".join(repr(float(v)) if isinstance(v, (float, np.floating)) else str(v) for v in row) + "\n")


def plane_parts(n=400, L=40.0, seed=3):
    rng = np.random.default_rng(seed)
    th = rng.uniform(0, 2 * np.pi, n)
    return dict(x=rng.uniform(-L / 2, L / 2, n), y=rng.uniform(-L / 2, L / 2, n), z=np.zeros(n),
                nx=np.cos(th), ny=np.sin(th), nz=np.zeros(n), radius=rng.uniform(0.9, 1.1, n)), L


def run_host(conf_path, *flags):
    return subprocess.run([BIN, *flags, conf_path], capture_output=True, text=True, timeout=600)


def check(tmp_path, conf_text, parts=None, style="keys"):
    parts = parts or plane_parts()[0]
    write_particles(tmp_path / "p.dat", parts, style)
    (tmp_path / "c.conf").write_text(conf_text)
    return run_host(str(tmp_path / "c.conf"), "--check", "--quiet")


CONF = """# comment line
messages msg.txt
box periodic { lx = 40.0;  ly = 40.0;  lz = 10.0 }
input p.dat
nlist { rcut = 2.4; pad = 0.3 }
constraint plane { }
pair_potential soft { k = 10.0; use_particle_radii }
pair_align polar { J = 0.1 }
timestep 0.001
integrator brownian_pos { seed = 7; mu = 1.0 }
integrator brownian_align { seed = 8; nu = 0.1, mur = 1.0 }
run 10
"""


def parse_describe(out):
    rows = {}
    for line in out.splitlines():
        parts = line.split()
        rows.setdefault(parts[0], []).append(parts[1:])
    return rows


@pytest.fixture(scope="module", autouse=True)
def host_binary():
    if not os.path.exists(BIN):
        from samos_b200 import build
        build.build_all()
    assert os.path.exists(BIN)


def test_check_mode_resolves_like_the_python_plugins(tmp_path):
    r = check(tmp_path, CONF)
    assert r.returncode == 0, r.stderr
    rows = parse_describe(r.stdout)
    assert rows["particles"][0][:1] == ["400"]
    assert rows["nlist"][0] == ["2.4", "0.3"]
    pair = PL.resolve_pair("soft", {"k": "10.0", "use_particle_radii": ""}, 1, 2.4)
    assert [float(v) for v in rows["pair"][0][2:2 + 8]] == list(pair.glob)
    assert rows["align"][0] == ["polar", "0.1", "2.4"]
    # integrators in std::map key order: brownian_align_all before brownian_pos_all
    assert [r[0] for r in rows["integrator"]] == ["brownian_align_all", "brownian_pos_all"]
    _, p_align, _ = PL.resolve_integrator("brownian_align", {"seed": "8", "nu": "0.1", "mur": "1.0"}, 1e-3)
    assert [float(v) for v in rows["integrator"][0][2:]] == list(p_align[:12])
    assert rows["steps"][0] == ["11"]  # `run 10` is 11 steps


@pytest.mark.parametrize("bad,msg", [
    ("pair_potential soft { k = 10.0; kk = 2 }", 'Unknown parameter "kk"'),
    ("pair_potential coulomb { }", "Unknown pair potential coulomb"),
    ("integrator brownian { v0 = 1; foo }", 'Unknown parameter "foo"'),
    ("integrator nosuch { }", "not part of the GPU path"),
    ("box cubic { lx = 4 }", "Unknown box type"),
    ("pair_potential soft { k = 10.0; ", "Error parsing"),
    ("group g { type = 1 }", "not part of the GPU path"),
])
def test_errors_follow_the_reference(tmp_path, bad, msg):
    lines = CONF.splitlines()
    conf = "\n".join(lines[:9] + [bad] + lines[9:]) + "\n"
    r = check(tmp_path, conf)
    assert r.returncode == 1
    assert msg in r.stderr, r.stderr


def test_command_order_rules(tmp_path):
    r = check(tmp_path, "box periodic { lx = 40; ly = 40; lz = 10 }\ninput p.dat\ntimestep 0.001\n"
                        "integrator brownian { }\n")
    assert r.returncode == 1 and "Constraint not defined" in r.stderr
    r = check(tmp_path, "input p.dat\n")
    assert r.returncode == 1 and "Simulation box not defined" in r.stderr
    r = check(tmp_path, "box periodic { lx = 40; ly = 40; lz = 10 }\ninput p.dat\nconstraint plane {}\n"
                        "timestep 0.001\nintegrator brownian { }\nintegrator brownian { seed = 2 }\n")
    assert r.returncode == 1 and "already exists" in r.stderr
    r = check(tmp_path, CONF + "disable brownian_pos { }\nrun 5\n")
    assert r.returncode == 0, r.stderr
    assert [x[0] for x in parse_describe(r.stdout)["integrator"]] == ["brownian_align_all"]
    r = check(tmp_path, CONF + "disable nve { }\n")
    assert r.returncode == 1 and "non-existent integrator" in r.stderr


@pytest.mark.parametrize("line,kind", [
    ("constraint peanut { a = 8; b = 10 }", 6),
    ("constraint gyroid { }", 7),
    ("constraint hourglass { R = 10; A = 2; n = 2 }", 8),
    ("constraint gaussian_bump { A = 2; a = 3; b = 4 }", 9),
    ("constraint slab { z_lo = -1; z_hi = 1 }", 10),
    ("constraint walls { l = 15 }", 11),
    ("constraint tetrahedron { scale = 10; value = 0.3 }", 12),
])
def test_implicit_surface_constraints_parse(tmp_path, line, kind):
    r = check(tmp_path, CONF.replace("constraint plane { }", line))
    assert r.returncode == 0, r.stderr
    assert parse_describe(r.stdout)["constraint"][0][0] == str(kind)


@pytest.mark.parametrize("line,msg", [
    ("constraint peanut { }", "Parameter b has to be larger than parameter a"),
    ("constraint peanut { a = 5; b = 5 }", "Parameter b has to be larger than parameter a"),
    ("constraint hourglass { R = 3; A = 4 }", "Amplitude has to be smaller than the radius"),
])
def test_implicit_surface_parameter_errors(tmp_path, line, msg):
    r = check(tmp_path, CONF.replace("constraint plane { }", line))
    assert r.returncode == 1 and msg in r.stderr, r.stderr


def test_vicsek_and_nve_integrators_parse(tmp_path):
    conf = CONF.replace("integrator brownian_pos { seed = 7; mu = 1.0 }\nintegrator brownian_align { seed = 8; nu = 0.1, mur = 1.0 }\n",
                        "integrator vicsek { v0 = 0.5; eta = 0.3; seed = 2 }\n")
    r = check(tmp_path, conf)
    assert r.returncode == 0, r.stderr
    row = parse_describe(r.stdout)["integrator"][0]
    _, p, _ = PL.resolve_integrator("vicsek", {"v0": "0.5", "eta": "0.3", "seed": "2"}, 1e-3)
    assert row[0] == "vicsek_all" and [float(v) for v in row[2:]] == list(p[:12])
    r = check(tmp_path, conf + "disable vicsek { }\nintegrator nve { limit = 0.001 }\nrun 5\n")
    assert r.returncode == 0, r.stderr


def test_old_input_formats(tmp_path):
    parts, _ = plane_parts(50)
    for style in ("hash", "old"):
        r = check(tmp_path, CONF, parts, style)
        assert r.returncode == 0, (style, r.stderr)
        assert parse_describe(r.stdout)["particles"][0][0] == "50"


def parse_params(text):
    r = subprocess.run([BIN, "--params", text], capture_output=True, text=True, timeout=60)
    if r.returncode != 0:
        return None
    return dict(line.split("=", 1) for line in r.stdout.splitlines())


def test_parameter_block_grammar():
    # key_value_sequence: '{}' or pairs separated by ';' or ',', trailing ';' allowed
    assert parse_params("{}") == {}
    assert parse_params("{ k = 10.0; use_particle_radii }") == {"k": "10.0", "use_particle_radii": ""}
    assert parse_params("{a=1,b=2;;}") == {"a": "1", "b": "2"}
    assert parse_params("{ seed = 1;  mu = 1.0; group = all }")["group"] == "all"
    assert parse_params("{ k = }") is None
    assert parse_params("{ 1k = 2 }") is None


# ---- GPU: the host and the Python binding give the same bits ---------------------------
def python_run(parts, L, segments):
    from samos_b200 import Engine
    from scenarios import drive
    e = Engine(len(parts["x"]))
    sim = drive(e, parts, (L, L, 10.0), nlist=(2.4, 0.3), constraint=("plane", {}),
                pairs=[("soft", {"k": "10.0", "use_particle_radii": ""})], aligns=[("polar", {"J": "0.1"})],
                dt=1e-3, integrators=segments[0])
    sim.run(segments[1])
    e.enforce()  # the start-of-step enforce a dump at the next step sees
    return {f: e.download(f) for f in ("x", "y", "nx", "ny")}


def read_dump(path):
    rows = np.loadtxt(path, skiprows=1)
    return {"x": rows[:, 3], "y": rows[:, 4], "nx": rows[:, 9], "ny": rows[:, 10]}


@pytest.mark.gpu
@pytest.mark.parametrize("dump_freq,last_dump", [(400, 400), (37, 444)])
def test_host_run_matches_python_binding(tmp_path, dump_freq, last_dump):
    # `run 480` is iterations 0..480; a dump acts at the top of an iteration
    # (after that step's constraint enforce), so the last dump written is at
    # the last multiple of the frequency <= 480, and the host splits the run
    # there (sg_run, then sg_run_continue).
    parts, L = plane_parts(900, 50.0, seed=9)
    write_particles(tmp_path / "p.dat", parts)
    dump = f"dump out {{ type=input; start=0; freq={dump_freq} }}\n"
    conf = CONF.replace("lx = 40.0;  ly = 40.0", "lx = 50.0;  ly = 50.0").replace("run 10\n", dump + "run 480\n")
    (tmp_path / "c.conf").write_text(conf)
    r = subprocess.run([BIN, "--quiet", str(tmp_path / "c.conf")], capture_output=True, text=True, timeout=600,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    got = read_dump(tmp_path / "out.dat")
    want = python_run(parts, L, ([("brownian_pos", {"seed": "7", "mu": "1.0"}),
                                  ("brownian_align", {"seed": "8", "nu": "0.1", "mur": "1.0"})], last_dump - 1))
    for f in ("x", "y", "nx", "ny"):
        np.testing.assert_array_equal(got[f], want[f], err_msg=f)


@pytest.mark.gpu
def test_host_disable_and_new_integrator_between_runs(tmp_path):
    # the example configurations' pattern: relax with nve {limit}, disable it,
    # then run Brownian dynamics; the host must drive the engine exactly as
    # the same ABI calls made directly (integrator inserted at its map position)
    from samos_b200 import Engine, engine as E
    parts, L = plane_parts(700, 45.0, seed=12)
    write_particles(tmp_path / "p.dat", parts)
    conf = ("box periodic { lx = 45.0;  ly = 45.0;  lz = 10.0 }\ninput p.dat\nnlist { rcut = 2.4; pad = 0.3 }\n"
            "constraint plane { }\npair_potential soft { k = 1.0 }\npair_align polar { J = 1.0 }\n"
            "timestep 0.001\nintegrator nve { limit = 0.0001 }\nrun 199\ndisable nve { group = all }\n"
            "external self_propulsion { alpha = 1.0 }\ntimestep 0.01\n"
            "integrator brownian_pos { seed = 1;  mu = 1.0; group = all }\n"
            "integrator brownian_align { seed = 1;  mur = 1.0; nu = 0.1; group = all }\n"
            "dump out { type=input; start=0; freq=50 }\nrun 249\n")
    (tmp_path / "c.conf").write_text(conf)
    r = subprocess.run([BIN, "--quiet", str(tmp_path / "c.conf")], capture_output=True, text=True, timeout=600,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    got = read_dump(tmp_path / "out.dat")  # written at global step 400 (top of the run's iteration 200)

    e = Engine(len(parts["x"]))
    e.set_box(45.0, 45.0, 10.0, True)
    for f in ("x", "y", "z", "nx", "ny", "nz", "radius"):
        e.upload(f, parts[f])
    e.set_nlist(2.4, 0.3)
    kind, cp = PL.resolve_constraint("plane", {})
    e.add_constraint(kind, cp)
    soft = PL.resolve_pair("soft", {"k": "1.0"}, 1, 2.4)
    polar = PL.resolve_align("polar", {"J": "1.0"}, 1, 2.4)
    sp = PL.resolve_external("self_propulsion", {"alpha": "1.0"}, 1)
    e.set_timestep(0.001)
    e.add_pair(soft.kind, soft.glob, soft.table.reshape(-1), soft.use_radii, False, False, False, soft.phase_value)
    e.add_align(polar.kind, polar.J, polar.rcut, polar.table.reshape(-1), False)
    k, p, t = PL.resolve_integrator("nve", {"limit": "0.0001"}, 0.001)
    e.insert_integrator(0, k, p, t)
    e.run(199)
    e.disable_integrator(0)
    e.set_timestep(0.01)
    e.clear_forces()
    e.add_pair(soft.kind, soft.glob, soft.table.reshape(-1), soft.use_radii, False, False, False, soft.phase_value)
    e.add_align(polar.kind, polar.J, polar.rcut, polar.table.reshape(-1), False)
    e.add_external(sp.kind, sp.alpha, sp.type_alpha, sp.has_params)
    k, p, t = PL.resolve_integrator("brownian_pos", {"seed": "1", "mu": "1.0", "group": "all"}, 0.01)
    e.insert_integrator(0, k, p, t)
    k, p, t = PL.resolve_integrator("brownian_align", {"seed": "1", "mur": "1.0", "nu": "0.1", "group": "all"}, 0.01)
    e.insert_integrator(0, k, p, t)  # "brownian_align_all" < "brownian_pos_all"
    e.run(199)                       # global steps 200..399
    e.begin_step()                   # the dump at global step 400 sees the next step's enforce
    for f in ("x", "y", "nx", "ny"):
        np.testing.assert_array_equal(got[f], e.download(f), err_msg=f)
