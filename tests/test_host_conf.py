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
    # from the conf file's directory, where its dumps and logs land
    return subprocess.run([BIN, *flags, conf_path], capture_output=True, text=True, timeout=600,
                          cwd=os.path.dirname(os.path.abspath(conf_path)))


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
    ("group g { molecule = 1 }", "Group criterion molecule is not part of the GPU path."),
    ("group tissue { type = 1 }", 'Groups "tissue" and "boundary" are reserved'),
    ("integrator brownian { group = nosuch }", "Group nosuch is not defined."),
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


@pytest.mark.parametrize("line,msg", [
    ("dump a { start = 0 }", "No dump type specified."),
    ("dump a { type = mol2 }", "Dump type mol2 is not part of the GPU path."),
    ("dump a { type = foo }", "Unsupported dump type foo."),
    ("dump a { type = dcd; multi }", "DCD files cannot be split."),
    ("log a.log { area }", "Log quantity area is not part of the GPU path."),
    ("log a.log { foo }", "Unknown log quantity : foo."),
])
def test_dump_and_log_errors_follow_the_reference(tmp_path, line, msg):
    r = check(tmp_path, CONF.replace("run 10\n", line + "\nrun 10\n"))
    assert r.returncode == 1 and msg in r.stderr, r.stderr


def test_dump_files_and_log_header_at_construction(tmp_path):
    # the reference opens a dump's single file (writing the DCD header) and a
    # log's file (writing its header) when the command is read
    extra = ("dump traj { type = dcd; freq = 5 }\ndump pos { type = xyz; freq = 5 }\n"
             "dump frames { type = full; multi; coordinate }\nlog run.log { freq = 5; velocity; soft_energy }\n"
             "config c { type = json }\n")
    r = check(tmp_path, CONF.replace("run 10\n", extra + "run 10\n"))
    assert r.returncode == 0, r.stderr
    head = (tmp_path / "traj.dcd").read_bytes()
    assert len(head) == 4 + 84 + 4 + 4 + 164 + 4 + 4 + 4 + 4 and head[4:8] == b"CORD"
    assert np.frombuffer(head[-8:-4], np.int32)[0] == 400  # particles
    assert (tmp_path / "pos.xyz").read_text() == ""
    assert not list(tmp_path.glob("frames*"))  # multi: one file per dump, none yet
    log = (tmp_path / "run.log").read_text().splitlines()
    assert log[0] == "# Log file : run.log" and log[1].startswith("# Generated on : ")
    assert log[2].split() == ["#", "(1)", "step", "(2)", "soft_energy", "(3)", "velocity"]


def test_groups_and_grouped_integrators_parse(tmp_path):
    # the two-component example's pattern: groups by type, one integrator per group
    parts, _ = plane_parts()
    parts["type"] = np.where(np.arange(len(parts["x"])) % 3 == 0, 2, 1)
    conf = CONF.replace("integrator brownian_pos { seed = 7; mu = 1.0 }\nintegrator brownian_align { seed = 8; nu = 0.1, mur = 1.0 }\n",
                        "group passive { type = 1 }\ngroup active { type = 2 }\n"
                        "integrator brownian { group = active; seed = 1; v0 = 0.5 }\n"
                        "integrator brownian { group = passive; seed = 4; v0 = 0.0; temperature_control = constant; "
                        "min_val = 0.3 }\n")
    r = check(tmp_path, conf, parts=parts)
    assert r.returncode == 0, r.stderr
    assert [x[0] for x in parse_describe(r.stdout)["integrator"]] == ["brownian_active", "brownian_passive"]


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


def read_dump(path, n):
    """Last frame of a `type=full; coordinate; director` dump (one file, frames
    appended, as the reference writes it without `multi`)."""
    rows = np.array([[float(v) for v in line.split()] for line in open(path)
                     if line.strip() and not line.startswith(("#", "keys"))])
    rows = rows[-n:]
    return {"x": rows[:, 0], "y": rows[:, 1], "nx": rows[:, 3], "ny": rows[:, 4]}


def assert_dump_matches(got, want):
    # x, y printed with %16.10e, directors with %10.6f (dump.cpp:616-625)
    for f in ("x", "y"):
        np.testing.assert_allclose(got[f], want[f], rtol=0, atol=1e-8, err_msg=f)
    for f in ("nx", "ny"):
        np.testing.assert_allclose(got[f], want[f], rtol=0, atol=1e-6, err_msg=f)


@pytest.mark.gpu
@pytest.mark.parametrize("dump_freq,last_dump", [(400, 400), (37, 444)])
def test_host_run_matches_python_binding(tmp_path, dump_freq, last_dump):
    # `run 480` is iterations 0..480; a dump acts at the top of an iteration
    # (after that step's constraint enforce), so the last dump written is at
    # the last multiple of the frequency <= 480, and the host splits the run
    # there (sg_run, then sg_run_continue).
    parts, L = plane_parts(900, 50.0, seed=9)
    write_particles(tmp_path / "p.dat", parts)
    dump = f"dump out {{ type=full; start=0; freq={dump_freq}; coordinate; director }}\n"
    conf = CONF.replace("lx = 40.0;  ly = 40.0", "lx = 50.0;  ly = 50.0").replace("run 10\n", dump + "run 480\n")
    (tmp_path / "c.conf").write_text(conf)
    r = subprocess.run([BIN, "--quiet", str(tmp_path / "c.conf")], capture_output=True, text=True, timeout=600,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    got = read_dump(tmp_path / "out.dat", len(parts["x"]))
    want = python_run(parts, L, ([("brownian_pos", {"seed": "7", "mu": "1.0"}),
                                  ("brownian_align", {"seed": "8", "nu": "0.1", "mur": "1.0"})], last_dump - 1))
    assert_dump_matches(got, want)


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
            "dump out { type=full; start=0; freq=50; coordinate; director }\nrun 249\n")
    (tmp_path / "c.conf").write_text(conf)
    r = subprocess.run([BIN, "--quiet", str(tmp_path / "c.conf")], capture_output=True, text=True, timeout=600,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    got = read_dump(tmp_path / "out.dat", len(parts["x"]))  # last frame: global step 400 (top of iteration 200)

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
    assert_dump_matches(got, {f: e.download(f) for f in ("x", "y", "nx", "ny")})


@pytest.mark.gpu
def test_host_dump_types_and_log_columns(tmp_path):
    # every dump type and log column of the GPU path, from one host run,
    # against the Python binding's state at the last dump step (at the
    # precision each format prints, dump.cpp / log_*.hpp)
    from samos_b200 import Engine
    from scenarios import drive
    parts, L = plane_parts(900, 50.0, seed=9)
    write_particles(tmp_path / "p.dat", parts)
    extra = ("dump pos { type = xyz; freq = 50 }\n"
             "dump vel { type = velocity; freq = 50; header; scale = 0.5 }\n"
             "dump dirs { type = director; freq = 50 }\n"
             "dump arrows { type = xyzv; freq = 50; velocity; scale = 2 }\n"
             "dump inp { type = input; freq = 50 }\n"
             "dump traj { type = dcd; freq = 50 }\n"
             "dump pic { type = vtp; freq = 50 }\n"
             "dump frames { type = full; freq = 50; multi; keys; id; tp; radius; coordinate; velocity; force; "
             "director; image_flags; normal }\n"
             "log run.log { freq = 50; velocity; vec_velocity; kinetic_energy; soft_energy; polar_align }\n")
    conf = CONF.replace("lx = 40.0;  ly = 40.0", "lx = 50.0;  ly = 50.0").replace("run 10\n", extra + "run 100\n")
    (tmp_path / "c.conf").write_text(conf)
    r = subprocess.run([BIN, "--quiet", str(tmp_path / "c.conf")], capture_output=True, text=True, timeout=600,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    n = len(parts["x"])
    e = Engine(n)
    drive(e, parts, (L, L, 10.0), nlist=(2.4, 0.3), constraint=("plane", {}),
          pairs=[("soft", {"k": "10.0", "use_particle_radii": ""})], aligns=[("polar", {"J": "0.1"})], dt=1e-3,
          integrators=[("brownian_pos", {"seed": "7", "mu": "1.0"}),
                       ("brownian_align", {"seed": "8", "nu": "0.1", "mur": "1.0"})]).run(99)
    e.begin_step()  # the dumps at step 100 see that step's enforce
    e.compute(1e-3)
    S = {f: e.download(f) for f in ("x", "y", "z", "vx", "vy", "vz", "nx", "ny", "nz", "fx", "fy", "fz", "omega",
                                     "ix", "iy", "iz", "Nx", "Ny", "Nz", "radius")}

    def last(path, width, skip=()):
        rows = [line for line in open(path) if line.strip() and not line.startswith(skip)]
        return rows[-n:] if width is None else [line.split("\t") for line in rows[-n:]]

    xyz = np.array([[float(v) for v in row] for row in last(tmp_path / "pos.xyz", 0, skip=("Generated",))])[:, 1:]
    np.testing.assert_allclose(xyz[:, 0], S["x"], atol=1e-6)
    np.testing.assert_allclose(xyz[:, 1], S["y"], atol=1e-6)
    assert open(tmp_path / "pos.xyz").read().count("Generated by SAMoS code.") == 3  # steps 0, 50, 100
    vel = np.array([[float(v) for v in row] for row in last(tmp_path / "vel.vel", 0, skip=("#",))])
    np.testing.assert_allclose(vel[:, 3], 0.5 * S["vx"], rtol=1e-7, atol=1e-12)
    np.testing.assert_allclose(vel[:, 0], S["x"] - 0.25 * S["vx"], rtol=1e-7, atol=1e-12)
    assert open(tmp_path / "vel.vel").readline() == "# scale a = 0.5\n"
    dirs = np.array([[float(v) for v in row] for row in last(tmp_path / "dirs.dir", 0)])
    np.testing.assert_allclose(dirs[:, 3], S["nx"], rtol=1e-7, atol=1e-12)
    arrows = last(tmp_path / "arrows.xyzv", 0, skip=("Generated",))
    assert {row[0] for row in arrows} == {"A"}
    np.testing.assert_allclose([float(row[4]) for row in arrows], 2 * S["vx"], rtol=1e-7, atol=1e-12)
    inp = np.array([[float(v) for v in row.split()] for row in last(tmp_path / "inp.inp", None, skip=("keys",))])
    np.testing.assert_allclose(inp[:, 4], S["x"], atol=1e-6)
    np.testing.assert_allclose(inp[:, 10], S["nx"], atol=1e-6)
    np.testing.assert_allclose(inp[:, 13], S["omega"], atol=1e-6)  # the `length` column carries omega
    raw = (tmp_path / "traj.dcd").read_bytes()
    frame = 4 + 48 + 4 + 3 * (4 + 4 * n + 4)
    assert (len(raw) - 276) == 3 * frame
    zc = np.frombuffer(raw[-(4 + 4 * n):-4], np.float32)
    xc = np.frombuffer(raw[-(3 * (4 + 4 * n + 4)) + 4:-(3 * (4 + 4 * n + 4)) + 4 + 4 * n], np.float32)
    np.testing.assert_allclose(xc, S["x"].astype(np.float32))
    np.testing.assert_array_equal(zc, S["z"].astype(np.float32))
    assert (tmp_path / "pic.vtp").stat().st_size == 0  # opened at construction, frames go to pic_<step>.vtp
    import re
    xml = (tmp_path / "pic_0000000100.vtp").read_text()

    def arr(name, comps=1):
        body = re.search(r'Name="%s"[^>]*>(.*?)</DataArray>' % name, xml, re.S).group(1)
        return np.array(body.split(), float).reshape(-1, comps)

    np.testing.assert_array_equal(arr("Id")[:, 0], np.arange(n))
    np.testing.assert_allclose(arr("Velocity", 3)[:, 0], S["vx"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(arr("Force", 3)[:, 1], S["fy"], rtol=1e-15, atol=0)
    np.testing.assert_array_equal(arr("NDirector", 3), -arr("Director", 3))
    np.testing.assert_allclose(arr("NativeArea")[:, 0], 3.14159265359 * S["radius"] ** 2, rtol=1e-15)
    assert not arr("Pressure").any()
    np.testing.assert_array_equal(arr("NumNeigh")[:, 0], e.coordination())
    pts = re.search(r"<Points>\s*<DataArray[^>]*>(.*?)</DataArray>", xml, re.S).group(1)
    np.testing.assert_array_equal(np.array(pts.split(), float).reshape(-1, 3)[:, 0], S["x"])
    full = np.loadtxt(tmp_path / "frames_0000000100.dat", skiprows=1)
    keys = open(tmp_path / "frames_0000000100.dat").readline().split()[1:]
    # (omega left out: its "%8.5f " runs into the director column when negative, as in the reference)
    assert keys == ["id", "type", "radius", "x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "nx", "ny", "nz",
                    "ix", "iy", "iz", "nvx", "nvy", "nvz"]
    col = {k: full[:, i] for i, k in enumerate(keys)}
    np.testing.assert_array_equal(col["id"], np.arange(n))
    for k, f, tol in (("x", "x", 1e-8), ("vx", "vx", 1e-6), ("fx", "fx", 1e-6), ("ny", "ny", 1e-6),
                      ("nvz", "Nz", 1e-6)):
        np.testing.assert_allclose(col[k], S[f], rtol=1e-7, atol=tol, err_msg=k)
    np.testing.assert_array_equal(col["ix"], S["ix"])
    log = [line.split() for line in open(tmp_path / "run.log") if not line.startswith("#")]
    assert [int(r[0]) for r in log] == [0, 50, 100]
    step, kin, polar, soft, vec, speed = (float(v) for v in log[-1])  # step, then std::map key order
    v2 = S["vx"] ** 2 + S["vy"] ** 2 + S["vz"] ** 2
    assert speed == pytest.approx(np.mean(np.sqrt(v2)), rel=1e-6)
    vs = np.array([S["vx"].sum(), S["vy"].sum(), S["vz"].sum()])
    assert vec == pytest.approx(np.linalg.norm(vs) / n, rel=1e-6, abs=1e-12)
    assert kin == pytest.approx(np.mean(0.5 * v2), rel=1e-6)
    assert soft == pytest.approx(e.energy(0, 0), rel=1e-6)
    assert polar == pytest.approx(e.energy(1, 0), rel=1e-6)
