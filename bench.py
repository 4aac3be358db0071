"""Benchmark of the SAMoS hot path on B200: particle-steps/s of the FP64
active-Brownian step at 4,194,304 particles.

Workload (the single-GPU headline shape): 4,194,304 soft disks in a 2D
periodic box at packing fraction 0.8, radii 1.0 / 1.4 (50:50), positions
uniform from a seed, soft repulsion k=10 on particle radii, nematic aligner
J=0.5, brownian v0=0.3 nu=0.1, dt=5e-4, neighbour list rcut 2.8 + pad 0.3.
A step is one full integration step (forces, torques, integration, skin test,
rebuilds when triggered) of that system.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs one independent replica per rank (weak scaling, no data-path
collective; the path has no exchange step).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s @4M ABPs; batched vs serial; FIRE s to Fmax<1e-10 ML vs plain"
UNIT = "particle-steps/s"
N_PART = 4_194_304
PHI = 0.8
RADII = (1.0, 1.4)
BYTES_PER_PARTICLE_STEP = 88  # 2-D: read x,y,nx,ny,r (40 B) + write x,y,nx,ny,vx,vy (48 B)
WORKLOAD = ("4,194,304 active soft disks, 2D periodic box, phi=0.8, radii 1.0/1.4 50:50, soft k=10 "
            "(particle radii) + nematic J=0.5, brownian v0=0.3 nu=0.1 dt=5e-4, nlist rcut 2.8 pad 0.3, FP64")


def make_particles(n, seed):
    rng = np.random.default_rng(seed)
    r = np.where(np.arange(n) % 2 == 0, RADII[0], RADII[1]).astype(np.float64)
    rng.shuffle(r)
    L = float(np.sqrt(np.sum(np.pi * r * r) / PHI))
    th = rng.uniform(0.0, 2.0 * np.pi, n)
    parts = dict(x=rng.uniform(-L / 2, L / 2, n), y=rng.uniform(-L / 2, L / 2, n), z=np.zeros(n),
                 vx=np.zeros(n), vy=np.zeros(n), vz=np.zeros(n),
                 nx=np.cos(th), ny=np.sin(th), nz=np.zeros(n), radius=r)
    return parts, L


def configure(sim, parts, L):
    sim.box(L, L, 10.0, True)
    sim.input(**parts)
    sim.nlist(2.8, 0.3)
    sim.constraint("plane", {})
    sim.pair_potential("soft", {"k": "10", "use_particle_radii": ""})
    sim.pair_align("nematic", {"J": "0.5"})
    sim.timestep(5e-4)
    sim.integrator("brownian", {"v0": "0.3", "nu": "0.1", "mu": "1", "mur": "1", "seed": "1"})
    sim.commit()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.path or not os.path.exists(self.path):
            return out
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if sm:
            out.update(sm_mhz=float(np.median(sm)), sm_max_mhz=float(max(smax)), reasons=sorted(reasons),
                       samples=len(sm))
        return out


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own hot-path sources (oracle/_ref, built from
# the SAMoS tree with its Release flags) on a bounded sample of the same
# workload; the C oracle when that build is absent
# ---------------------------------------------------------------------------
class _Quiet:
    """Sends this process's stdout (fd 1) to /dev/null: the reference's
    particle reader prints one line per input column."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(null, 1)
        os.close(null)
        return self

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def _cpu_sample(args):
    n, warm, steps, seed, kind = args
    from samos_b200.plugins import Simulation
    parts, L = make_particles(n, seed)
    if kind == "reference":
        from oracle.refsrc import RefSimulation
        with _Quiet():
            sim = RefSimulation(fast=True)
            configure(sim, parts, L)
            sim.run(warm - 1)
            t0 = time.perf_counter()
            sim.run(steps - 1)
            dt = time.perf_counter() - t0
    else:
        from oracle.oracle import OracleSystem
        o = OracleSystem(n)
        sim = Simulation(o)
        configure(sim, parts, L)
        sim.run(warm - 1)
        t0 = time.perf_counter()
        o.run(steps - 1)
        dt = time.perf_counter() - t0
    return n * steps / dt


def cpu_baseline(n=131_072, warm=100, steps=60, procs=1):
    import multiprocessing as mp
    from oracle import refsrc
    kind = "reference" if refsrc.available(fast=True) else "port"
    if procs == 1:
        v = _cpu_sample((n, warm, steps, 11, kind))
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(procs) as pool:
            v = sum(pool.map(_cpu_sample, [(n, warm, steps, 11 + i, kind) for i in range(procs)]))
    what = ("SAMoS's own hot-path sources built with its Release flags (-O3 -funroll-loops -ffast-math, "
            "x86-64-v3), driven through their classes" if kind == "reference" else
            "the C oracle (a restatement of the reference's loops, -O2 strict IEEE)")
    return dict(value=v, unit=UNIT, cores=procs, kind=kind,
                sample=f"{n} particles of the same density/composition (box scaled), {warm} untimed + "
                       f"{steps} timed steps per process, {procs} single-threaded process(es); {what}")


# ---------------------------------------------------------------------------
# batched replicas vs the same replicas launched one at a time
# ---------------------------------------------------------------------------
def sphere_parts(n, seed):
    rng = np.random.default_rng(seed)
    R = float(np.sqrt(n / 4.0))  # packing fraction 1 at radius 1: n pi = 4 pi R^2
    z = rng.uniform(-R, R, n)
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    s = np.sqrt(np.maximum(R * R - z * z, 0.0))
    pos = np.stack([s * np.cos(ph), s * np.sin(ph), z], 1)
    nrm = pos / R
    a = rng.normal(size=(n, 3))
    t = a - np.sum(a * nrm, 1)[:, None] * nrm
    t /= np.linalg.norm(t, axis=1)[:, None]
    return dict(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=z, nx=t[:, 0].copy(), ny=t[:, 1].copy(),
                nz=t[:, 2].copy(), radius=np.ones(n)), R


def ensemble_replicas(n_rep=256, seed=7):
    """256 sphere systems, N log-uniform in [1024, 65536], R = sqrt(N/4), v0 ~ U[0.01,1],
    J ~ U[0,1], nu ~ logU[1e-3,1], own seeds; soft k=10 + polar, dt=1e-3."""
    from samos_b200.ensemble import SphereReplica
    rng = np.random.default_rng(seed)
    reps = []
    for i in range(n_rep):
        n = int(round(np.exp(rng.uniform(np.log(1024), np.log(65536)))))
        parts, R = sphere_parts(n, seed * 1000 + i)
        reps.append(SphereReplica(parts=parts, R=R, v0=float(rng.uniform(0.01, 1.0)), J=float(rng.uniform(0.0, 1.0)),
                                  nu=float(np.exp(rng.uniform(np.log(1e-3), 0.0))), seed=int(rng.integers(1, 2**31 - 1))))
    return reps


def ensemble_only(variant=-1, warm=80, steps=100, device=0):
    """The batched half of batched_leg alone (profiling runs): one engine over
    the 256 replicas, `warm` untimed steps, then `steps` timed ones."""
    from samos_b200 import Engine
    from samos_b200.ensemble import sphere_ensemble
    reps = ensemble_replicas()
    eng = sphere_ensemble(reps, engine=Engine([len(r.parts["x"]) for r in reps], device=device))
    if variant >= 0:
        eng.set_variant(variant)
    eng.run(warm - 1)
    st = eng.run(steps - 1)
    out = dict(workload="256-replica sphere ensemble", particles=sum(len(r.parts["x"]) for r in reps),
               ms_per_step=st.device_ms / st.steps_done, nlist_builds=st.nlist_builds,
               rebuild_ms_per_step=st.rebuild_ms / st.steps_done, kernel_variant=eng.variant())
    eng.close()
    return out


def batched_leg(n_rep=256, warm=80, steps=100, seed=7, device=0):
    """The replicas of ensemble_replicas stepped in one engine, then one at a time."""
    from samos_b200 import Engine
    from samos_b200.ensemble import sphere_ensemble
    reps = ensemble_replicas(n_rep, seed)
    total = sum(len(r.parts["x"]) for r in reps)
    eng = sphere_ensemble(reps, engine=Engine([len(r.parts["x"]) for r in reps], device=device))
    eng.run(warm - 1)
    st = eng.run(steps - 1)
    batched_s = st.device_ms * 1e-3
    final_b = [eng.download("x", replica=i) for i in range(n_rep)]
    eng.close()
    serial_s, identical = 0.0, True
    t_wall = time.perf_counter()
    for i, r in enumerate(reps):
        e1 = sphere_ensemble([r], engine=Engine([len(r.parts["x"])], device=device))
        e1.run(warm - 1)
        s1 = e1.run(steps - 1)
        serial_s += s1.device_ms * 1e-3
        identical = identical and bool(np.array_equal(e1.download("x"), final_b[i]))
        e1.close()
    t_wall = time.perf_counter() - t_wall
    return dict(replicas=n_rep, particles=total, steps=steps,
                batched_particle_steps_per_s=total * steps / batched_s,
                serial_particle_steps_per_s=total * steps / serial_s,
                speedup=serial_s / batched_s, identical_results=identical,
                timing="CUDA events on the engine stream around the timed steps (serial: summed over the "
                       "256 one-at-a-time runs)", serial_wall_s=t_wall)


def ml_leg(count=48, seed=4242, device=0):
    """Learned FIRE warm start vs plain FIRE (to Fmax < 1e-10, FP64) on `count`
    fresh quenches (N log-uniform in [1024, 16384], phi uniform in [0.84, 0.90]),
    with the network trained by `python -m samos_b200.warmstart train` on 2,000
    GPU-FIRE relaxations at N = 4096 (samos_b200/data/warmstart_c5.npz)."""
    path = os.path.join(ROOT, "samos_b200", "data", "warmstart_c5.npz")
    if not os.path.exists(path):
        return {"unavailable": "no trained warm-start parameters (samos_b200/data/warmstart_c5.npz)"}
    import torch
    torch.cuda.set_device(device)
    from samos_b200.warmstart import WarmStartNet, quench_set, relax, summarize
    net = WarmStartNet(device=f"cuda:{device}")
    net.load(path)
    insts = quench_set(count, 1024, 16384, 0.84, 0.90, seed=seed)
    plain = relax(insts, None)
    warm = relax(insts, net)
    rep = summarize(plain, warm, insts)
    rep["timing"] = "CUDA events on the engine stream: inference + apply + fallback + minimisation (warm), minimisation (plain)"
    rep["sample"] = (f"{count} fresh quenches, a subsample of the configuration's 512 evaluation instances "
                     "(the full 512 and the hand-off sweep: python -m samos_b200.warmstart eval / sweep)")
    return rep


# ---------------------------------------------------------------------------
# per-component rows: every potential, aligner, integrator and constraint
# family of the hot path timed on the GPU beside the reference's own code
# (the C oracle when that build is absent) on one core
# ---------------------------------------------------------------------------
def plane_mono(n, phi, seed):
    """n radius-1 disks on a square lattice of spacing sqrt(pi/phi) (> 2 below
    phi = 0.78: no overlaps, so the steep potentials start finite), jittered
    by up to 0.1, in a periodic square box."""
    rng = np.random.default_rng(seed)
    m = int(np.ceil(np.sqrt(n)))
    a = float(np.sqrt(np.pi / phi))
    L = m * a
    k = np.arange(n)
    th = rng.uniform(0.0, 2.0 * np.pi, n)
    z = np.zeros(n)
    x = -L / 2 + (k % m + 0.5) * a + rng.uniform(-0.1, 0.1, n)
    y = -L / 2 + (k // m + 0.5) * a + rng.uniform(-0.1, 0.1, n)
    return dict(x=x, y=y, z=z, vx=z, vy=z, vz=z, nx=np.cos(th), ny=np.sin(th), nz=z, radius=np.ones(n)), L


def torus_parts(n, seed):
    """n radius-1 particles on a torus of tube radius a = c/3 at packing fraction 0.5."""
    rng = np.random.default_rng(seed)
    c = float(np.sqrt(3.0 * n / (2.0 * np.pi)))
    a = c / 3.0
    u, v = rng.uniform(0.0, 2.0 * np.pi, n), rng.uniform(0.0, 2.0 * np.pi, n)
    x, y, z = (c + a * np.cos(v)) * np.cos(u), (c + a * np.cos(v)) * np.sin(u), a * np.sin(v)
    t = np.stack([-np.sin(u), np.cos(u), np.zeros(n)])
    zero = np.zeros(n)
    return dict(x=x, y=y, z=z, vx=zero, vy=zero, vz=zero, nx=t[0], ny=t[1], nz=t[2], radius=np.ones(n)), c, a


BROWNIAN_ROW = ("brownian", {"v0": "0.5", "nu": "0.1", "mu": "1", "mur": "1", "seed": "3"})
ROWS = (
    # name, geometry, pair, aligner, integrator, dt, state bytes per particle-step
    ("brownian, soft (particle radii) + nematic, plane", "bidisperse",
     ("soft", {"k": "10", "use_particle_radii": ""}), ("nematic", {"J": "0.5"}), BROWNIAN_ROW, 5e-4, 88),
    ("brownian, lj (shifted) + polar, plane", "mono",
     ("lj", {"epsilon": "1", "sigma": "1", "rcut": "2.5", "shifted": ""}), ("polar", {"J": "0.2"}), BROWNIAN_ROW,
     1e-4, 88),
    ("brownian, morse (shifted) + polar, plane", "mono",
     ("morse", {"D": "1", "a": "2", "re": "2", "rcut": "2.5", "shifted": ""}), ("polar", {"J": "0.2"}),
     BROWNIAN_ROW, 1e-3, 88),
    ("brownian, gaussian + polar, plane", "mono",
     ("gaussian", {"A": "2", "B": "-1", "alpha": "1", "beta": "3", "rA": "0", "rB": "1.5", "rcut": "2.5"}),
     ("polar", {"J": "0.2"}), BROWNIAN_ROW, 1e-3, 88),
    ("vicsek integrator, soft + vicsek aligner, plane", "mono", ("soft", {"k": "10"}), ("vicsek", {"rcut": "2.0"}),
     ("vicsek", {"v0": "0.5", "eta": "0.3", "mu": "0.1", "seed": "5"}), 1e-2, 88),
    ("langevin baoab, lj (shifted), plane", "mono",
     ("lj", {"epsilon": "1", "sigma": "1", "rcut": "2.5", "shifted": ""}), None,
     ("langevin", {"gamma": "1", "seed": "7", "method": "baoab", "min_val": "0.5"}), 1e-4, 88),
    ("nve (limit 1e-4), soft + polar, plane", "mono", ("soft", {"k": "1"}), ("polar", {"J": "1"}),
     ("nve", {"limit": "0.0001"}), 1e-3, 88),
    ("fire, soft (particle radii), plane", "bidisperse", ("soft", {"k": "1", "use_particle_radii": ""}), None,
     ("fire", {"dt_max": "0.1", "fmax_tolerance": "1e-10"}), 1e-2, 88),
    ("brownian, soft + polar, sphere", "sphere", ("soft", {"k": "10"}), ("polar", {"J": "0.2"}),
     ("brownian", {"v0": "1.0", "nu": "0.05", "mu": "1", "mur": "1", "seed": "3"}), 1e-3, 128),
    ("brownian, soft + polar, torus (SHAKE projection)", "torus", ("soft", {"k": "10"}), ("polar", {"J": "0.2"}),
     ("brownian", {"v0": "1.0", "nu": "0.05", "mu": "1", "mur": "1", "seed": "3"}), 1e-3, 128),
)


def row_system(backend, row, n, seed):
    """The row's program on a backend (engine or C oracle), or, given a
    RefSimulation, on the reference's own classes."""
    from samos_b200.plugins import Simulation
    name, geom, pair, align, integ, dt, _ = row
    sim = backend if hasattr(backend, "input_file") else Simulation(backend)
    if geom == "sphere":
        parts, R = sphere_parts(n, seed)
        zero = np.zeros(n)
        parts.update(vx=zero, vy=zero, vz=zero)
        sim.box(2 * R + 20, 2 * R + 20, 2 * R + 20, False)
        cons, rc = ("sphere", {"r": repr(R)}), (2.4, 0.3)
    elif geom == "torus":
        parts, c, a = torus_parts(n, seed)
        sim.box(2 * (c + a) + 20, 2 * (c + a) + 20, 2 * a + 20, False)
        cons, rc = ("torus", {"c": repr(c), "a": repr(a)}), (2.4, 0.3)
    else:
        if geom == "bidisperse":
            parts, L = make_particles(n, seed)
            rc = (2.8, 0.3)
        else:
            parts, L = plane_mono(n, 0.6, seed)
            rc = (2.8, 0.3)
        sim.box(L, L, 10.0, True)
        cons = ("plane", {})
    sim.input(**parts)
    sim.nlist(*rc)
    sim.constraint(*cons)
    sim.pair_potential(*pair)
    if align:
        sim.pair_align(*align)
    sim.timestep(dt)
    sim.integrator(*integ)
    sim.commit()
    return sim


def rows_leg(n=1_048_576, warm=50, steps=200, cpu_n=16_384, cpu_warm=5, cpu_steps=20, device=0, only=None):
    """Each row of ROWS: `warm` untimed then `steps` device-timed steps (CUDA
    events on the engine stream, rebuilds included) at n particles, and the
    oracle on one core at cpu_n particles of the same density.  `state_gbs` is
    the row's state bytes per particle-step (plane: read x, y, nx, ny, r, write
    x, y, nx, ny, vx, vy; 3-D: the same with z components) over the whole step
    time, a floor on the traffic a step must move."""
    from oracle.oracle import OracleSystem
    from samos_b200 import Engine
    peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs", 6650.0)) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0
    out = []
    for i, row in enumerate(ROWS):
        if only is not None and i != only:
            continue
        eng = Engine(n, device=device)
        sim = row_system(eng, row, n, 100 + i)
        sim.run(warm - 1)
        extra = 0  # the autotuner of the specialised kernels finishes untimed
        while eng.variant() < 0 and extra < 100:
            eng.run(19)
            extra += 20
        st = eng.run(steps - 1)
        ms = st.device_ms / st.steps_done
        occ = eng.generic_occupancy()
        eng.close()
        cpu, cpu_kind = None, "reference"
        try:  # the reference's own sources (Release flags), else the C oracle
            from oracle.refsrc import RefSimulation, available
            if not available(fast=True):
                raise FileNotFoundError
            with _Quiet():
                ref = row_system(RefSimulation(fast=True), row, cpu_n, 100 + i)
                ref.run(cpu_warm - 1)
                t0 = time.perf_counter()
                ref.run(cpu_steps - 1)
                cpu = cpu_n * cpu_steps / (time.perf_counter() - t0)
        except Exception:
            cpu_kind = "port"
            o = OracleSystem(cpu_n)
            row_system(o, row, cpu_n, 100 + i).run(cpu_warm - 1)
            t0 = time.perf_counter()
            o.run(cpu_steps - 1)
            cpu = cpu_n * cpu_steps / (time.perf_counter() - t0)
        gbs = n * row[6] / (ms * 1e-3) / 1e9
        out.append(dict(row=row[0], particles=n, steps=int(st.steps_done), ms_per_step=ms,
                        particle_steps_per_s=n / (ms * 1e-3), nlist_builds=int(st.nlist_builds),
                        state_bytes_per_particle_step=row[6], state_gbs=gbs, frac_of_hbm=gbs / peak,
                        cpu_particles=cpu_n, cpu_particle_steps_per_s=cpu, cpu_kind=cpu_kind,
                        gpu_over_cpu=n / (ms * 1e-3) / cpu, generic_blocks_per_sm=occ or None))
    return out


def step_kernel_name(variant):
    """The fused step kernel the autotuner kept for the headline program
    (soft + nematic + brownian on a periodic plane)."""
    if variant == 5:
        return "k_abp_flat<plane,nematic>"
    if variant in (6, 7):
        return f"k_abp_staged<plane,nematic,variant={variant}>"
    if variant == 8:
        return "k_abp_tile<plane,nematic>"
    return f"k_abp_step<plane,nematic,variant={variant}>"


def measured_traffic(kernel, n_part):
    """DRAM bytes per launch of the step kernel from the committed ncu
    summary (`dram_bytes_per_particle_step:` line, scaled to this system
    size), or None when no summary covers this kernel variant."""
    path = os.path.join(ROOT, "profiles", "k_abp_step_plane_nematic.md")
    if not os.path.exists(path):
        return None
    per = {}
    for line in open(path):
        if line.startswith("dram_bytes_per_particle_step"):
            # dram_bytes_per_particle_step[<kernel>]: <bytes>
            key = line.split("[", 1)[1].split("]", 1)[0]
            per[key] = float(line.rsplit(":", 1)[1])
    return per[kernel] * n_part if kernel in per else None


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def pg_backend():
    """NCCL between the GPUs of a node; gloo where no GPU is visible (the
    multi-process plumbing is exercised on CPU that way)."""
    import torch
    return "nccl" if torch.cuda.is_available() else "gloo"


def init_ranks(local):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    dist.init_process_group(pg_backend(), timeout=timedelta(seconds=120))


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return 0
    procs = os.cpu_count() or 1
    per = max(4096, min(262_144, int(4e7 / max(1, args.steps + args.warmup))))
    per = (per // 2) * 2
    base = cpu_baseline(per, args.warmup, args.steps, procs)
    line = dict(metric=METRIC, value=base["value"], unit=UNIT, n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=None, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic", impl="reference",
                config=dict(workload=WORKLOAD + " (CPU: bounded sample, see cpu_baseline)", parallelism="processes"),
                cpu_baseline=base, e2e=dict(value=base["value"], unit=UNIT, h2d_bytes_per_step=0,
                                            d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-vs-serial replica leg")
    ap.add_argument("--no-ml", action="store_true", help="skip the learned FIRE warm-start leg")
    ap.add_argument("--variant", type=int, default=-1,
                    help="pin the step-kernel variant instead of autotuning (profiling runs: ncu distorts the tuner's timings)")
    ap.add_argument("--build", type=int, default=0,
                    help="neighbour-list build kernel (0 automatic, 1 one thread per particle, 2 teams, 3 cell tiles)")
    ap.add_argument("--particles", type=int, default=N_PART,
                    help="system size (profiling runs use a smaller system of the same density)")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="run only the batched 256-replica ensemble (profiling runs) and print its timing")
    ap.add_argument("--rows", action="store_true",
                    help="time every potential / aligner / integrator / constraint family at 1,048,576 particles "
                         "beside the oracle on one core, print one JSON line per family")
    ap.add_argument("--row", type=int, default=None, help="with --rows: time only this row (index into ROWS)")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    if ws > 1:
        init_ranks(local)
    if args.impl == "reference":
        rc = run_reference_arm(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc
    args.warmup = max(args.warmup, 3)
    if args.ensemble_only:
        out = ensemble_only(args.variant, device=local)
        if rank == 0:
            print(json.dumps(out), flush=True)
        return 0
    if args.rows:
        if rank == 0:
            for r in rows_leg(device=local, only=args.row):
                print(json.dumps(r), flush=True)
        return 0

    from samos_b200 import Engine
    from samos_b200.plugins import Simulation

    n_part = args.particles
    parts, L = make_particles(n_part, seed=1 + rank)
    eng = Engine(n_part, device=local)
    eng.set_build(args.build)
    sim = Simulation(eng)
    configure(sim, parts, L)

    # warm-up (untimed); the engine's autotuner picks the step-kernel variant here
    if args.variant >= 0:
        eng.set_variant(args.variant)
    sim.run(args.warmup - 1)
    # a short warm-up ends before the tuner has tried every variant: finish
    # the tuning untimed (bounded), so the timed steps all run the kept one
    tuning_steps = 0
    while eng.variant() < 0 and tuning_steps < 400:
        eng.run(19)
        tuning_steps += 20

    # timed region: K steps with inputs resident in HBM (state 1.4 GB >> 126 MB L2)
    barrier(ws)
    launches0 = eng.kernel_launches()
    with ClockSampler(local) as clocks:
        st = eng.run(args.steps - 1)
    launches = eng.kernel_launches() - launches0
    variant = eng.variant()
    t_ms = max_over_ranks(st.device_ms, ws)
    value = ws * n_part * args.steps / (t_ms * 1e-3)

    # dominant kernel: per-launch CUDA-event time of the fused step kernel
    eng.set_profiling(True)
    pst = eng.run(min(args.steps, 200) - 1)
    eng.set_profiling(False)
    k_ms = pst.step_kernel_ms / max(1, pst.step_kernels)
    rebuild_ms = pst.rebuild_ms / pst.nlist_builds if pst.nlist_builds else None
    achieved = n_part * BYTES_PER_PARTICLE_STEP / (k_ms * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    kernel = step_kernel_name(variant)
    traffic = measured_traffic(kernel, n_part)

    # end to end through the C ABI with host buffers: inputs in page-locked
    # host memory (filled before the clock starts, as a caller's staging
    # buffers would be), uploaded, run, results read back into page-locked
    # arrays inside the timed region
    from samos_b200.engine import pinned_copy, pinned_empty
    barrier(ws)
    e2e_steps = args.steps
    fields_in = ("x", "y", "z", "vx", "vy", "vz", "nx", "ny", "nz", "radius")
    fields_out = ("x", "y", "nx", "ny", "vx", "vy")
    host_in = {f: pinned_copy(parts[f]) for f in fields_in}
    host_out = {f: pinned_empty(n_part) for f in fields_out}
    for a in host_out.values():
        a[:] = 0.0
    # one untimed pass of the same sequence first (the transfer path's first
    # use maps the page-locked buffers; a caller's staging buffers are reused)
    eng.upload_fields(host_in)
    eng.build_nlist()
    eng.run(e2e_steps - 1)
    eng.download_fields(fields_out, out=host_out)
    barrier(ws)
    t0 = time.perf_counter()
    eng.upload_fields(host_in)  # all fields' copies back to back, one wait
    t_up = time.perf_counter()
    eng.build_nlist()
    est = eng.run(e2e_steps - 1)
    t_run = time.perf_counter()
    outs = eng.download_fields(fields_out, out=host_out)
    t_end = time.perf_counter()
    e2e_s = max_over_ranks(t_end - t0, ws)
    e2e_split = dict(upload_ms=(t_up - t0) * 1e3, build_and_run_ms=(t_run - t_up) * 1e3,
                     download_ms=(t_end - t_run) * 1e3, untimed_passes_before=1)
    h2d = len(fields_in) * 8 * n_part / e2e_steps
    d2h = len(fields_out) * 8 * n_part / e2e_steps
    e2e_value = ws * n_part * e2e_steps / e2e_s
    finite = all(np.isfinite(v).all() for v in outs.values())

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline()
    batched = None
    if ws == 1 and not args.no_batched and args.particles == N_PART:
        eng.close()
        batched = batched_leg(device=local)
    ml = None
    if ws == 1 and not args.no_ml and args.particles == N_PART:
        ml = ml_leg(device=local)

    if rank == 0:
        line = dict(
            metric=METRIC, value=value, unit=UNIT, n_gpus=ws, steps=args.steps, warmup=args.warmup,
            ms_per_step=t_ms / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
            dtype="f64", data="synthetic",
            config=dict(workload=WORKLOAD if n_part == N_PART else WORKLOAD.replace("4,194,304", f"{n_part:,}"),
                        n_particles=n_part, box=L, parallelism=f"replicas x{ws}",
                        l2="state resident in HBM, 1.4 GB per buffer set >> 126 MB L2 (no flush needed)",
                        nlist_builds_timed=st.nlist_builds, kernel_variant=variant, untimed_tuning_steps=tuning_steps),
            roofline=dict(bound="hbm", achieved=achieved, peak=peak, unit="GB/s", frac=achieved / peak,
                          traffic=traffic, kernel=kernel, kernel_ms=k_ms,
                          algorithmic_bytes_per_particle_step=BYTES_PER_PARTICLE_STEP,
                          list_build_ms=rebuild_ms, list_builds_profiled=int(pst.nlist_builds),
                          peak_source="MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s"),
            e2e=dict(value=e2e_value, unit=UNIT, h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h,
                     steps=e2e_steps, finite=bool(finite), **e2e_split),
            gpu_launches=int(launches),
            clocks=clocks.summary(),
            cpu_baseline=cpu,
            batched=batched,
            fire_warm_start=ml,
        )
        print(json.dumps(line), flush=True)
    if eng.h:
        eng.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
