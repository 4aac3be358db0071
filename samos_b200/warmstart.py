"""Learned FIRE warm start.

A two-layer message-passing network (hidden width 64, neighbours within
rc = 2.8; kernels in csrc/sg_ml.cu) predicts, from a configuration, each
particle's displacement to its FIRE minimum.  Two places to apply it: at the
quench itself, or at the hand-off -- plain FIRE runs until max |F_i| first
drops below a hand-off tolerance, the network moves the particles from
there, and a fresh FIRE finishes to the final tolerance.  Up to the hand-off
both arms share every bit, so they start the last stretch in the same basin.  Training data are
quench-then-FIRE relaxations run by the engine's own GPU FIRE; training runs
the project's forward/backward kernels (BF16 tensor-core GEMMs, FP32
accumulation) with Adam.  At use, the predicted displacement is applied only
where it lowers a replica's energy; otherwise that replica starts from its
quench (plain FIRE is the fallback).

Device memory for parameters and activations is held in torch tensors
(allocation and plumbing only; every computation is a call into
libsamos_gpu.so).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch

from . import engine as E

F = 64
OFF = dict(W1a=(0, (64, 4)), b1a=(256, (64,)), W1b=(320, (64, 64)), b1b=(4416, (64,)), Wpq=(4480, (64, 128)),
           b2=(12672, (64,)), W2e=(12736, (64, 4)), w2=(12992, (64,)), c=(13056, (1,)))


def _p(t: torch.Tensor | None):
    return C.c_void_p(0) if t is None else C.c_void_p(t.data_ptr())


def _bind(lib):
    P, I, D, Fl = C.c_void_p, C.c_int, C.c_double, C.c_float
    vp = C.POINTER(E.View)
    sig = {
        "sg_mlp_param_count": (I, []), "sg_mlp_edge_blocks": (I, []), "sg_mlp_part_floats": (I, []),
        "sg_mlp_prepare": (I, [P] * 6),
        "sg_mlp_forward": (I, [vp, P, D, P, P, P, P, P, P, P, P]),
        "sg_mlp_backward": (I, [vp, P, D, P, P, P, P, P, P, P, P, Fl, P, P, P, P, P, P, P, P, P, P]),
        "sg_mlp_adam": (I, [P, P, P, P, I, Fl, Fl, Fl, Fl, I, P]),
        "sg_mlp_apply": (I, [vp, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


def _ok(rc, what):
    if rc != 0:
        raise E.EngineError(rc, what)


class WarmStartNet:
    def __init__(self, seed: int = 0, rc: float = 2.8, device: str = "cuda"):
        self.lib = _bind(E.load())
        self.rc = float(rc)
        self.dev = torch.device(device)
        n = self.lib.sg_mlp_param_count()
        self.params = torch.zeros(n, dtype=torch.float32, device=self.dev)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.W1b16 = torch.zeros(F * F, dtype=torch.bfloat16, device=self.dev)
        self.W1bT16 = torch.zeros_like(self.W1b16)
        self.Wpq16 = torch.zeros(F * 2 * F, dtype=torch.bfloat16, device=self.dev)
        self.WpqT16 = torch.zeros_like(self.Wpq16)
        self.step = 0
        self._ws = {}
        self.set_params(self.init_params(seed))

    @staticmethod
    def init_params(seed: int) -> np.ndarray:
        """Uniform fan-in initialisation; the output weights start small."""
        rng = np.random.default_rng(seed)
        p = np.zeros(13057, np.float32)
        def put(name, fan_in, scale=1.0):
            off, shape = OFF[name]
            b = scale / np.sqrt(fan_in)
            p[off:off + int(np.prod(shape))] = rng.uniform(-b, b, int(np.prod(shape)))
        put("W1a", 4); put("b1a", 4); put("W1b", 64); put("b1b", 64); put("Wpq", 64)
        put("b2", 64); put("W2e", 4); put("w2", 64, 0.1)
        return p

    def set_params(self, p: np.ndarray) -> None:
        self.params.copy_(torch.from_numpy(np.asarray(p, np.float32)))
        self._refresh()

    def get_params(self) -> np.ndarray:
        return self.params.detach().cpu().numpy().copy()

    def _refresh(self):
        _ok(self.lib.sg_mlp_prepare(_p(self.params), _p(self.W1b16), _p(self.W1bT16), _p(self.Wpq16),
                                    _p(self.WpqT16), None), "sg_mlp_prepare")

    def _work(self, slots: int):
        if slots not in self._ws:
            d = self.dev
            nb = self.lib.sg_mlp_edge_blocks()
            self._ws[slots] = dict(
                s16=torch.zeros(slots * F, dtype=torch.bfloat16, device=d),
                h16=torch.zeros(slots * F, dtype=torch.bfloat16, device=d),
                PQ=torch.zeros(slots * 2 * F, dtype=torch.float32, device=d),
                disp=torch.zeros(slots * 2, dtype=torch.float32, device=d),
                gPQ=torch.zeros(slots * 2 * F, dtype=torch.float32, device=d),
                gPQ16=torch.zeros(slots * 2 * F, dtype=torch.bfloat16, device=d),
                gh=torch.zeros(slots * F, dtype=torch.float32, device=d),
                gpre16=torch.zeros(slots * F, dtype=torch.bfloat16, device=d),
                gs=torch.zeros(slots * F, dtype=torch.float32, device=d),
                part=torch.zeros(self.lib.sg_mlp_part_floats(), dtype=torch.float32, device=d),
                red=torch.zeros(512, dtype=torch.float32, device=d),
                loss=torch.zeros(nb, dtype=torch.float32, device=d))
        return self._ws[slots]

    # -- graph helpers ---------------------------------------------------------------
    def box_array(self, eng: E.Engine, replicas=None) -> torch.Tensor:
        """(Lx, Ly) per slot of the selected replicas, 0 elsewhere."""
        view = eng.view()
        box = np.zeros(view.slots * 2)
        for r in (range(len(eng.n)) if replicas is None else replicas):
            off, n = eng.replica_slots(r)
            lx, ly, _, _ = eng.boxes[r]
            box[2 * off:2 * (off + n):2] = lx
            box[2 * off + 1:2 * (off + n):2] = ly
        return torch.from_numpy(box).to(self.dev)

    def slot_ids(self, eng: E.Engine) -> np.ndarray:
        view = eng.view()
        ids = np.zeros(view.slots, np.int32)
        _ok(self.lib.sg_memcpy(ids.ctypes.data_as(C.c_void_p), C.c_void_p(view.id), ids.nbytes), "ids")
        return ids

    def slot_targets(self, eng: E.Engine, targets: list[np.ndarray]) -> torch.Tensor:
        """Per-replica (n, 2) arrays in particle-id order -> slot-ordered float32."""
        ids = self.slot_ids(eng)
        t = np.zeros(len(ids) * 2, np.float32)
        for r, tr in enumerate(targets):
            off, n = eng.replica_slots(r)
            sl = ids[off:off + n]
            t[2 * off:2 * (off + n):2] = tr[sl, 0]
            t[2 * off + 1:2 * (off + n):2] = tr[sl, 1]
        return torch.from_numpy(t).to(self.dev)

    # -- network ----------------------------------------------------------------------
    def forward(self, eng: E.Engine, box: torch.Tensor) -> torch.Tensor:
        view = eng.view()
        w = self._work(view.slots)
        _ok(self.lib.sg_mlp_forward(C.byref(view), _p(box), self.rc, _p(self.params), _p(self.W1bT16),
                                    _p(self.WpqT16), _p(w["s16"]), _p(w["h16"]), _p(w["PQ"]), _p(w["disp"]), None),
            "sg_mlp_forward")
        return w["disp"]

    def loss_and_grad(self, eng: E.Engine, box: torch.Tensor, target: torch.Tensor, n_valid: int) -> float:
        """Mean squared displacement error; gradient into self.grad (overwritten)."""
        view = eng.view()
        w = self._work(view.slots)
        self.forward(eng, box)
        self.grad.zero_()
        _ok(self.lib.sg_mlp_backward(C.byref(view), _p(box), self.rc, _p(self.params), _p(self.W1b16),
                                     _p(self.Wpq16), _p(w["s16"]), _p(w["h16"]), _p(w["PQ"]), _p(w["disp"]),
                                     _p(target), 1.0 / n_valid, _p(w["gPQ"]), _p(w["gPQ16"]), _p(w["gh"]),
                                     _p(w["gpre16"]), _p(w["gs"]), _p(w["part"]), _p(w["red"]), _p(w["loss"]),
                                     _p(self.grad), None), "sg_mlp_backward")
        return float(w["loss"].sum().item()) / n_valid

    def adam_step(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.step += 1
        _ok(self.lib.sg_mlp_adam(_p(self.params), _p(self.grad), _p(self.m), _p(self.v), self.params.numel(),
                                 lr, beta1, beta2, eps, self.step, None), "sg_mlp_adam")
        self._refresh()

    def apply(self, eng: E.Engine, box: torch.Tensor, disp: torch.Tensor) -> None:
        view = eng.view()
        _ok(self.lib.sg_mlp_apply(C.byref(view), _p(box), _p(disp), C.c_void_p(view.ix), C.c_void_p(view.iy),
                                  None), "sg_mlp_apply")
        torch.cuda.synchronize()
        eng.positions_changed()

    def save(self, path: str, handoff: float | None = None) -> None:
        np.savez(path, params=self.get_params(), rc=self.rc, handoff=np.nan if handoff is None else handoff)

    def load(self, path: str) -> float | None:
        """Loads the parameters; returns the hand-off tolerance they were
        trained for (None: trained on quenches)."""
        d = np.load(path)
        self.rc = float(d["rc"])
        self.set_params(d["params"])
        h = float(d["handoff"]) if "handoff" in d.files else float("nan")
        return None if np.isnan(h) else h


def min_image(d: np.ndarray, L: float) -> np.ndarray:
    return d - L * np.round(d / L)


# -- data: quench-then-FIRE relaxations on the GPU ---------------------------------------
class Batch:
    """One engine holding `R` systems, with their relaxation targets
    (displacement from the network's input state to the FIRE minimum, slot
    order) kept on the device.  The input state is the quench, or with
    `handoff` the state where FIRE from the quench first has max |F_i| below
    `handoff` (the minimum then comes from FIRE continued from there)."""

    def __init__(self, net: WarmStartNet, insts, k: float = 1.0, dt: float = 0.01, dt_max: float = 0.2,
                 fmax: float = 1e-10, max_steps: int = 400000, handoff: float | None = None):
        from .ensemble import plane_fire_ensemble
        self.insts = insts
        self.handoff = handoff
        self.eng = plane_fire_ensemble(insts, k=k, dt=dt, dt_max=dt_max, fmax=handoff or fmax)
        self.eng.build_nlist()
        t0 = time.perf_counter()
        start = insts
        if handoff is not None:
            self.conv_handoff, st_h = self.eng.minimize(max_steps)
            start = snapshot(self.eng, insts)
            for r in range(len(insts)):
                self.eng.set_replica_param(r, 4, 0, 11, fmax)  # FIRE's max |F_i| tolerance
        self.conv, st = self.eng.minimize(max_steps)
        self.fire_s = time.perf_counter() - t0
        self.fire_device_ms = st.device_ms + (st_h.device_ms if handoff is not None else 0.0)
        self.energy = np.array([self.eng.energy(0, 0, r) for r in range(len(insts))])
        targets = []
        for r, (parts, L) in enumerate(start):
            fx, fy = self.eng.download("x", r), self.eng.download("y", r)
            targets.append(np.stack([min_image(fx - parts["x"], L), min_image(fy - parts["y"], L)], 1))
        self.targets = targets
        restore_quench(self.eng, start)
        self.start = start
        self.box = net.box_array(self.eng)
        self.target = net.slot_targets(self.eng, targets)
        self.n_valid = int(sum(len(p["x"]) for p, _ in insts))


def snapshot(eng: E.Engine, insts):
    """The engine's current positions as new instances (same radii and box,
    zero velocities): [(parts, L), ...]."""
    out = []
    for r, (parts, L) in enumerate(insts):
        p = dict(parts)
        p["x"], p["y"] = eng.download("x", r), eng.download("y", r)
        z = np.zeros(len(p["x"]))
        p["vx"], p["vy"] = z, z.copy()
        out.append((p, L))
    return out


def restore_quench(eng: E.Engine, insts, replicas=None) -> None:
    """Put the quench positions (and zero velocities) back into the engine."""
    for r in (range(len(insts)) if replicas is None else replicas):
        parts, _ = insts[r]
        for f in ("x", "y", "vx", "vy"):
            eng.upload(f, parts[f], replica=r)
        z = np.zeros(len(parts["x"]), np.int32)
        eng.upload("ix", z, replica=r)
        eng.upload("iy", z, replica=r)
    eng.positions_changed()


def quench_set(count: int, n_lo: int, n_hi: int, phi_lo: float, phi_hi: float, seed: int):
    """`count` quenches; N log-uniform in [n_lo, n_hi] (fixed if equal), phi uniform."""
    from .ensemble import quench_disks
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = n_lo if n_lo == n_hi else int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        n += n % 2
        out.append(quench_disks(n, float(rng.uniform(phi_lo, phi_hi)), int(rng.integers(1 << 31))))
    return out


def train(net: WarmStartNet, batches, steps: int, lr: float = 2e-3, lr_end: float = 1e-4, log_every: int = 0):
    """Adam on the mean squared displacement error, cycling through the
    batches; the learning rate decays geometrically from lr to lr_end."""
    hist = []
    for s in range(steps):
        b = batches[s % len(batches)]
        cur = lr * (lr_end / lr) ** (s / max(1, steps - 1))
        loss = net.loss_and_grad(b.eng, b.box, b.target, b.n_valid)
        net.adam_step(cur)
        hist.append(loss)
        if log_every and s % log_every == 0:
            print(f"step {s} loss {loss:.5f} lr {cur:.2e}", flush=True)
    return hist


def mean_target_sq(batch: Batch) -> float:
    """Loss of the zero displacement (the quench itself) on a batch."""
    return float(sum(np.sum(t * t) for t in batch.targets)) / batch.n_valid


def eval_loss(net: WarmStartNet, batch: Batch) -> float:
    disp = net.forward(batch.eng, batch.box)
    d = disp.view(-1, 2) - batch.target.view(-1, 2)
    return float((d * d).sum().item()) / batch.n_valid


# -- use: warm-started FIRE with plain FIRE as the fallback ----------------------------
def relax(insts, net: WarmStartNet | None, k: float = 1.0, dt: float = 0.01, dt_max: float = 0.2,
          fmax: float = 1e-10, max_steps: int = 400000, handoff: float | None = None) -> dict:
    """Relax every instance to Fmax < fmax in one engine.  With a network,
    the predicted displacement is applied first, and every replica whose
    energy it raises goes back to its start (plain FIRE is the fallback).
    With `handoff`, plain FIRE first runs every instance to max |F_i| <
    handoff, and the network then acts on that state before a fresh FIRE
    finishes.  Returns per-replica steps (both stretches summed), final
    energies and the device time of minimisation + inference."""
    from .ensemble import plane_fire_ensemble
    head_ms, head_steps = 0.0, np.zeros(len(insts), np.int64)
    if handoff is not None and net is not None:
        eng0 = plane_fire_ensemble(insts, k=k, dt=dt, dt_max=dt_max, fmax=handoff)
        eng0.build_nlist()
        head_steps, st0 = eng0.minimize(max_steps)
        head_ms = st0.device_ms
        insts = snapshot(eng0, insts)
        eng0.close()
    eng = plane_fire_ensemble(insts, k=k, dt=dt, dt_max=dt_max, fmax=fmax)
    eng.build_nlist()
    R = len(insts)
    start = torch.cuda.Event(enable_timing=True)
    mid = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    fallback = np.zeros(R, bool)
    if net is not None:
        eng.compute(dt)
        e0 = np.array([eng.energy(0, 0, r) for r in range(R)])
        box = net.box_array(eng)
        disp = net.forward(eng, box)
        net.apply(eng, box, disp)
        eng.compute(dt)
        e1 = np.array([eng.energy(0, 0, r) for r in range(R)])
        fallback = e1 > e0
        if fallback.any():
            restore_quench(eng, insts, np.nonzero(fallback)[0])
    mid.record()
    torch.cuda.synchronize()
    warm_ms = start.elapsed_time(mid)
    conv, st = eng.minimize(max_steps)
    energy = np.array([eng.energy(0, 0, r) for r in range(R)])
    steps = np.where((conv >= 0) & (head_steps >= 0), conv + head_steps, -1)
    out = dict(steps=steps, energy=energy, fire_ms=st.device_ms + head_ms, warm_ms=warm_ms, fallback=fallback,
               total_ms=warm_ms + st.device_ms + head_ms, head_ms=head_ms, head_steps=head_steps)
    eng.close()
    return out


# -- command line: the full train / evaluate pipeline --------------------------------------
def summarize(plain: dict, warm: dict, insts) -> dict:
    """Plain vs warm-started FIRE over the same instances."""
    ok = (plain["steps"] > 0) & (warm["steps"] > 0)
    rel = np.abs(warm["energy"] - plain["energy"]) / np.maximum(np.abs(plain["energy"]), 1e-300)
    signed = (warm["energy"] - plain["energy"]) / np.maximum(np.abs(plain["energy"]), 1e-300)
    n = np.array([len(p["x"]) for p, _ in insts])
    return dict(
        instances=len(insts), particles=int(n.sum()),
        plain_s=plain["total_ms"] / 1e3, warm_s=warm["total_ms"] / 1e3,
        speedup=plain["total_ms"] / warm["total_ms"],
        inference_ms=warm["warm_ms"],
        plain_steps_mean=float(plain["steps"][ok].mean()), warm_steps_mean=float(warm["steps"][ok].mean()),
        plain_steps_max=int(plain["steps"].max()), warm_steps_max=int(warm["steps"].max()),
        steps_ratio_median=float(np.median(plain["steps"][ok] / warm["steps"][ok])),
        steps_ratio_p10=float(np.percentile(plain["steps"][ok] / warm["steps"][ok], 10)),
        steps_ratio_p90=float(np.percentile(plain["steps"][ok] / warm["steps"][ok], 90)),
        handoff_steps_mean=float(np.mean(warm.get("head_steps", np.zeros(1)))),
        handoff_s=warm.get("head_ms", 0.0) / 1e3,
        unconverged_plain=int((plain["steps"] < 0).sum()), unconverged_warm=int((warm["steps"] < 0).sum()),
        fallback=int(warm["fallback"].sum()),
        energy_rel_diff_median=float(np.median(rel[ok])), energy_rel_diff_max=float(rel[ok].max()),
        energy_within_1e8=float(np.mean(rel[ok] < 1e-8)),
        energy_warm_lower_frac=float(np.mean(signed[ok] < 0)),
        energy_signed_rel_mean=float(signed[ok].mean()))


def main(argv=None) -> int:
    import argparse
    import json
    ap = argparse.ArgumentParser(description="learned FIRE warm start: train on GPU-FIRE relaxations, evaluate")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--count", type=int, default=2000)
    t.add_argument("--n", type=int, default=4096)
    t.add_argument("--per-engine", type=int, default=500)
    t.add_argument("--steps", type=int, default=2000)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--handoff", type=float, default=None,
                   help="train on hand-off states (max |F_i| first below this) instead of quenches")
    t.add_argument("--out", required=True)
    e = sub.add_parser("eval")
    e.add_argument("--params", required=True)
    e.add_argument("--count", type=int, default=512)
    e.add_argument("--seed", type=int, default=99)
    e.add_argument("--handoff", type=float, default=None, help="default: the value stored with the parameters")
    e.add_argument("--out")
    sw = sub.add_parser("sweep", help="hand-off sweep: per tolerance, train on hand-off states and evaluate")
    sw.add_argument("--handoffs", default="1e-2,1e-3,1e-4")
    sw.add_argument("--count", type=int, default=500)
    sw.add_argument("--steps", type=int, default=1000)
    sw.add_argument("--eval", type=int, default=128)
    pr = sub.add_parser("profile", help="a few training steps and one inference on one batch (for profilers)")
    pr.add_argument("--count", type=int, default=64)
    pr.add_argument("--n", type=int, default=4096)
    pr.add_argument("--steps", type=int, default=3)
    pr.add_argument("--fmax", type=float, default=1e-3, help="FIRE tolerance of the targets (loose: fast)")
    a = ap.parse_args(argv)
    if a.cmd == "sweep":
        data = quench_set(a.count + 64, 4096, 4096, 0.84, 0.90, seed=1)
        insts = quench_set(a.eval, 1024, 16384, 0.84, 0.90, seed=99)
        plain = relax(insts, None)
        for tau in (float(t) for t in a.handoffs.split(",")):
            net = WarmStartNet(seed=1)
            batches = [Batch(net, data[i:i + 500], handoff=tau) for i in range(0, a.count, 500)]
            held = Batch(net, data[a.count:], handoff=tau)
            hist = train(net, batches, a.steps)
            rep = dict(handoff=tau, loss_first=hist[0], loss_last=float(np.mean(hist[-5:])),
                       held_out_start_loss=mean_target_sq(held), held_out_loss=eval_loss(net, held))
            rep.update(summarize(plain, relax(insts, net, handoff=tau), insts))
            print(json.dumps(rep), flush=True)
        return 0
    if a.cmd == "profile":
        net = WarmStartNet(seed=1)
        b = Batch(net, quench_set(a.count, a.n, a.n, 0.84, 0.90, seed=5), fmax=a.fmax)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        for _ in range(a.steps):
            net.loss_and_grad(b.eng, b.box, b.target, b.n_valid)
            net.adam_step(1e-3)
        ev[1].record()
        net.forward(b.eng, b.box)
        ev[2].record()
        torch.cuda.synchronize()
        print(json.dumps(dict(slots=b.eng.view().slots, particles=b.n_valid,
                              train_step_ms=ev[0].elapsed_time(ev[1]) / a.steps,
                              inference_ms=ev[1].elapsed_time(ev[2]))), flush=True)
        return 0
    if a.cmd == "train":
        net = WarmStartNet(seed=a.seed)
        data = quench_set(a.count + 64, a.n, a.n, 0.84, 0.90, seed=a.seed)
        t0 = time.perf_counter()
        batches = [Batch(net, data[i:i + a.per_engine], handoff=a.handoff) for i in range(0, a.count, a.per_engine)]
        held = Batch(net, data[a.count:], handoff=a.handoff)
        gen_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        hist = train(net, batches, a.steps, log_every=max(1, a.steps // 10))
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t0
        net.save(a.out, handoff=a.handoff)
        rep = dict(relaxations=a.count, handoff=a.handoff, n=a.n, generation_s=gen_s, fire_device_s=sum(b.fire_device_ms for b in batches) / 1e3,
                   fire_steps_max=[int(b.conv.max()) for b in batches],
                   unconverged=int(sum((b.conv < 0).sum() for b in batches)), adam_steps=a.steps, train_s=train_s,
                   loss_first=hist[0], loss_last=float(np.mean(hist[-len(batches):])),
                   held_out_quench_loss=mean_target_sq(held), held_out_loss=eval_loss(net, held))
        print(json.dumps(rep), flush=True)
        return 0
    net = WarmStartNet()
    stored = net.load(a.params)
    handoff = a.handoff if a.handoff is not None else stored
    insts = quench_set(a.count, 1024, 16384, 0.84, 0.90, seed=a.seed)
    plain = relax(insts, None)
    warm = relax(insts, net, handoff=handoff)
    rep = summarize(plain, warm, insts)
    rep["handoff"] = handoff
    print(json.dumps(rep), flush=True)
    if a.out:
        np.savez(a.out, plain_steps=plain["steps"], warm_steps=warm["steps"], plain_energy=plain["energy"],
                 warm_energy=warm["energy"], fallback=warm["fallback"])
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
