"""The learned FIRE warm start: its CUDA forward/backward kernels against the
float64 CPU reference network (oracle/warmstart_ref.py), the reference's own
backward pass against finite differences, and what training buys over the
quench it starts from."""
import numpy as np
import pytest

from oracle import warmstart_ref as W


def small_system(n=60, phi=0.86, seed=5):
    from samos_b200.ensemble import quench_disks
    parts, L = quench_disks(n, phi, seed)
    return parts, L


def test_bf16_rounding_known_answers():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 1.0 + 2.0 ** -8 + 2.0 ** -20])
    want = np.array([1.0, 1.0, 1.0 + 2.0 ** -6, 1.0, -2.5, 1.0 + 2.0 ** -7])
    np.testing.assert_array_equal(W.bf16_round(x), want)


def test_reference_backward_matches_finite_differences():
    parts, L = small_system()
    n = len(parts["x"])
    I, J, e, u = W.edges(parts["x"], parts["y"], parts["radius"], L, 2.8)
    assert len(I) > 4 * n
    rng = np.random.default_rng(1)
    p = rng.normal(0.0, 0.2, W.NPARAM)
    target = rng.normal(0.0, 0.3, (n, 2))
    loss, _, g = W.Net(p, bf16=False).loss_and_grad(n, I, J, e, u, target, 1.0 / n)
    assert loss == pytest.approx(W.loss_only(p, n, I, J, e, u, target, 1.0 / n))
    idx = np.concatenate([rng.choice(W.NPARAM, 48, replace=False), [W.NPARAM - 1, 0, 300, 4500, 12700]])
    h = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (W.loss_only(pp, n, I, J, e, u, target, 1.0 / n) - W.loss_only(pm, n, I, J, e, u, target, 1.0 / n)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(g[k])), (k, fd, g[k])


def _ref_for_engine(eng, net_params, insts, targets):
    """Reference loss, per-replica displacements (id order) and gradient,
    summed over the replicas with the engine's 1/n normalisation."""
    n_valid = sum(len(p["x"]) for p, _ in insts)
    loss, disps, grad = 0.0, [], np.zeros(W.NPARAM)
    for (parts, L), t in zip(insts, targets):
        x, y = eng.download("x", len(disps)), eng.download("y", len(disps))
        I, J, e, u = W.edges(x, y, parts["radius"], L, 2.8)
        l, d, g = W.Net(net_params, bf16=True).loss_and_grad(len(x), I, J, e, u, t, 1.0 / n_valid)
        loss += l
        disps.append(d)
        grad += g
    return loss, disps, grad


@pytest.mark.gpu
def test_gpu_forward_backward_match_cpu_reference():
    import torch
    from samos_b200.ensemble import plane_fire_ensemble, quench_disks
    from samos_b200.warmstart import OFF, WarmStartNet

    insts = [quench_disks(300, 0.86, 11), quench_disks(210, 0.89, 12)]
    eng = plane_fire_ensemble(insts)
    eng.build_nlist()
    net = WarmStartNet(seed=3)
    rng = np.random.default_rng(4)
    p = net.get_params()
    p[OFF["w2"][0]:OFF["w2"][0] + 64] = rng.normal(0.0, 0.3, 64)  # larger output layer than the init
    p[OFF["c"][0]] = 0.05
    net.set_params(p)
    targets = [rng.normal(0.0, 0.3, (len(pp["x"]), 2)) for pp, _ in insts]
    box = net.box_array(eng)
    tgt = net.slot_targets(eng, targets)
    n_valid = sum(len(pp["x"]) for pp, _ in insts)
    loss = net.loss_and_grad(eng, box, tgt, n_valid)
    g_gpu = net.grad.cpu().numpy().astype(np.float64)
    disp = net._work(eng.view().slots)["disp"].cpu().numpy().reshape(-1, 2).astype(np.float64)
    ids = net.slot_ids(eng)

    ref_loss, ref_disp, g_ref = _ref_for_engine(eng, p.astype(np.float64), insts, targets)
    for r, d_ref in enumerate(ref_disp):
        off, n = eng.replica_slots(r)
        d_gpu = np.zeros_like(d_ref)
        d_gpu[ids[off:off + n]] = disp[off:off + n]
        err = np.linalg.norm(d_gpu - d_ref) / np.linalg.norm(d_ref)
        assert err < 5e-3, (r, err)
    assert loss == pytest.approx(ref_loss, rel=5e-3)
    for name, (o, s) in OFF.items():
        size = int(np.prod(s))
        a, b = g_gpu[o:o + size], g_ref[o:o + size]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 2e-2, (name, err)
    # padding slots stay untouched by the apply kernel and displacements are finite
    assert np.isfinite(disp).all()
    eng.close()


@pytest.mark.gpu
def test_training_beats_the_quench_on_held_out_systems():
    from samos_b200.warmstart import Batch, WarmStartNet, eval_loss, mean_target_sq, quench_set, train

    net = WarmStartNet(seed=0)
    data = quench_set(40, 1024, 1024, 0.84, 0.90, seed=21)
    batches = [Batch(net, data[i:i + 8]) for i in range(0, 32, 8)]
    held = Batch(net, data[32:40])
    assert all((b.conv > 0).all() for b in batches + [held]), "FIRE did not converge"
    base = mean_target_sq(held)
    before = eval_loss(net, held)
    hist = train(net, batches, 300, lr=2e-3, lr_end=2e-4)
    after = eval_loss(net, held)
    assert np.isfinite(hist).all()
    assert after < 0.8 * base, (before, after, base)
