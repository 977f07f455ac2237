"""Scenario surrogate: the CPU reference's gradients against finite differences,
the GPU network (BF16 tensor cores, FP32 accumulation) against that reference,
training, and what screening with the trained network gains over screening
without it, judged by the simulator."""
import numpy as np
import pytest

import surrogate_ref as ref


def _case(n, seed):
    rng = np.random.default_rng(seed)
    flat = ref.init_params(seed).astype(np.float64)
    flat += rng.normal(0.0, 0.02, flat.shape)          # non-zero biases too
    x = rng.random((n, ref.N_IN))
    target = rng.normal(0.0, 1.0, (n, ref.T_OUT, ref.N_OUT))
    return flat, x, target


def test_reference_gradients_match_finite_differences():
    flat, x, target = _case(3, 5)
    _, g = ref.loss_and_grads(flat, x, target)
    rng = np.random.default_rng(1)
    ofs = np.cumsum([0] + [o * i + o for _, (o, i) in ref.layer_shapes()])
    idx = np.concatenate([rng.choice(flat.size, 30, replace=False), ofs[:-1] + 3, ofs[1:] - 1])
    eps, rel = 1e-6, []
    for j in idx:
        f1, f2 = flat.copy(), flat.copy()
        f1[j] += eps
        f2[j] -= eps
        num = (ref.loss_and_grads(f1, x, target)[0] - ref.loss_and_grads(f2, x, target)[0]) / (2 * eps)
        rel.append(abs(num - g[j]) / max(abs(num) + abs(g[j]), 1e-9))
    # a coordinate next to a ReLU kink may differ; the bulk must agree to rounding
    assert np.median(rel) < 1e-7 and np.quantile(rel, 0.95) < 1e-3, (np.median(rel), max(rel))


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
def test_forward_matches_reference():
    from covidsim_b200 import surrogate
    flat, x, _ = _case(70, 7)                  # 70 rows: exercises the padding to 128
    net = surrogate.Surrogate(max_batch=128, params=flat.astype(np.float32))
    y = net.predict(x.astype(np.float32))
    y_ref = ref.forward(flat.astype(np.float32), x.astype(np.float32), round_bf16=True)
    # tolerance: accumulation order and the rare activation that rounds to the
    # neighbouring bfloat16 value
    assert _rel(y, y_ref) < 1e-2, _rel(y, y_ref)
    # more rows than one batch: the forward pass runs in batches
    y2 = net.predict(np.concatenate([x, x, x]).astype(np.float32))
    assert np.array_equal(y2[:70], y) and np.array_equal(y2[140:], y)
    net.close()


@pytest.mark.gpu
def test_gradients_match_reference():
    from covidsim_b200 import surrogate
    flat, x, target = _case(64, 9)
    net = surrogate.Surrogate(max_batch=64, params=flat.astype(np.float32))
    loss, g = net.loss_grad(x.astype(np.float32), target.astype(np.float32))
    loss_ref, g_ref = ref.loss_and_grads(flat.astype(np.float32), x.astype(np.float32), target.astype(np.float32),
                                         round_bf16=True)
    assert abs(loss - loss_ref) <= 1e-3 * abs(loss_ref)
    k = 0
    for name, (o, i) in ref.layer_shapes():
        for part, n in (("W", o * i), ("b", o)):
            e = _rel(g[k:k + n], g_ref[k:k + n])
            # gradients flow through bfloat16 activations and gradients
            assert e < 5e-2, (name, part, e)
            k += n
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 200])
def test_tcgen05_and_mma_sync_agree(n):
    """The two GEMM paths on the same BF16 operands: only FP32 summation order
    differs (n = 64 pads the batch to one 128-row tile half full; 200 to 256 rows)."""
    from covidsim_b200 import surrogate
    flat, x, target = _case(n, 11)
    out = {}
    for impl in ("tcgen05", "mma.sync"):
        net = surrogate.Surrogate(max_batch=256, params=flat.astype(np.float32))
        net.set_gemm(impl)
        y = net.predict(x.astype(np.float32))
        loss, g = net.loss_grad(x.astype(np.float32), target.astype(np.float32))
        out[impl] = (y, loss, g)
        net.close()
    (y1, l1, g1), (y2, l2, g2) = out["tcgen05"], out["mma.sync"]
    assert _rel(y1, y2) < 2e-3, _rel(y1, y2)
    assert abs(l1 - l2) <= 1e-4 * abs(l2)
    k = 0
    for name, (o, i) in ref.layer_shapes():
        for part, m in (("W", o * i), ("b", o)):
            e = _rel(g1[k:k + m], g2[k:k + m])
            assert e < 1e-2, (name, part, e)
            k += m


@pytest.mark.gpu
def test_ensemble_averages_members_on_the_natural_scale():
    from covidsim_b200 import surrogate
    x = np.random.default_rng(4).random((30, ref.N_IN)).astype(np.float32)
    ens = surrogate.Ensemble(3, max_batch=64, seed=7)
    members = [net.predict(x) for net in ens.nets]
    want = np.log1p(np.mean([np.expm1(p) for p in members], axis=0))
    assert np.allclose(ens.predict(x), want, rtol=1e-6, atol=1e-6)
    # distinct initial weights give distinct members
    assert not np.array_equal(members[0], members[1])
    ens.close()


@pytest.mark.gpu
def test_training_reduces_loss():
    from covidsim_b200 import surrogate
    rng = np.random.default_rng(3)
    x = rng.random((256, ref.N_IN)).astype(np.float32)
    t = np.arange(ref.T_OUT) / ref.T_OUT
    # smooth curves whose height, timing and width depend on the parameters
    amp = 1 + 3 * x[:, 0:1]
    mid = 0.2 + 0.5 * x[:, 1:2]
    wid = 0.05 + 0.1 * x[:, 2:3]
    curve = amp * np.exp(-((t[None, :] - mid) / wid) ** 2)
    y = np.stack([curve, 0.5 * curve, 0.2 * curve * x[:, 3:4], 0.1 * curve], axis=2).astype(np.float32)
    net = surrogate.Surrogate(max_batch=128, seed=1)
    hist = net.fit(x, y, epochs=60, lr=1e-3, batch=128)
    assert hist[-1] < 0.1 * hist[0], hist[::10]
    net.close()


@pytest.mark.gpu
def test_screening_with_surrogate_beats_screening_without():
    """Equal simulator budget: 8 scenarios chosen by the trained surrogate (lowest
    predicted critical-care peak among 2048 candidates) against 8 chosen without
    it (drawn at random from the same candidates); the simulator judges both."""
    from covidsim_b200 import surrogate, sim
    from tests.helpers import tiny_world
    pop, P, lk, hr = tiny_world()
    train = surrogate.sample_scenarios(48, seed=11)
    idx, ys = surrogate.simulate(pop, P, lk, hr, train, seeds_per=2, days=surrogate.DAYS, batch_size=48, n_seed=20)
    xs = surrogate.to_unit(train[idx]).astype(np.float32)
    net = surrogate.Surrogate(max_batch=128, seed=2)
    hist = net.fit(xs, ys, epochs=300, lr=1e-3, batch=96)
    assert hist[-1] < hist[0]
    cand = surrogate.sample_scenarios(2048, seed=12)
    pred = net.predict(surrogate.to_unit(cand).astype(np.float32))
    picked = np.argsort(pred[:, :, 2].max(axis=1))[:8]
    rand = np.random.default_rng(13).choice(len(cand), 8, replace=False)
    _, y_pick = surrogate.simulate(pop, P, lk, hr, cand[picked], seeds_per=2, batch_size=16, n_seed=20, seed0=5000)
    _, y_rand = surrogate.simulate(pop, P, lk, hr, cand[rand], seeds_per=2, batch_size=16, n_seed=20, seed0=5000)
    peak_pick = np.expm1(y_pick[:, :, 2]).max(axis=1).mean()
    peak_rand = np.expm1(y_rand[:, :, 2]).max(axis=1).mean()
    assert peak_pick < peak_rand, (peak_pick, peak_rand)
    net.close()
