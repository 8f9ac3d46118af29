"""The learned launch planner: its network's CUDA kernels against a CPU
restatement (gradients, training, prediction), and what the trained planner
gains over the default launch on measured timings, with its regret against
exhaustive autotuning."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def cpu_forward_backward(p, x, t, D, H):
    """float64 restatement: L = (1/2n) sum (y - t)^2, y = w2 . relu(W1 x + b1) + b2."""
    p = p.astype(np.float64)
    W1 = p[: H * D].reshape(H, D)
    b1 = p[H * D: H * D + H]
    w2 = p[H * D + H: H * D + 2 * H]
    b2 = p[-1]
    x = x.astype(np.float64)
    z = x @ W1.T + b1
    h = np.maximum(z, 0.0)
    y = h @ w2 + b2
    n = len(t)
    r = y - t
    loss = 0.5 * np.sum(r * r) / n
    dy = r / n
    dz = (dy[:, None] * w2[None, :]) * (z > 0)
    grad = np.concatenate([(dz.T @ x).ravel(), dz.sum(0), h.T @ dy, [dy.sum()]])
    return loss, grad, y


def test_gradients_match_the_cpu_restatement(gpu):
    from zindex_b200.planner import Mlp

    rng = np.random.default_rng(0)
    D, H = 20, 32
    net = Mlp(D, H, seed=3)
    p = net.params()
    assert len(p) == H * D + 2 * H + 1
    for n in (1, 63, 64, 65, 1000):
        x = rng.normal(size=(n, D)).astype(np.float32)
        t = rng.normal(size=n).astype(np.float32)
        loss, g = net.loss_grad(x, t)
        want_loss, want_g, _ = cpu_forward_backward(p, x, t, D, H)
        # FP32 kernels against float64: relative 1e-4 of the gradient scale.
        np.testing.assert_allclose(loss, want_loss, rtol=1e-5)
        np.testing.assert_allclose(g, want_g, rtol=1e-4, atol=1e-4 * np.abs(want_g).max())
    # The CPU restatement itself, by central differences in float64.
    x = rng.normal(size=(50, D)).astype(np.float32)
    t = rng.normal(size=50).astype(np.float32)
    _, g64, _ = cpu_forward_backward(p, x, t, D, H)
    for q in rng.choice(len(p), 25, replace=False):
        e = np.zeros(len(p))
        e[q] = 1e-6
        lp = cpu_forward_backward(p + e, x, t, D, H)[0]
        lm = cpu_forward_backward(p - e, x, t, D, H)[0]
        assert abs((lp - lm) / 2e-6 - g64[q]) <= 1e-6 + 1e-4 * abs(g64[q])


def test_training_fits_and_prediction_matches_cpu(gpu):
    from zindex_b200.planner import Mlp

    rng = np.random.default_rng(1)
    D, H = 4, 32
    x = rng.uniform(-1, 1, size=(2000, D)).astype(np.float32)
    t = (np.sin(2 * x[:, 0]) + x[:, 1] ** 2 - 0.5 * x[:, 2]).astype(np.float32)
    net = Mlp(D, H, seed=5)
    start, _ = net.loss_grad(x, t)
    final = net.train(x, t, epochs=3000, lr=3e-3)
    assert final < 0.05 * start
    _, _, y = cpu_forward_backward(net.params(), x, t, D, H)
    np.testing.assert_allclose(net.predict(x), y, rtol=1e-4, atol=1e-4)


def test_planner_gain_over_default_and_regret(gpu):
    """Leave-one-setting-out on the committed autotuner measurements: for each
    setting the planner is trained on the other settings' timings only, ranks
    that setting's launches, and its shortlist (3 predictions and the default)
    is scored with the measured times against the exhaustive best over all
    candidates (regret) and the default launch (gain); the cut decision is
    scored the same way on the end-to-end rows."""
    from zindex_b200 import planner as pl

    rows, defaults = pl.load_rows()
    settings = sorted({r.setting for r in rows})
    assert len(settings) >= 8
    dev, e2e = [], []
    for held in settings:
        p = pl.Planner(seed=7)
        p.fit([r for r in rows if r.setting != held])
        test = [r for r in rows if r.setting == held]
        dev.append(pl.evaluate(p, test, defaults[held]))
        e2e.append(pl.evaluate(p, test, defaults[held], e2e=True))
    gm = lambda v: float(np.exp(np.mean(np.log(v))))
    gain = gm([r["gain_over_default"] for r in dev])
    regret = gm([1 + r["regret"] for r in dev]) - 1
    top1 = gm([r["top1_gain_over_default"] for r in dev])
    timed = float(np.mean([r["timed_per_setting"] for r in dev]))
    cands = float(np.mean([r["candidates_per_setting"] for r in dev]))
    e2e_gain = gm([r["gain_over_default"] for r in e2e])
    guarded = gm([r["top1_guarded_gain_over_default"] for r in dev])
    rand = gm([r["random_shortlist_gain_over_default"] for r in dev])
    heur = gm([r["heuristic_shortlist_gain_over_default"] for r in dev])
    wide = gm([r["network_over_all_launches_gain_over_default"] for r in dev])
    nearby = gm([r["top1_nearby_guarded_gain_over_default"] for r in dev])
    print(f"launch: gain over the default {gain:.3f}, regret {regret:.3f} with {timed:.1f} of "
          f"{cands:.0f} candidates timed (network ranking every launch: {wide:.3f}; its top "
          f"pick alone, untimed: {top1:.3f}, guarded by a {pl.TOP1_MARGIN:.0%} margin: "
          f"{guarded:.3f}; among the default's {pl.POOL} nearest, guarded: {nearby:.3f}); "
          f"the same budget without the network: random shortlist {rand:.3f}, "
          f"nearest-to-default shortlist {heur:.3f}; cut: gain over the default {e2e_gain:.3f}")
    # What the network earns: its shortlist (ranking the default's
    # neighbourhood) against untrained shortlists of the same size, all of
    # which also time the default.
    assert gain > rand
    assert gain >= heur - 0.01
    # Untimed, the planner's own pick (the default's neighbourhood, kept only
    # when predicted faster by the margin) does not lose to the default.
    assert nearby >= 1.0
    # The default launch is itself fitted to these measurements, so the gain
    # is over a strong baseline; the shortlist can only match or beat it.
    assert gain >= 1.02
    assert regret <= 0.08
    assert timed <= 4.0 and cands >= 40
    assert e2e_gain >= 1.0
