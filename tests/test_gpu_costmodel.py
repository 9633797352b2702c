"""The learned cost model: GPU gradients against a float64 CPU oracle, training on the
GPU, and what the trained network gains over the default choice on real autotuner
timings (regret against exhaustive tuning)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def oracle_grads(params, dims, X, Y, M):
    """float64 forward/backward of the same network: in -> h -> h -> h (ReLU) -> out,
    loss = sum(mask * (pred - y)^2) / sum(mask). Parameter order per layer: W (out x in)
    then b."""
    p = params.astype(np.float64)
    layers, off = [], 0
    for l in range(len(dims) - 1):
        K, N = dims[l], dims[l + 1]
        W = p[off: off + N * K].reshape(N, K)
        off += N * K
        b = p[off: off + N]
        off += N
        layers.append((W, b))
    acts = [X.astype(np.float64)]
    for l, (W, b) in enumerate(layers):
        z = acts[-1] @ W.T + b
        acts.append(np.maximum(z, 0) if l + 1 < len(layers) else z)
    cnt = M.sum()
    d = (acts[-1] - Y) * M
    loss = float((d * d).sum() / cnt)
    g = 2 * d / cnt
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        W, b = layers[l]
        grads.append((g.T @ acts[l], g.sum(axis=0)))
        if l:
            g = (g @ W) * (acts[l] > 0)
    flat = []
    for dW, db in reversed(grads):
        flat += [dW.ravel(), db.ravel()]
    return np.concatenate(flat), loss


def test_gradients_match_float64_oracle(gpu):
    from reed_solomon_b200 import tuner

    m = tuner.CostModel(hidden=64, seed=3)
    rng = np.random.default_rng(0)
    B = 97
    X = rng.normal(size=(B, tuner.N_FEATURES)).astype(np.float32)
    Y = rng.normal(size=(B, len(tuner.CONFIGS))).astype(np.float32)
    M = (rng.random((B, len(tuner.CONFIGS))) < 0.7).astype(np.float32)
    g, loss = m.gradients(X, Y, M)
    dims = [tuner.N_FEATURES, 64, 64, 64, len(tuner.CONFIGS)]
    want, want_loss = oracle_grads(m.params(), dims, X, Y, M)
    assert abs(loss - want_loss) <= 1e-4 * max(1.0, abs(want_loss))
    # FP32 accumulation against float64: relative to the gradient's scale.
    scale = np.abs(want).max()
    assert np.abs(g - want).max() <= 2e-4 * scale, np.abs(g - want).max() / scale


def test_training_reduces_loss(gpu):
    from reed_solomon_b200 import tuner

    rng = np.random.default_rng(1)
    X = rng.random((2048, tuner.N_FEATURES)).astype(np.float32)
    # A smooth synthetic cost surface, positive "times".
    T = np.exp(X @ rng.normal(size=(tuner.N_FEATURES, len(tuner.CONFIGS))) * 0.8
               + np.sin(3 * X[:, :1]))
    T[:, 5] = np.nan
    m = tuner.CostModel(hidden=64, seed=2)
    hist = m.fit(X, T, epochs=60, lr=3e-3, batch=256)
    assert hist[-1] < 0.1 * hist[0], hist[:: max(1, len(hist) // 6)]
    choice = m.choose(X, T)
    assert np.all(np.isfinite(T[np.arange(len(T)), choice]))


def test_model_gains_over_default_on_tuner_timings(gpu):
    """Exhaustive tuning of sampled workloads, train on most, judge regret on the rest."""
    from reed_solomon_b200 import tuner

    work = tuner.sample_workloads(160, seed=11, max_bytes=8 << 20)
    X, T = tuner.collect(work, reps=2)
    tr, te = slice(0, 120), slice(120, 160)
    m = tuner.CostModel(hidden=64, seed=5)
    m.fit(X[tr], T[tr], epochs=300, lr=3e-3, batch=64)
    r_model = tuner.regret(T[te], m.choose(X[te], T[te]))
    r_default = tuner.regret(T[te], tuner.default_choice(work[te], T[te]))
    print("held-out regret: model %.3f, default %.3f" % (r_model, r_default))
    assert r_model <= r_default + 0.02
