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


def test_shipped_model_gains_over_default_on_held_out_timings(gpu):
    """The shipped cost model (cost_model.rsmlp, trained on this library's autotuner
    timings) against the default choice on fresh workloads it was not trained on
    (another seed), both judged by regret against exhaustive tuning of the same
    timings: the model's regret is at most 5% and below the default's."""
    from reed_solomon_b200 import tuner

    model = tuner.shipped_model()
    assert model is not None, "the shipped cost model is missing"
    work = tuner.sample_workloads(150, seed=9001, max_bytes=8 << 20)
    X, T = tuner.collect(work, reps=3)
    r_model = tuner.regret(T, model.choose(X, T))
    r_default = tuner.regret(T, tuner.default_choice(work, T))
    print("held-out regret: model %.4f, default %.4f" % (r_model, r_default))
    assert r_model <= 0.05
    assert r_model < r_default


def test_batch_with_model_choice_is_bit_exact(gpu, O):
    """Launch configurations chosen by the model (rs_batch_choose) or forced per item
    (rs_batch_create_configured) change kernels, never bytes: a mixed batch under the
    model's choice, under every FFT configuration and on the matrix route gives the
    default batch's bytes, which match the oracle."""
    import torch

    from reed_solomon_b200 import tuner

    rng = np.random.default_rng(12)
    shapes = [(32, 32), (16, 16), (10, 10), (7, 13), (20, 30)]
    specs = []
    for i in range(40):
        k, m = shapes[i % len(shapes)]
        S = int(rng.integers(64, 5000)) if i % 3 else int(rng.integers(4, 300)) * 16
        specs.append((k, m, S, S if i % 4 == 3 else (S + 15) // 16 * 16))  # every 4th packed (unaligned)
    codecs = {sh: gpu.ReedSolomon(*sh) for sh in shapes}

    def make():
        g = torch.Generator(device="cuda").manual_seed(5)
        return [torch.randint(0, 256, ((k + m) * st,), dtype=torch.uint8, device="cuda", generator=g)
                for k, m, S, st in specs]

    def items(rows):
        return [(codecs[(k, m)], r, st, S, gpu.ENCODE, None) for (k, m, S, st), r in zip(specs, rows)]

    base = make()
    b = gpu.Batch(items(base))
    b.launch()
    torch.cuda.synchronize()
    for (k, m, S, st), r in zip(specs[:6], base[:6]):
        stripe = r.view(k + m, st)[:, :S].cpu().numpy()
        assert np.array_equal(stripe[k:], O.encode8(k, m, stripe[:k]))
    variants = [{"model": tuner.shipped_model()}]
    for c, (route, _) in enumerate(tuner.CONFIGS):
        cfgs = []
        for k, m, S, st in specs:
            fft = k == m and k in tuner.FFT_K
            gen = (k, m) in tuner.GEN_SHAPES
            ok = route == "matrix" or (route == "fft" and fft) or (route == "gen" and gen)
            cfgs.append(c if ok else -1)
        variants.append({"configs": cfgs})
    for kw in variants:
        rows = make()
        bb = gpu.Batch(items(rows), **kw)
        assert bb.statuses == [0] * len(specs)
        bb.launch()
        torch.cuda.synchronize()
        for r0, r1 in zip(base, rows):
            assert torch.equal(r0, r1), kw.get("configs")
