"""Autotuner and learned cost model for route and tile choice.

The autotuner times every candidate launch configuration of a workload on the GPU
(exhaustive tuning); those timings train the cost model, an FP32 MLP trained and run by
this library's CUDA kernels (rs_mlp_*), which then predicts the best configuration for
unseen workloads without timing them. Configurations only choose kernels and launch
shapes, never arithmetic, so every choice yields the same bytes.

Candidates (GF(2^8)):
  matrix route, tile variant 0..3 (parity rows per thread x output rows per CTA)
  FFT route ((K,K) shapes), lane-group width narrow/wide x launch shape (threads x CTAs
  per SM) 128x3 / 128x4 / 128x2 / 256x1
  generator route (the compiled generator kernel of (7,13), (10,10), (14,14), (18,6),
  (20,12) and the storage codes (4,2), (6,3), (8,4), (10,4), (12,4), (16,4), (17,3))
"""
import ctypes
import math
import os

import numpy as np

from . import _lib
from .coder import ReedSolomon, _check

CONFIGS = [("matrix", 0), ("matrix", 1), ("matrix", 2), ("matrix", 3),
           ("fft", (0, 0)), ("fft", (0, 1)), ("fft", (1, 0)), ("fft", (1, 1)),
           ("fft", (0, 2)), ("fft", (1, 2)), ("fft", (0, 3)), ("fft", (1, 3)), ("gen", 0)]
N_FEATURES = 6
MAX_BATCH_LOG2 = 9  # stripes per timed launch: 1 .. 512 (the library clamps the feature there)
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cost_model.rsmlp")
TIMINGS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cost_model_timings.npz")
FFT_K = (2, 4, 8, 16, 32, 64, 128)
GEN_SHAPES = ((7, 13), (10, 10), (14, 14), (18, 6), (20, 12), (4, 2), (6, 3), (8, 4), (10, 4), (12, 4),
              (16, 4), (17, 3))


class Workload:
    """k data + m parity shards of `shard_bytes`, `erasures` rebuilt per stripe
    (0 = encode), `batch` stripes per launch."""

    def __init__(self, k, m, shard_bytes, erasures=0, batch=1):
        self.k, self.m, self.shard_bytes, self.erasures, self.batch = k, m, shard_bytes, erasures, batch

    def aligned(self):
        """Rows are packed shard_bytes apart, so they are 16-byte aligned iff that is."""
        return self.shard_bytes % 16 == 0

    def features(self):
        """As the library computes them (tuning.hpp tune_features)."""
        batch = min(max(self.batch, 1), 1 << MAX_BATCH_LOG2)
        return [math.log2(self.k) / 8.0, math.log2(self.m) / 8.0, math.log2(self.shard_bytes) / 20.0,
                self.erasures / max(self.m, 1), math.log2(batch) / 8.0, 0.0 if self.aligned() else 1.0]

    def bytes(self):
        return self.batch * self.shard_bytes * (self.k + (self.erasures or self.m))

    def __repr__(self):
        return "Workload(k=%d, m=%d, bytes=%d, erasures=%d, batch=%d)" % (
            self.k, self.m, self.shard_bytes, self.erasures, self.batch)


def applicable(w, cfg):
    route, _ = cfg
    if route == "fft":
        return w.erasures == 0 and w.k == w.m and w.k in FFT_K and w.shard_bytes >= 64
    if route == "gen":
        return w.erasures == 0 and (w.k, w.m) in GEN_SHAPES and w.shard_bytes >= 64
    return True


def apply_config(codec, w, cfg):
    """Set the library's tuning hooks for `cfg`."""
    L = _lib.load()
    route, v = cfg
    if route == "matrix":
        codec.set_route("matrix")
        L.rs_set_matrix_variant(v)
    elif route == "gen":
        codec.set_route("fft")  # the shape's compiled kernel
    else:
        codec.set_route("fft")
        L.rs_set_fft_lanes(w.k, v[0])
        L.rs_set_fft_variant(w.k, v[1])


class Bench:
    """Device buffers and a timing loop for one workload."""

    def __init__(self, w, seed=0):
        import torch

        self.w = w
        self.codec = ReedSolomon(w.k, w.m)
        g = torch.Generator(device="cuda").manual_seed(seed)
        n = w.k + w.m
        self.rows = torch.randint(0, 256, (w.batch, n, w.shard_bytes), dtype=torch.uint8, device="cuda",
                                  generator=g)
        self.present = None
        if w.erasures:
            rng = np.random.default_rng(seed)
            self.present = np.ones((w.batch, n), np.uint8)
            for s in range(w.batch):
                self.present[s, rng.choice(n, size=w.erasures, replace=False)] = 0

    def run(self):
        w = self.w
        if w.erasures:
            self.codec.reconstruct_batch_dev(self.rows, w.batch, w.shard_bytes, self.present)
        else:
            stride = (w.k + w.m) * w.shard_bytes
            parity = self.rows[:, w.k:]
            self.codec.encode_batch_dev(self.rows, parity, w.shard_bytes, w.batch, data_stride=stride,
                                        parity_stride=stride)

    def time(self, cfg, reps=3):
        import torch

        apply_config(self.codec, self.w, cfg)
        self.run()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.run()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best


def reset_defaults():
    """Back to the library's automatic choices."""
    L = _lib.load()
    L.rs_set_matrix_variant(0)
    for k in DEFAULT_FFT:
        L.rs_set_fft_lanes(k, -1)
        L.rs_set_fft_variant(k, -1)


def exhaustive(w, reps=3, seed=0):
    """Time every applicable configuration: (times in ms per config, NaN if n/a)."""
    b = Bench(w, seed)
    t = np.full(len(CONFIGS), np.nan)
    for i, cfg in enumerate(CONFIGS):
        if applicable(w, cfg):
            t[i] = b.time(cfg, reps)
    reset_defaults()
    return t


def sample_workloads(n, seed, max_bytes=64 << 20):
    """GF(2^8) workloads spread like the serving mix: k log-uniform, shard bytes
    log-uniform 512 B .. 1 MiB (half of them rounded to a multiple of 16, so that rows
    packed back to back are 16-byte aligned), a quarter reconstruct; (K,K) power-of-two
    shapes over-sampled so the FFT candidates are exercised."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        u = rng.random()
        if u < 0.4:
            k = int(rng.choice([16, 32, 64, 128]))
            m = k
        elif u < 0.5:
            k, m = GEN_SHAPES[int(rng.integers(0, len(GEN_SHAPES)))]
        else:
            k = int(math.exp(rng.uniform(math.log(4), math.log(200))))
            m = int(rng.integers(2, min(3 * k, 256 - k) + 1)) if 256 - k >= 2 else 1
            if k + m > 256 or m < 1:
                continue
        shard = int(math.exp(rng.uniform(math.log(512), math.log(1 << 20))))
        if rng.random() < 0.5:  # half on 16-byte aligned rows (as separately allocated shards are)
            shard = max(16, shard // 16 * 16)
        erasures = int(rng.integers(1, m + 1)) if rng.random() < 0.25 else 0
        batch = int(2 ** rng.integers(0, MAX_BATCH_LOG2 + 1))
        w = Workload(k, m, shard, erasures, batch)
        while w.bytes() > max_bytes and w.batch > 1:
            w.batch //= 2
        if w.bytes() > max_bytes:
            continue
        out.append(w)
    return out


def collect(workloads, reps=3):
    X = np.array([w.features() for w in workloads], np.float32)
    T = np.stack([exhaustive(w, reps, seed=i) for i, w in enumerate(workloads)])
    return X, T


class CostModel:
    """FP32 MLP on the GPU (rs_mlp_*): features -> log(ms) per configuration."""

    def __init__(self, hidden=64, seed=1, path=None):
        self._L = _lib.load()
        h = ctypes.c_void_p()
        if path is not None:
            _check(self._L.rs_mlp_load(os.fsencode(path), ctypes.byref(h)))
        else:
            _check(self._L.rs_mlp_create(N_FEATURES, hidden, len(CONFIGS), seed, ctypes.byref(h)))
        self._h = h

    def save(self, path):
        _check(self._L.rs_mlp_save(self._h, os.fsencode(path)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.rs_mlp_free(h)

    def n_params(self):
        return self._L.rs_mlp_param_count(self._h)

    def params(self):
        out = np.zeros(self.n_params(), np.float32)
        _check(self._L.rs_mlp_get_params(self._h, out.ctypes.data, out.size))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(self._L.rs_mlp_set_params(self._h, p.ctypes.data, p.size))

    @staticmethod
    def _targets(T):
        mask = np.isfinite(T).astype(np.float32)
        Y = np.where(mask > 0, np.log(np.where(mask > 0, T, 1.0)), 0.0).astype(np.float32)
        return Y, mask

    def gradients(self, X, Y, mask):
        import torch

        x, y, mk = (torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda() for a in (X, Y, mask))
        g = np.zeros(self.n_params(), np.float32)
        loss = ctypes.c_float()
        _check(self._L.rs_mlp_gradients(self._h, x.data_ptr(), y.data_ptr(), mk.data_ptr(), x.shape[0],
                                        float(mask.sum()), g.ctypes.data, g.size, ctypes.byref(loss)))
        return g, loss.value

    def fit(self, X, T, epochs=400, lr=3e-3, batch=512, seed=0):
        import torch

        Y, mask = self._targets(T)
        x = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
        y = torch.from_numpy(Y).cuda()
        mk = torch.from_numpy(mask).cuda()
        rng = np.random.default_rng(seed)
        n = x.shape[0]
        loss = ctypes.c_float()
        history = []
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(n)).cuda()
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                xb, yb, mb = x[idx].contiguous(), y[idx].contiguous(), mk[idx].contiguous()
                _check(self._L.rs_mlp_train_step(self._h, xb.data_ptr(), yb.data_ptr(), mb.data_ptr(), xb.shape[0],
                                                 float(mb.sum().item()), lr, ctypes.byref(loss)))
            history.append(loss.value)
        return history

    def predict(self, X):
        import torch

        x = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
        out = torch.empty((x.shape[0], len(CONFIGS)), dtype=torch.float32, device="cuda")
        _check(self._L.rs_mlp_predict(self._h, x.data_ptr(), x.shape[0], out.data_ptr()))
        return out.cpu().numpy()

    def choose(self, X, T):
        """Index of the predicted-fastest applicable configuration per row (T gives
        applicability: NaN = not applicable)."""
        P = self.predict(X)
        P = np.where(np.isfinite(T), P, np.inf)
        return P.argmin(axis=1)


def shipped_model():
    """The cost model trained on this library's autotuner timings (cost_model.rsmlp,
    made by `bench.py --workload tuner --save-model`), or None when absent."""
    return CostModel(path=MODEL_PATH) if os.path.exists(MODEL_PATH) else None


def library_configs():
    """The library's configuration table (rs_tuning_config), as CONFIGS spells it."""
    L = _lib.load()
    out = []
    for i in range(L.rs_tuning_config_count()):
        r, a, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(L.rs_tuning_config(i, ctypes.byref(r), ctypes.byref(a), ctypes.byref(b)))
        out.append(("matrix", a.value) if r.value == 0 else ("fft", (a.value, b.value)) if r.value == 1
                   else ("gen", 0))
    return out


DEFAULT_FFT = {2: (0, 0), 4: (0, 1), 8: (0, 1), 16: (0, 1), 32: (0, 3), 64: (0, 3), 128: (1, 3)}
# The library's automatic choice on rows that are not 16-byte aligned (K >= 16).
UNALIGNED_FFT = {16: (1, 1), 32: (1, 1), 64: (1, 1), 128: (1, 1)}


def default_choice(workloads, T):
    """The method without the model: the library's default route and tile (the FFT
    kernel with its launch shape for the rows' alignment, or the generator kernel,
    where the shape has one, else matrix tile 0)."""
    out = np.zeros(len(workloads), np.int64)
    for i, w in enumerate(workloads):
        if applicable(w, ("fft", (0, 0))) and np.isfinite(T[i, 4]):
            aligned = w.shard_bytes % 16 == 0  # rows packed shard_bytes apart
            out[i] = CONFIGS.index(("fft", DEFAULT_FFT[w.k] if aligned or w.k < 16 else UNALIGNED_FFT[w.k]))
        elif applicable(w, ("gen", 0)):
            out[i] = CONFIGS.index(("gen", 0))
    return out


def regret(T, choice):
    """Mean of time(chosen) / time(best) - 1 over workloads."""
    best = np.nanmin(T, axis=1)
    chosen = T[np.arange(len(T)), choice]
    return float(np.mean(chosen / best - 1.0))
