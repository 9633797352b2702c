"""Measured workloads beyond the RS(32,32) encode headline: one function per workload,
each returning a dict that bench.py prints as one JSON line.

All inputs are seeded synthetic bytes generated on the device. Times are CUDA-event
times on the launching stream after warm-up, except where a workload is defined by
host-side arrival times (the Poisson request stream), which uses the host monotonic
clock the server stamps its completions with. Algorithmic bytes: (k+m)*S per encoded
stripe, (k+e)*S per reconstructed stripe rebuilding e shards.
"""
import math
import time

import numpy as np

from . import _lib
from .coder import ENCODE, MATRIX_ONLY, RECONSTRUCT, Batch, ReedSolomon, ReedSolomon16, _dev_ptr

MIXED_SHAPES = [(7, 13), (10, 10), (14, 14), (16, 16), (18, 6), (32, 32), (20, 12), (64, 64), (128, 128)]


def _events():
    import torch

    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _time(fn, reps, warmup=1):
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = _events()
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / 1e3 / reps


def _erasures(rng, n, m):
    present = np.ones(n, np.uint8)
    present[rng.choice(n, size=int(rng.integers(1, m + 1)), replace=False)] = 0
    return present


# ---- RS(32,32) / RS(16,16) encode and reconstruct, 4096 stripes per launch ----

def stripes_sweep(shapes=((32, 32), (16, 16)), sizes=(4096, 65536, 1 << 20), n_stripes=4096, seed=2,
                  wave_bytes=24 << 30, reps=3):
    """Encode on the FFT and matrix routes and reconstruct with an independent erasure
    pattern of 1..m shards per stripe. Launches larger than `wave_bytes` run in waves
    over the same device buffers (4096 x 64 x 1 MiB is 256 GiB)."""
    import torch

    rng = np.random.default_rng(seed)
    out = []
    for k, m in shapes:
        n = k + m
        rs = ReedSolomon(k, m)
        for S in sizes:
            wave = max(1, min(n_stripes, wave_bytes // (n * S)))
            waves = (n_stripes + wave - 1) // wave
            g = torch.Generator(device="cuda").manual_seed(seed + S)
            rows = torch.randint(0, 256, (wave, n, S), dtype=torch.uint8, device="cuda", generator=g)
            stride = n * S
            res = {"k": k, "m": m, "shard_bytes": S, "stripes": n_stripes, "stripes_per_launch": wave,
                   "launches": waves}
            for route in ("fft", "matrix"):
                rs.set_route(route)

                def enc():
                    for _ in range(waves):
                        rs.encode_batch_dev(rows, rows[:, k:], S, wave, data_stride=stride, parity_stride=stride)

                t = _time(enc, reps)
                res["encode_%s_gbs" % route] = waves * wave * n * S / t / 1e9
            rs.set_route("auto")
            res["encode_route"] = rs.encode_route(S)  # what the "fft" (compiled) timing ran
            rs.encode_batch_dev(rows, rows[:, k:], S, wave, data_stride=stride, parity_stride=stride)
            full = rows.clone()
            present = np.stack([_erasures(rng, n, m) for _ in range(wave)])
            mask = torch.from_numpy(present).cuda().bool()
            erased = int((present == 0).sum())

            def rec():
                for _ in range(waves):
                    rs.reconstruct_batch_dev(rows, wave, S, present)

            rows.mul_(mask[:, :, None])  # erase
            t = _time(rec, reps)
            res["reconstruct_gbs"] = waves * (wave * k + erased) * S / t / 1e9
            res["reconstruct_bit_exact"] = bool(torch.equal(rows, full))
            out.append(res)
            del rows, full
            torch.cuda.empty_cache()
    return out


# ---- mixed batch: 10,000 stripes of nine shapes, 25% reconstruct ----

def mixed_batch(n=10000, seed=3, reps=5, packed=False, tuned_compare=True):
    """Batched+tuned (one graph: one compiled-kernel launch per FFT or generator shape + one
    ragged matrix launch) against
    the plain path (one matrix-kernel call per stripe; reconstructs build their decode
    rows per call), same stripes."""
    import torch

    rng = np.random.default_rng(seed)
    codecs = {s: ReedSolomon(*s) for s in MIXED_SHAPES}
    specs = []
    off = 0
    for _ in range(n):
        k, m = MIXED_SHAPES[int(rng.integers(len(MIXED_SHAPES)))]
        S = int(math.exp(rng.uniform(math.log(1024), math.log(1 << 20))))
        op = RECONSTRUCT if rng.random() < 0.25 else ENCODE
        present = _erasures(rng, k + m, m) if op == RECONSTRUCT else None
        # Each shard starts on a 16-byte boundary, as separately allocated shard buffers
        # do; its length S is any integer (most are not multiples of 16 or 64). With
        # `packed` the rows lie back to back at S apart, so most rows start unaligned.
        stride = S if packed else (S + 15) & ~15
        specs.append((k, m, S, stride, op, present, off))
        off += ((k + m) * stride + 255) & ~255
    pool = torch.empty(off, dtype=torch.uint8, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(seed)
    chunk = 1 << 30
    for c0 in range(0, off, chunk):
        c1 = min(off, c0 + chunk)
        pool[c0:c1] = torch.randint(0, 256, (c1 - c0,), dtype=torch.uint8, device="cuda", generator=g)
    base = pool.data_ptr()
    items = [(codecs[(k, m)], base + o, st, S, op, present) for k, m, S, st, op, present, o in specs]
    nbytes = 0
    for k, m, S, st, op, present, _ in specs:
        nbytes += (k + m) * S if op == ENCODE else (k + int((present == 0).sum())) * S

    t0 = time.perf_counter()
    batch = Batch(items)
    create_s = time.perf_counter() - t0
    assert all(s == 0 for s in batch.statuses)
    t_batched = _time(batch.launch, reps, warmup=2)
    stats = batch.stats()
    # Plain: one launch per stripe on the matrix kernel (plus the decode-row build of
    # each reconstruct).
    for c in codecs.values():
        c.set_route("matrix")

    # The single-stripe entry points through shard pointer tables, the tables built
    # before timing (a caller holds its shard pointers already).
    import ctypes

    lib = _lib.load()
    calls = []
    for k, m, S, st, op, present, o in specs:
        n_sh = k + m
        ptrs = (ctypes.c_void_p * n_sh)(*[base + o + i * st for i in range(n_sh)])
        h = codecs[(k, m)]._h
        if op == ENCODE:
            calls.append((lib.rs8_encode_dev, (h, ptrs, n_sh, S, 0), ptrs))
        else:
            lens = (ctypes.c_size_t * n_sh)(*([S] * n_sh))
            flags = np.ascontiguousarray(present, np.uint8)
            calls.append((lib.rs8_reconstruct_dev,
                          (h, ptrs, lens, flags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n_sh, 0, 0),
                          (ptrs, lens, flags)))

    def plain():
        for fn, args, _ in calls:
            st = fn(*args)
            if st:
                raise RuntimeError("plain call status %d" % st)

    launches0 = _lib.load().rs_kernel_launch_count()
    # Host-bound (one library call per stripe): the better of two timed runs.
    t_plain = min(_time(plain, 1, warmup=1), _time(plain, 1, warmup=0))
    plain_launches = (_lib.load().rs_kernel_launch_count() - launches0) // 3
    # Batched, matrix route only (isolates the gain of batching from the FFT route).
    batch_m = Batch(items, flags=MATRIX_ONLY)
    t_batched_matrix = _time(batch_m.launch, reps, warmup=2)
    for c in codecs.values():
        c.set_route("auto")
    tuned = tuned_vs_exhaustive(items, t_batched, reps) if tuned_compare else {}
    queue = queue_session(items, nbytes) if tuned_compare else {}
    return {"stripes": n, "bytes": nbytes, "batched_gbs": nbytes / t_batched / 1e9,
            "batched_ms": t_batched * 1e3, "batched_launches": stats["launches"],
            "fft_items": stats["fft_items"], "matrix_items": stats["matrix_items"],
            "batched_matrix_only_gbs": nbytes / t_batched_matrix / 1e9,
            "plain_gbs": nbytes / t_plain / 1e9, "plain_ms": t_plain * 1e3, "plain_launches": plain_launches,
            "batched_over_plain": t_plain / t_batched, "create_s": create_s,
            "batched_incl_create_over_plain": t_plain / (t_batched + create_s),
            **tuned, **({"exhaustive_gbs": nbytes / tuned["exhaustive_ms"] * 1e3 / 1e9} if tuned else {}),
            **({"model_gbs": nbytes / tuned["model_ms"] * 1e3 / 1e9} if "model_ms" in tuned else {}), **queue}


def queue_session(items, nbytes):
    """The same stripes through the persistent work queue (one launch, all on the matrix
    route): pushed in chunks of 500 while the kernel runs; host time from start to the
    end of finish(), pushes (validation, host decode rows) included; best of two."""
    from .coder import Queue

    q = Queue(max_units=1 << 18, arena_bytes=256 << 20, timeout_s=10.0)
    best = None
    for _ in range(2):
        t0 = time.perf_counter()
        q.start()
        for c0 in range(0, len(items), 500):
            st = q.push(items[c0:c0 + 500])
            assert all(x == 0 for x in st)
        code = q.finish()
        t = time.perf_counter() - t0
        assert code == 0
        best = t if best is None else min(best, t)
    done, published = q.progress()
    return {"queue_gbs": nbytes / best / 1e9, "queue_s": best, "queue_units": published}


def tuned_vs_exhaustive(items, t_default, reps):
    """The batch's launch configurations three ways: the library's defaults (t_default,
    timed by the caller), the shipped cost model's choice (rs_batch_choose), and the
    exhaustive best: every launch group (encodes of one compiled shape and row
    alignment) timed alone under each applicable configuration, the fastest kept per
    group. Returns the replay times and the regrets against the exhaustive best."""
    from . import tuner

    model = tuner.shipped_model()
    out = {}
    groups = {}
    for i, (codec, rows, stride, S, op, present) in enumerate(items):
        sh = (codec.data_shard_count(), codec.parity_shard_count())
        if op != ENCODE or (sh not in tuner.GEN_SHAPES and not (sh[0] == sh[1] and sh[0] in tuner.FFT_K)):
            continue
        aligned = (_dev_ptr(rows) | stride) % 16 == 0
        groups.setdefault((sh, aligned), []).append(i)
    best_cfg = [-1] * len(items)
    tried = 0
    for (sh, aligned), idx in groups.items():
        sub = [items[i] for i in idx]
        gen = sh in tuner.GEN_SHAPES
        cands = [c for c, (route, _) in enumerate(tuner.CONFIGS)
                 if (route == "matrix" and c == 0) or (route == "gen" and gen) or (route == "fft" and not gen)]
        times = []
        for c in cands:
            b = Batch(sub, configs=[c] * len(sub))
            times.append(_time(b.launch, reps, warmup=1))
            tried += 1
        pick = cands[int(np.argmin(times))]
        for i in idx:
            best_cfg[i] = pick
    t_exh = _time(Batch(items, configs=best_cfg).launch, reps, warmup=2)
    out["exhaustive_ms"] = t_exh * 1e3
    out["exhaustive_groups"] = len(groups)
    out["exhaustive_timed_configs"] = tried
    out["regret_default"] = t_default / t_exh - 1.0
    if model is not None:
        bm = Batch(items, model=model)
        t_model = _time(bm.launch, reps, warmup=2)
        out["model_ms"] = t_model * 1e3
        out["regret_model"] = t_model / t_exh - 1.0
        def resolved(sh, aligned, cfg):  # -1: the automatic choice, as its table entry
            if cfg >= 0:
                return cfg
            if sh in tuner.GEN_SHAPES:
                return tuner.CONFIGS.index(("gen", 0))
            table = tuner.DEFAULT_FFT if aligned or sh[0] < 16 else tuner.UNALIGNED_FFT
            return tuner.CONFIGS.index(("fft", table[sh[0]]))

        out["model_groups_matching_exhaustive"] = sum(
            1 for (sh, al), idx in groups.items() if resolved(sh, al, bm.configs[idx[0]]) == best_cfg[idx[0]])
        out["groups"] = [{"shape": list(sh), "aligned": al, "stripes": len(idx),
                          "model": resolved(sh, al, bm.configs[idx[0]]), "model_kept_automatic": bm.configs[idx[0]] < 0,
                          "exhaustive": best_cfg[idx[0]]} for (sh, al), idx in groups.items()]
    return out


# ---- ReedSolomon16: (1024,1024) and (4096,12288), 2 KiB shards ----

def rs16_shapes(shapes=((1024, 1024, 64), (4096, 12288, 2)), S=2048, seed=4, reps=2):
    """Each shape is (k, m, stripes) at S-byte shards, or (k, m, stripes, shard_bytes)."""
    import torch

    out = []
    rng = np.random.default_rng(seed)
    for shape in shapes:
        k, m, stripes = shape[:3]
        S = shape[3] if len(shape) > 3 else S
        n = k + m
        rs = ReedSolomon16(k, m)
        g = torch.Generator(device="cuda").manual_seed(seed + k)
        rows = torch.randint(0, 256, (stripes, n, S), dtype=torch.uint8, device="cuda", generator=g)
        stride = n * S

        def enc():
            rs.encode_batch_dev(rows, rows[:, k:], S, stripes, data_stride=stride, parity_stride=stride)

        t_enc = _time(enc, reps)
        route = rs.encode_route(S, stripes)
        rs.set_route("matrix")
        t_mat = _time(enc, 1)
        t_fft = None
        if route != "fft" and k >= 2:  # the tower FFT, for comparison
            rs.set_route("fft")
            t_fft = _time(enc, 1)
        rs.set_route("auto")
        full = rows[0].clone()
        present = np.ones(n, np.uint8)
        present[rng.choice(n, size=m, replace=False)] = 0  # m erasures at random positions
        erased = torch.from_numpy(present == 0).cuda()
        rows[0][erased] = 0
        # The C ABI call with its pointer, length and flag arrays built once, as a caller
        # holding its shard pointers would (building them from tensor views in Python
        # takes longer than the decode at 16384 shards).
        import ctypes

        ptrs = (ctypes.c_void_p * n)(*[rows[0][i].data_ptr() for i in range(n)])
        lens = (ctypes.c_size_t * n)(*([S] * n))
        flags = np.ascontiguousarray(present, np.uint8)
        fptr = flags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        lib = _lib.load()

        def rec():
            st = lib.rs16_reconstruct_dev(rs._h, ptrs, lens, fptr, n, 0, 0)
            if st:
                raise RuntimeError("rs16_reconstruct_dev status %d" % st)

        # Cold: the first call of a pattern builds (and caches) its decode plan; warm:
        # the same pattern again, as a service decoding many stripes of one pattern does.
        t_cold = _time(rec, 1, warmup=0)
        exact_cold = bool(torch.equal(rows[0], full))
        rows[0][erased] = 0
        t_rec = _time(rec, 1, warmup=0)
        exact = bool(torch.equal(rows[0], full))
        out.append({"k": k, "m": m, "shard_bytes": S, "stripes": stripes, "route": route,
                    "encode_gbs": stripes * n * S / t_enc / 1e9, "encode_ms_per_stripe": t_enc / stripes * 1e3,
                    "encode_matrix_gbs": stripes * n * S / t_mat / 1e9,
                    "encode_tower_fft_gbs": stripes * n * S / t_fft / 1e9 if t_fft else None,
                    "reconstruct_m_erasures_gbs": (k + m) * S / t_rec / 1e9,
                    "reconstruct_ms": t_rec * 1e3, "reconstruct_cold_ms": t_cold * 1e3,
                    "reconstruct_bit_exact": exact and exact_cold})
        del rows
        torch.cuda.empty_cache()
    return out


# ---- autotuner and learned cost model ----

def tuner_regret(n_workloads=1500, seed=11, train_frac=0.8, max_bytes=64 << 20, epochs=300, save_model=None,
                 save_timings=None):
    """Exhaustive tuning of sampled GF(2^8) workloads (every applicable route / tile,
    timed on the GPU), the FP32 MLP cost model trained on most of them by the library's
    CUDA kernels, and its regret on the held-out rest against exhaustive tuning, beside
    the regret of the default choice (the method without the model)."""
    from . import tuner

    t0 = time.perf_counter()
    work = tuner.sample_workloads(n_workloads, seed=seed, max_bytes=max_bytes)
    X, T = tuner.collect(work, reps=2)
    collect_s = time.perf_counter() - t0
    n_tr = int(len(work) * train_frac)
    m = tuner.CostModel(hidden=64, seed=seed)
    t1 = time.perf_counter()
    hist = m.fit(X[:n_tr], T[:n_tr], epochs=epochs, lr=3e-3, batch=256)
    train_s = time.perf_counter() - t1
    if save_model:  # the model whose held-out regret is reported below
        m.save(save_model)
    if save_timings:
        np.savez_compressed(save_timings, X=X, T=T, train=n_tr, seed=seed,
                            configs=np.array([str(c) for c in tuner.CONFIGS]))
    te = slice(n_tr, len(work))
    choice = m.choose(X[te], T[te])
    default = tuner.default_choice(work[te], T[te])
    best = np.nanargmin(T[te], axis=1)
    return {"workloads": len(work), "timings": int(np.isfinite(T).sum()), "train": n_tr,
            "held_out": len(work) - n_tr, "collect_s": collect_s, "train_s": train_s,
            "final_loss": hist[-1], "regret_model": tuner.regret(T[te], choice),
            "regret_default": tuner.regret(T[te], default),
            "model_picks_best": float(np.mean(choice == best)),
            "default_picks_best": float(np.mean(default == best))}


# ---- serving: Poisson request stream through the request server ----

def poisson_requests(count, rate, seed):
    """Arrival offsets (ns) and request shapes: k log-uniform in 4..4096, m uniform in
    2..min(3k, 65536-k), GF(2^8) when k+m <= 256 else GF(2^16), shard bytes log-uniform
    in 512 B..1 MiB (even for GF(2^16)), encode:reconstruct 3:1, reconstructs erasing
    1..m shards at random positions."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        k = int(math.floor(math.exp(rng.uniform(math.log(4), math.log(4096)))))
        m = int(rng.integers(2, min(3 * k, 65536 - k) + 1))
        field = 8 if k + m <= 256 else 16
        S = int(math.exp(rng.uniform(math.log(512), math.log(1 << 20))))
        if field == 16:
            S += S % 2
        op = ENCODE if rng.random() < 0.75 else RECONSTRUCT
        present = _erasures(rng, k + m, m) if op == RECONSTRUCT else None
        out.append({"arrival_ns": int(t * 1e9), "field": field, "op": op, "k": k, "m": m, "row_len": S,
                    "present": present, "tag": i})
    return out


def serve_poisson(count=400, rate=50000.0, seed=5, arena_bytes=4 << 30, slots=64, streams=16, max_batch=64,
                  lookahead=64, route_hints=None, tuned=True):
    """Submits `count` requests at their Poisson arrival times (device-resident stripes
    carved from one synthetic pool; overlapping stripes share bytes, which changes no
    timing because the arithmetic is data-independent) and reports latency from arrival
    to completion, and throughput over the whole run. With `tuned` the server's FFT
    launch shapes come from the shipped cost model."""
    import torch

    from . import tuner
    from .server import Server

    reqs = poisson_requests(count, rate, seed)
    biggest = max((r["k"] + r["m"]) * r["row_len"] for r in reqs)
    pool = torch.empty(biggest + 256, dtype=torch.uint8, device="cuda")
    pool.random_(0, 256, generator=torch.Generator(device="cuda").manual_seed(seed))
    rng = np.random.default_rng(seed + 1)
    base = pool.data_ptr()
    for r in reqs:
        span = (r["k"] + r["m"]) * r["row_len"]
        r["rows"] = base + (int(rng.integers(0, biggest - span + 1)) & ~255)
    model = tuner.shipped_model() if tuned else None
    srv = Server(arena_bytes=arena_bytes, slots=slots, streams=streams, max_batch=max_batch, lookahead=lookahead,
                 model=model)
    for k, log2b, route in (route_hints or []):
        srv.set_fft_route(k, log2b, route)
    torch.cuda.synchronize()
    t0 = time.monotonic_ns() + 2_000_000
    for r in reqs:
        r["arrival_ns"] += t0
    done = []
    i = 0
    while i < len(reqs):
        now = time.monotonic_ns()
        j = i
        while j < len(reqs) and reqs[j]["arrival_ns"] <= now:
            j += 1
        if j > i:
            st = srv.submit(reqs[i:j])
            if any(st):
                raise RuntimeError("server rejected requests: %s" % [s for s in st if s])
            i = j
        done.extend(srv.poll(timeout_ms=0))
    while len(done) < len(reqs):
        got = srv.poll(timeout_ms=600000)
        if not got:
            raise TimeoutError("server stalled")
        done.extend(got)
    stats = srv.stats()
    srv.close()
    arrival = {r["tag"]: r["arrival_ns"] for r in reqs}
    lat = np.array([(c["done_ns"] - arrival[c["tag"]]) / 1e6 for c in done])
    wait = np.array([(c["admit_ns"] - arrival[c["tag"]]) / 1e6 for c in done])
    service = np.array([(c["done_ns"] - c["admit_ns"]) / 1e6 for c in done])
    span_s = (max(c["done_ns"] for c in done) - min(arrival.values())) / 1e9
    nbytes = sum(c["bytes"] for c in done)
    by_field = {f: sum(1 for r in reqs if r["field"] == f) for f in (8, 16)}
    return {"requests": count, "offered_rate": rate, "gf8_requests": by_field[8], "gf16_requests": by_field[16],
            "statuses_ok": all(c["status"] == 0 for c in done),
            "latency_ms_p50": float(np.percentile(lat, 50)), "latency_ms_p99": float(np.percentile(lat, 99)),
            "queue_ms_p50": float(np.percentile(wait, 50)), "queue_ms_p99": float(np.percentile(wait, 99)),
            "service_ms_p50": float(np.percentile(service, 50)), "service_ms_p99": float(np.percentile(service, 99)),
            "gbs": nbytes / span_s / 1e9, "bytes": nbytes, "makespan_s": span_s,
            "completed_rate": count / span_s, "arena_bytes": arena_bytes, "arena_peak": stats["arena_peak"],
            "groups": stats["groups"], "merged": stats["merged"], "launches": stats["launches"],
            "table_builds": stats["table_builds"], "table_hits": stats["table_hits"],
            "evictions": stats["evictions"]}
