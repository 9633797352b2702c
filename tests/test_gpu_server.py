"""Request server (rs_server_*): continuous batching, admission by device memory.

Every result is checked against the oracle (encode) or the pre-erasure stripe
(reconstruct, which is unique), and a set of probe requests must give the same bytes
when each runs alone and when it runs in a mix with other requests on the GPU.
Validation errors are the ones the single-stripe calls of the reference return.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ENC, REC, REC_DATA = 0, 1, 2


def _stripe(O, field, k, m, row_len, seed):
    rng = np.random.default_rng(seed)
    data = rng.integers(0, 256, size=(k, row_len), dtype=np.uint8)
    parity = O.encode8(k, m, data) if field == 8 else O.encode16(k, m, data)
    return np.concatenate([data, parity])


def _make(O, spec, seed):
    """spec: (field, op, k, m, row_len, on_host). Returns (request dict, expected rows)."""
    import torch

    field, op, k, m, row_len, on_host = spec
    full = _stripe(O, field, k, m, row_len, seed)
    work = full.copy()
    present = None
    if op == ENC:
        work[k:] = 0x5A
        expect = full
    else:
        rng = np.random.default_rng(seed + 1)
        n = k + m
        present = np.ones(n, np.uint8)
        present[rng.choice(n, size=int(rng.integers(1, m + 1)), replace=False)] = 0
        work[present == 0] = 0
        expect = full.copy()
        if op == REC_DATA:
            expect[k:][present[k:] == 0] = 0  # absent parity stays as it was
    rows = work if on_host else torch.from_numpy(work).cuda()
    req = {"field": field, "op": op, "k": k, "m": m, "row_len": row_len, "rows": rows, "present": present}
    return req, expect


def _result(req):
    rows = req["rows"]
    return rows.copy() if isinstance(rows, np.ndarray) else rows.cpu().numpy()


PROBES = [
    (8, ENC, 32, 32, 4096, False),    # FFT K=32
    (8, ENC, 16, 16, 333, True),      # FFT K=16, ragged length, host staged
    (8, ENC, 128, 128, 2048, False),  # FFT K=128
    (8, ENC, 10, 10, 1000, True),     # generator kernel
    (8, ENC, 20, 12, 4096, False),    # generator kernel, device rows
    (8, ENC, 20, 10, 1000, True),     # matrix (no compiled shape)
    (8, REC, 20, 12, 777, False),
    (8, REC_DATA, 7, 13, 2048, True),
    (8, REC, 64, 64, 4100, False),
    (16, ENC, 100, 50, 2048, False),
    (16, REC, 300, 200, 1024, True),
    (16, REC_DATA, 40, 30, 66, False),
]


def _background(O, count, seed):
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(count):
        field = 8 if rng.random() < 0.6 else 16
        k = int(rng.integers(1, 48)) if field == 8 else int(rng.integers(1, 150))
        m = int(rng.integers(1, 48)) if field == 8 else int(rng.integers(1, 150))
        if field == 8 and rng.random() < 0.3:
            k = m = int(rng.choice([2, 4, 8, 16, 32]))
        row_len = int(rng.integers(1, 3000))
        if field == 16:
            row_len += row_len % 2
        op = int(rng.choice([ENC, ENC, ENC, REC, REC_DATA]))
        specs.append((field, op, k, m, row_len, bool(rng.random() < 0.3)))
    return specs


@pytest.mark.parametrize("tuned", [False, True])
def test_alone_equals_in_mix(gpu, O, tuned):
    """With tuned=True the server's cost model (the shipped one) picks the FFT launch
    groups' launch shapes; results must not change."""
    from reed_solomon_b200 import tuner

    model = tuner.shipped_model() if tuned else None
    assert model is not None or not tuned
    srv = gpu.Server(arena_bytes=256 << 20, slots=32, streams=4, max_batch=16, lookahead=8, model=model)
    alone = []
    for i, spec in enumerate(PROBES):
        req, expect = _make(O, spec, seed=10 + i)
        req["tag"] = i
        assert srv.submit([req]) == [0]
        (c,) = srv.wait(1)
        assert c["status"] == 0 and c["tag"] == i
        got = _result(req)
        assert np.array_equal(got, expect), spec
        alone.append(got)

    # The same probes again, interleaved with background requests.
    bg = _background(O, 120, seed=7)
    batch, checks = [], {}
    tag = 1000
    for i, spec in enumerate(PROBES):
        for spec_bg in bg[i * 12:(i + 1) * 12]:
            req, expect = _make(O, spec_bg, seed=tag)
            req["tag"] = tag
            batch.append(req)
            checks[tag] = (req, expect)
            tag += 1
        req, expect = _make(O, spec, seed=10 + i)
        req["tag"] = i
        batch.append(req)
        checks[i] = (req, expect)
    # Submit in a few waves so that requests arrive while others run.
    for w in range(0, len(batch), 17):
        assert srv.submit(batch[w:w + 17]) == [0] * len(batch[w:w + 17])
    done = srv.wait(len(batch))
    assert sorted(c["tag"] for c in done) == sorted(checks)
    assert all(c["status"] == 0 for c in done)
    for t, (req, expect) in checks.items():
        got = _result(req)
        assert np.array_equal(got, expect), t
        if t < len(PROBES):
            assert np.array_equal(got, alone[t]), PROBES[t]
    st = srv.stats()
    assert st["completed"] == len(PROBES) + len(batch)
    assert st["merged"] > 0  # some GF(2^8) requests shared a launch group
    assert st["arena_used"] <= st["arena_bytes"]
    srv.close()


def test_admission_by_arena_space(gpu, O):
    # 1 MiB arena: a host-staged (16,16) x 16 KiB stripe needs 512 KiB of payload plus
    # its descriptors, so one is admitted at a time; the rest wait and still complete.
    srv = gpu.Server(arena_bytes=1 << 20, slots=16, streams=2)
    reqs, exp = [], []
    for i in range(24):
        req, expect = _make(O, (8, ENC if i % 3 else REC, 16, 16, 16384, True), seed=500 + i)
        req["tag"] = i
        reqs.append(req)
        exp.append(expect)
    big, _ = _make(O, (8, ENC, 32, 32, 65536, True), seed=1)  # 4 MiB: can never fit
    big["tag"] = 99
    st = srv.submit(reqs + [big])
    assert st[:-1] == [0] * len(reqs)
    assert gpu.ERROR_NAMES[st[-1]] == "TooLarge"
    done = srv.wait(len(reqs))
    assert all(c["status"] == 0 for c in done)
    for req, expect in zip(reqs, exp):
        assert np.array_equal(_result(req), expect)
    s = srv.stats()
    assert s["arena_peak"] <= 1 << 20
    assert s["rejected"] == 1
    # Admission waited for memory: later requests were admitted after earlier ones finished.
    by_tag = {c["tag"]: c for c in done}
    assert max(c["admit_ns"] for c in done) >= min(c["done_ns"] for c in done)
    assert by_tag[len(reqs) - 1]["admit_ns"] > by_tag[0]["admit_ns"]
    srv.close()


def test_resident_tables_hit_and_evict(gpu, O):
    srv = gpu.Server(arena_bytes=2 << 20, slots=8)
    # Same shape repeatedly: one table build, then hits.
    for i in range(6):
        req, expect = _make(O, (16, ENC, 200, 100, 512, False), seed=900 + i)
        req["tag"] = i
        srv.submit([req])
        srv.wait(1)
        assert np.array_equal(_result(req), expect)
    s = srv.stats()
    assert s["table_builds"] == 1 and s["table_hits"] == 5
    srv.close()
    # Matrix-route shapes (few data rows, short shards) whose generators (m*k*4 bytes,
    # 32 KB each) cannot all stay resident in a 256 KiB arena force evictions.
    srv = gpu.Server(arena_bytes=256 << 10, slots=8)
    for i in range(12):
        req, expect = _make(O, (16, ENC, 20, 400 + i, 64, False), seed=950 + i)
        req["tag"] = 100 + i
        srv.submit([req])
        srv.wait(1)
        assert np.array_equal(_result(req), expect)
    assert srv.stats()["evictions"] > 0
    srv.close()


def test_validation_matches_reference_errors(gpu):
    import torch

    srv = gpu.Server(arena_bytes=8 << 20)
    buf = torch.zeros(64 * 4, dtype=torch.uint8, device="cuda")
    cases = [
        ({"field": 8, "k": 0, "m": 4, "row_len": 4}, "TooFewDataShards"),
        ({"field": 8, "k": 4, "m": 0, "row_len": 4}, "TooFewParityShards"),
        ({"field": 8, "k": 200, "m": 57, "row_len": 4}, "TooManyShards"),
        ({"field": 16, "k": 60000, "m": 5537, "row_len": 4}, "TooManyShards"),
        ({"field": 8, "k": 4, "m": 4, "row_len": 0}, "EmptyShard"),
        ({"field": 16, "k": 4, "m": 4, "row_len": 3}, "IncorrectShardSize"),
        ({"field": 8, "k": 4, "m": 4, "row_len": 4, "op": REC, "present": [1, 1, 1, 0, 0, 0, 0, 0]},
         "TooFewShardsPresent"),
    ]
    for i, (r, name) in enumerate(cases):
        r = dict(r, rows=buf, tag=i)
        r.setdefault("op", ENC)
        (st,) = srv.submit([r])
        assert gpu.ERROR_NAMES[st] == name, (r, st)
    # Nothing to rebuild: completes at once with no work.
    (st,) = srv.submit([{"field": 8, "k": 4, "m": 4, "row_len": 4, "op": REC, "present": [1] * 8, "rows": buf,
                         "tag": 77}])
    assert st == 0
    (c,) = srv.wait(1)
    assert c["tag"] == 77 and c["status"] == 0 and c["group_size"] == 0
    srv.close()
