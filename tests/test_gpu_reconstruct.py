"""GF(2^8) reconstruct on the B200 through the C ABI.

Mirrors src/reedsolomon.rs:1023-1158 (round trip, pattern walk through the plan cache,
prepared decoder, data-only, contiguous rows) and the wire-compat gate's shapes, sizes
and erasure counts (tests/parity.rs:16-27,161). Decoding is unique, so every rebuilt
stripe must equal the pre-erasure stripe; the oracle supplies the encodes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def encoded(O, k, m, length, seed):
    data = np.random.default_rng(seed).integers(0, 256, size=(k, length), dtype=np.uint8)
    return np.concatenate([data, O.encode8(k, m, data)])


def erase_view(full, erased):
    shards = [s.copy() for s in full]
    view = []
    for i, s in enumerate(shards):
        if i in erased:
            s[:] = 0
        view.append((s, i not in erased))
    return shards, view


@pytest.mark.parametrize("length", [(1 << 20) + 333, (4 << 20) + 333])
def test_large_host_reconstruct(gpu, O, length):
    """Host-pointer reconstruct of one RS(32,32) stripe with m erasures: at 1 MiB + 333
    bytes the survivors are gathered into pinned memory by host threads (1 MiB pieces,
    a ragged last piece); past 256 MiB crossing the link (4 MiB + 333) each shard is
    copied on its own. The stripe is encoded on the host path and checked against the
    oracle at sampled columns; the rebuilt stripe must equal it."""
    k = m = 32
    rng = np.random.default_rng(length)
    full = [rng.integers(0, 256, size=length, dtype=np.uint8) for _ in range(k)]
    full += [np.zeros(length, np.uint8) for _ in range(m)]
    rs = gpu.ReedSolomon(k, m)
    rs.encode(full)
    cols = np.unique(np.concatenate([rng.choice(length, size=2048, replace=False), np.arange(length - 40, length)]))
    data = np.ascontiguousarray(np.stack(full[:k])[:, cols])
    assert np.array_equal(np.stack(full[k:])[:, cols], O.encode8(k, m, data))
    erased = set(rng.choice(k + m, size=m, replace=False).tolist())
    got, view = erase_view(full, erased)
    rs.reconstruct(view)
    for i in range(k + m):
        assert np.array_equal(got[i], full[i]), i


def test_round_trip_reconstruct(gpu):
    rs = gpu.ReedSolomon(4, 4)
    shards = [np.full(100, j + 1, np.uint8) for j in range(4)] + [np.zeros(100, np.uint8) for _ in range(4)]
    rs.encode(shards)
    original = [s.copy() for s in shards]
    got, view = erase_view(original, {0, 2, 5})
    rs.reconstruct(view)
    for i in range(8):
        assert np.array_equal(got[i], original[i])


@pytest.mark.parametrize("k,m", [(4, 2), (7, 13), (10, 10), (6, 4), (32, 32), (16, 16), (128, 127)])
def test_reconstruct_patterns(gpu, O, k, m):
    rs = gpu.ReedSolomon(k, m)
    for length in [15, 100, 1024]:
        full = encoded(O, k, m, length, k + m + length)
        patterns = [[0], [k - 1], [k], list(range(min(m, k))), list(range(k, k + m)),
                    sorted({(e * 2) % (k + m) for e in range(m)})]
        for erased in patterns:
            for _ in range(2):  # second call hits the cached plan
                got, view = erase_view(full, set(erased))
                rs.reconstruct(view)
                assert np.array_equal(np.array(got), full), (k, m, length, erased)


def test_prepared_decoder(gpu, O):
    k, m, length = 7, 13, 200
    rs = gpu.ReedSolomon(k, m)
    full = encoded(O, k, m, length, 1)
    erased = {1, 3, 8, 15}
    present = [i not in erased for i in range(k + m)]
    dec = rs.prepare_decode(present)
    for _ in range(3):
        got, view = erase_view(full, erased)
        dec.reconstruct(view)
        assert np.array_equal(np.array(got), full)
    got, view = erase_view(full, {0})
    with pytest.raises(gpu.RsError) as e:
        dec.reconstruct(view)
    assert e.value.name == "InvalidShardFlags"
    dec2 = dec.clone()
    got, view = erase_view(full, erased)
    dec2.reconstruct(view)
    assert np.array_equal(np.array(got), full)


def test_prepared_data_only(gpu, O):
    k, m, length = 6, 4, 128
    rs = gpu.ReedSolomon(k, m)
    full = encoded(O, k, m, length, 2)
    erased = {2, k + 1}
    dec = rs.prepare_decode([i not in erased for i in range(k + m)])
    got, view = erase_view(full, erased)
    dec.reconstruct_data(view)
    assert np.array_equal(got[2], full[2])
    assert not got[k + 1].any(), "missing parity must stay untouched"
    got, view = erase_view(full, erased)
    rs.reconstruct_data(view)
    assert np.array_equal(got[2], full[2]) and not got[k + 1].any()


def test_reconstruct_rows_roundtrip(gpu, O):
    k, m, row_len = 10, 10, 257
    rs = gpu.ReedSolomon(k, m)
    full = encoded(O, k, m, row_len, 3)
    rows = full.reshape(-1).copy()
    present = [True] * (k + m)
    for e in [0, 4, 12, 19]:
        present[e] = False
        rows[e * row_len:(e + 1) * row_len] = 0
    rs.reconstruct_rows(rows, row_len, present)
    assert np.array_equal(rows, full.reshape(-1))
    with pytest.raises(gpu.RsError) as e:
        rs.reconstruct_rows(rows, row_len, present[:-1])
    assert e.value.name == "InvalidShardFlags"
    with pytest.raises(gpu.RsError) as e:
        rs.reconstruct_rows(rows, 0, present)
    assert e.value.name == "EmptyShard"
    with pytest.raises(gpu.RsError) as e:
        rs.reconstruct_rows(rows[:-1], row_len, present)
    assert e.value.name == "IncorrectShardSize"


def test_option_shards(gpu, O):
    """None shards are allocated by the call (src/reedsolomon.rs:88-101)."""
    k, m, length = 5, 3, 77
    rs = gpu.ReedSolomon(k, m)
    full = encoded(O, k, m, length, 4)
    opt = [full[i].copy() for i in range(k + m)]
    opt[1] = None
    opt[6] = None
    rs.reconstruct(opt)
    assert all(np.array_equal(opt[i], full[i]) for i in range(k + m))
    opt = [full[i].copy() for i in range(k + m)]
    opt[0] = None
    opt[7] = None
    rs.reconstruct_data(opt)
    assert np.array_equal(opt[0], full[0]) and opt[7] is None


def test_reconstruct_errors(gpu, O):
    k, m, length = 4, 2, 16
    rs = gpu.ReedSolomon(k, m)
    full = encoded(O, k, m, length, 5)
    _, view = erase_view(full, {0, 1, 2})
    with pytest.raises(gpu.RsError) as e:
        rs.reconstruct(view)
    assert e.value.name == "TooFewShardsPresent"
    _, view = erase_view(full, {0})
    with pytest.raises(gpu.RsError) as e:
        rs.reconstruct(view[:-1])
    assert e.value.name == "TooFewShards"
    _, view = erase_view(full, {0})
    view[3] = (np.zeros(length + 1, np.uint8), True)
    with pytest.raises(gpu.RsError) as e:
        rs.reconstruct(view)
    assert e.value.name == "IncorrectShardSize"
    _, view = erase_view(full, {0})
    view[0] = (np.zeros(length - 1, np.uint8), False)  # absent buffer of the wrong size
    with pytest.raises(gpu.RsError) as e:
        rs.reconstruct(view)
    assert e.value.name == "IncorrectShardSize"
    _, view = erase_view(full, {0})
    view[2] = (np.zeros(0, np.uint8), True)
    with pytest.raises(gpu.RsError) as e:
        rs.reconstruct(view)
    assert e.value.name == "EmptyShard"
    # All present: a no-op.
    _, view = erase_view(full, set())
    rs.reconstruct(view)


PARAMS = [(2, 2), (4, 4), (6, 4), (7, 13), (10, 7), (10, 10), (17, 17), (20, 10), (32, 32)]
SIZES = [32, 1024, 32768]


def pick_erasures(total, e, rng):
    idx = list(range(total))
    for i in range(e):  # Fisher-Yates partial shuffle, tests/parity.rs:43-53
        j = i + int(rng.integers(0, 1 << 32)) % (total - i)
        idx[i], idx[j] = idx[j], idx[i]
    return sorted(idx[:e])


@pytest.mark.parametrize("k,m", PARAMS)
def test_wire_compat_gate_shapes(gpu, O, k, m):
    """(a) encode parity == oracle; (c) round trip; (d) prepared + rows."""
    rng = np.random.default_rng(0xC1A7 + k * 100 + m)
    rs = gpu.ReedSolomon(k, m)
    for sz in SIZES:
        data = rng.integers(0, 256, size=(k, sz), dtype=np.uint8)
        want = O.encode8(k, m, data)
        shards = [data[i].copy() for i in range(k)] + [np.zeros(sz, np.uint8) for _ in range(m)]
        rs.encode(shards)
        assert np.array_equal(np.array(shards[k:]), want)
        full = np.concatenate([data, want])
        for e in [0, 1, m // 2, m]:
            erased = pick_erasures(k + m, e, rng)
            got, view = erase_view(full, set(erased))
            rs.reconstruct(view)
            assert np.array_equal(np.array(got), full)
            present = [i not in erased for i in range(k + m)]
            dec = rs.prepare_decode(present)
            got, view = erase_view(full, set(erased))
            dec.reconstruct(view)
            assert np.array_equal(np.array(got), full)
            rows = full.reshape(-1).copy()
            for i in erased:
                rows[i * sz:(i + 1) * sz] = 0
            rs.reconstruct_rows(rows, sz, present)
            assert np.array_equal(rows, full.reshape(-1))


def test_reconstruct_dev_pointers(gpu, O):
    import torch

    k, m, length = 10, 10, 3000
    rs = gpu.ReedSolomon(k, m)
    full = encoded(O, k, m, length, 6)
    erased = {0, 3, 11, 19, 7}
    bufs = [torch.from_numpy(full[i].copy() if i not in erased else np.zeros(length, np.uint8)).cuda()
            for i in range(k + m)]
    rs.reconstruct_dev(bufs, [i not in erased for i in range(k + m)], length)
    torch.cuda.synchronize()
    got = np.array([b.cpu().numpy() for b in bufs])
    assert np.array_equal(got, full)


@pytest.mark.parametrize("k,m,row_len,stripes", [(32, 32, 4096, 40), (16, 16, 333, 17), (10, 10, 64, 50),
                                                 (64, 64, 2048, 12), (20, 12, 1000, 20), (128, 128, 512, 6),
                                                 (20, 10, 777, 9)])
def test_reconstruct_batch_device(gpu, O, k, m, row_len, stripes):
    """Many stripes, each with its own pattern of 1..m erasures, in one launch."""
    import torch

    rng = np.random.default_rng(k * stripes)
    full = np.stack([encoded(O, k, m, row_len, int(rng.integers(1 << 30))) for _ in range(stripes)])
    present = np.ones((stripes, k + m), np.uint8)
    for s in range(stripes):
        e = int(rng.integers(1, m + 1))
        present[s, rng.choice(k + m, size=e, replace=False)] = 0
    present[0, :] = 1  # one untouched stripe
    work = full.copy()
    work[present == 0] = 0
    for route in ("auto", "fft", "matrix"):  # "fft": missing parity on the compiled kernel
        rs = gpu.ReedSolomon(k, m)
        rs.set_route(route)
        d = torch.from_numpy(work).cuda()
        st = rs.reconstruct_batch_dev(d, stripes, row_len, present)
        torch.cuda.synchronize()
        assert st == [0] * stripes, (route, st)
        assert np.array_equal(d.cpu().numpy(), full), route
    # data-only: missing parity rows stay as they were (zero).
    d = torch.from_numpy(work).cuda()
    gpu.ReedSolomon(k, m).reconstruct_batch_dev(d, stripes, row_len, present, data_only=True)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    assert np.array_equal(got[:, :k], full[:, :k])
    assert not got[:, k:][present[:, k:] == 0].any()


@pytest.mark.parametrize("k,m", [(32, 32), (10, 10), (128, 128)])
def test_reconstruct_batch_device_stores_only_missing_parity(gpu, O, k, m):
    """Shapes with a compiled encode kernel regenerate missing parity with it, storing
    only the missing rows: present parity rows, here deliberately inconsistent with the
    data, are left exactly as they were, on every route."""
    import torch

    rng = np.random.default_rng(k + 7)
    stripes, row_len = 6, 1000
    full = np.stack([encoded(O, k, m, row_len, int(rng.integers(1 << 30))) for _ in range(stripes)])
    present = np.ones((stripes, k + m), np.uint8)
    work = full.copy()
    for s in range(stripes):
        lost = rng.choice(m, size=int(rng.integers(1, m + 1)), replace=False) + k
        present[s, lost] = 0
        work[s, lost] = 0
        kept = [i for i in range(k, k + m) if present[s, i]]
        work[s, kept] ^= 0x5A
    want = work.copy()
    want[present == 0] = full[present == 0]
    for route in ("fft", "auto", "matrix"):
        rs = gpu.ReedSolomon(k, m)
        rs.set_route(route)
        d = torch.from_numpy(work).cuda()
        st = rs.reconstruct_batch_dev(d, stripes, row_len, present)
        torch.cuda.synchronize()
        assert st == [0] * stripes
        assert np.array_equal(d.cpu().numpy(), want), route


@pytest.mark.parametrize("k,m,length", [(32, 32, 70000), (10, 4, 5000), (16, 16, 65536)])
def test_reconstruct_dev_stores_only_missing_parity(gpu, O, k, m, length):
    """Single-stripe device reconstruct on a shape with a compiled encode kernel: large
    shards (and the forced compiled route) rebuild missing data on the matrix route and
    regenerate missing parity with the compiled kernel, which leaves present parity rows
    untouched (the ones the decoder does not read are made inconsistent here, so a stray
    write would show); every route gives the same bytes."""
    import torch

    rng = np.random.default_rng(k * 3 + length)
    full = encoded(O, k, m, length, 99)
    n = k + m
    lost = sorted(rng.choice(n, size=m, replace=False).tolist())
    work = full.copy()
    work[lost] = 0
    survivors = [i for i in range(n) if i not in lost][:k]  # the first k present are read
    unread = [i for i in range(k, n) if i not in lost and i not in survivors]
    work[unread] ^= 0x3C
    want = work.copy()
    want[lost] = full[lost]
    for route in ("auto", "fft", "matrix"):
        rs = gpu.ReedSolomon(k, m)
        rs.set_route(route)
        bufs = [torch.from_numpy(work[i].copy()).cuda() for i in range(n)]
        rs.reconstruct_dev(bufs, [i not in lost for i in range(n)], length)
        torch.cuda.synchronize()
        got = np.array([b.cpu().numpy() for b in bufs])
        assert np.array_equal(got, want), route
