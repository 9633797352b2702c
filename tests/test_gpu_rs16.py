"""ReedSolomon16 (GF((2^8)^2) tower, split-plane wire) on the B200.

Mirrors src/reedsolomon16.rs:893-1256: encode == symbol-wise scalar oracle over shapes
and even lengths, the frozen wire vector, reconstruct patterns including past the
256-shard wall, prepared and data-only decoders, verify blocks, odd lengths rejected.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rand(k, length, seed):
    return np.random.default_rng(seed).integers(0, 256, size=(k, length), dtype=np.uint8)


def encode_gpu(rs, data, m):
    k, length = data.shape
    shards = [data[i].copy() for i in range(k)] + [np.full(length, 0xA5, np.uint8) for _ in range(m)]
    rs.encode(shards)
    return np.array(shards[k:])


def test_golden_wire_vector(gpu, golden):
    g = golden["gf16_wire_vector"]
    rs = gpu.ReedSolomon16(g["k"], g["m"])
    assert encode_gpu(rs, np.array(g["data"], np.uint8), g["m"]).tolist() == g["parity"]


@pytest.mark.parametrize("route", ["auto", "matrix"])
@pytest.mark.parametrize("k,m", [(4, 2), (7, 13), (10, 10), (17, 33), (1, 1), (300, 20)])
def test_encode_matches_symbolwise(gpu, O, k, m, route):
    """The automatic route (the GF(2^8) codec for k + m <= 256) and the tower matrix
    kernel both give the symbol-wise oracle's bytes."""
    rs = gpu.ReedSolomon16(k, m)
    rs.set_route(route)
    assert np.array_equal(rs.parity_matrix(), O.build_matrix(16, k, k + m)[k:])
    for length in [2, 30, 32, 34, 62, 64, 66, 200, 2048, 4098]:
        if k * m * length > 40_000_000:
            continue
        data = rand(k, length, k + length)
        assert np.array_equal(encode_gpu(rs, data, m), O.encode16(k, m, data)), (k, m, length)


def test_encode_sep_and_verify(gpu, O):
    for k, m in [(4, 2), (17, 33)]:
        rs = gpu.ReedSolomon16(k, m)
        for length in [34, 512]:
            data = rand(k, length, length)
            combined = encode_gpu(rs, data, m)
            parity = [np.zeros(length, np.uint8) for _ in range(m)]
            rs.encode_sep([data[i] for i in range(k)], parity)
            assert np.array_equal(np.array(parity), combined)
    k, m = 4, 3
    rs = gpu.ReedSolomon16(k, m)
    for length in [200, 2 * 16384, 2 * 16384 + 34]:
        data = rand(k, length, 9)
        shards = [data[i] for i in range(k)] + list(encode_gpu(rs, data, m))
        assert rs.verify(shards)
        for pos in [0, length // 2, length - 1]:
            bad = [s.copy() for s in shards]
            bad[k][pos] ^= 1
            assert not rs.verify(bad)


def test_odd_length_rejected(gpu):
    rs = gpu.ReedSolomon16(2, 2)
    with pytest.raises(gpu.RsError) as e:
        rs.encode([np.zeros(5, np.uint8) for _ in range(4)])
    assert e.value.name == "IncorrectShardSize"
    with pytest.raises(gpu.RsError) as e:
        rs.encode([np.zeros(0, np.uint8) for _ in range(4)])
    assert e.value.name == "EmptyShard"


@pytest.mark.parametrize("route", ["auto", "matrix"])
@pytest.mark.parametrize("k,m", [(4, 2), (17, 33), (10, 10), (100, 200)])
def test_reconstruct_patterns(gpu, O, k, m, route):
    rs = gpu.ReedSolomon16(k, m)
    rs.set_route(route)
    total = k + m
    for length in [2, 34, 512]:
        data = rand(k, length, length + k)
        full = np.concatenate([data, O.encode16(k, m, data)])
        patterns = [[0], [k - 1], [k], list(range(min(m, k))), list(range(k, k + m)),
                    sorted({(e * 3) % total for e in range(m)})]
        for erased in patterns:
            for _ in range(2):
                shards = [s.copy() for s in full]
                for e in erased:
                    shards[e][:] = 0
                view = [(s, i not in erased) for i, s in enumerate(shards)]
                rs.reconstruct(view)
                assert np.array_equal(np.array(shards), full), (k, m, length, erased)


@pytest.mark.parametrize("route", ["auto", "matrix"])
def test_prepared_and_data_only(gpu, O, route):
    """Prepared decoders; with k + m <= 256 the automatic route rebuilds on the GF(2^8)
    codec's prepared decoder after the tower's checks, the matrix route on the tower's."""
    k, m, length = 17, 33, 200
    rs = gpu.ReedSolomon16(k, m)
    rs.set_route(route)
    data = rand(k, length, 1)
    full = np.concatenate([data, O.encode16(k, m, data)])
    erased = {1, 3, 20, 40}
    dec = rs.prepare_decode([i not in erased for i in range(k + m)])
    for _ in range(3):
        shards = [s.copy() if i not in erased else np.zeros(length, np.uint8) for i, s in enumerate(full)]
        dec.reconstruct([(s, i not in erased) for i, s in enumerate(shards)])
        assert np.array_equal(np.array(shards), full)
    shards = [s.copy() for s in full]
    shards[0][:] = 0
    with pytest.raises(gpu.RsError) as e:
        dec.reconstruct([(s, i != 0) for i, s in enumerate(shards)])
    assert e.value.name == "InvalidShardFlags"
    k, m = 6, 4
    rs = gpu.ReedSolomon16(k, m)
    rs.set_route(route)
    data = rand(k, 128, 2)
    full = np.concatenate([data, O.encode16(k, m, data)])
    erased = {2, k + 1}
    dec = rs.prepare_decode([i not in erased for i in range(k + m)])
    shards = [s.copy() if i not in erased else np.zeros(128, np.uint8) for i, s in enumerate(full)]
    dec.reconstruct_data([(s, i not in erased) for i, s in enumerate(shards)])
    assert np.array_equal(shards[2], full[2]) and not shards[k + 1].any()


def test_reconstruct_rows_and_options(gpu, O):
    k, m, row_len = 11, 20, 258
    rs = gpu.ReedSolomon16(k, m)
    data = rand(k, row_len, 3)
    full = np.concatenate([data, O.encode16(k, m, data)])
    rows = full.reshape(-1).copy()
    present = [True] * (k + m)
    for e in [0, 5, 12, 30]:
        present[e] = False
        rows[e * row_len:(e + 1) * row_len] = 0
    rs.reconstruct_rows(rows, row_len, present)
    assert np.array_equal(rows, full.reshape(-1))
    with pytest.raises(gpu.RsError) as e:
        rs.reconstruct_rows(rows[: (k + m) * 3], 3, present)
    assert e.value.name == "IncorrectShardSize"
    opt = [full[i].copy() for i in range(k + m)]
    for i in range(min(k, m)):
        opt[i] = None
    rs.reconstruct_data(opt)
    assert all(np.array_equal(opt[i], full[i]) for i in range(k))


def test_large_shape_round_trip(gpu, O):
    """(4096, 12288) at 2 KiB shards: encode, erase m shards, rebuild, compare. Too
    large for the Gauss-Jordan oracle; decoding is unique, so the rebuilt stripe must
    equal the original, and at 16 sampled symbol columns every shard (the rebuilt
    ones included) must equal the oracle's Lagrange evaluation of the data."""
    import torch

    k, m, length = 4096, 12288, 2048
    rs = gpu.ReedSolomon16(k, m)
    rng = np.random.default_rng(44)
    data = torch.from_numpy(rng.integers(0, 256, size=(k, length), dtype=np.uint8)).cuda()
    parity = torch.zeros((m, length), dtype=torch.uint8, device="cuda")
    rs.encode_batch_dev(data, parity, length, 1)
    full = torch.cat([data, parity]).contiguous()
    torch.cuda.synchronize()
    ref = full.clone()
    erased = rng.choice(k + m, size=m, replace=False)
    present = np.ones(k + m, bool)
    present[erased] = False
    full[torch.from_numpy(erased).cuda()] = 0
    rs.reconstruct_dev([full[i] for i in range(k + m)], present.tolist(), length)
    torch.cuda.synchronize()
    rng_c = np.random.default_rng(45)
    cols = sorted({0, 31, 32, length // 2 - 1} | set(int(c) for c in rng_c.choice(length // 2, 12, replace=False)))
    want = O.eval_columns(16, k, data.cpu().numpy(), cols, range(k + m))
    assert np.array_equal(O.symbols(16, full.cpu().numpy(), cols), want)
    assert torch.equal(full, ref)
