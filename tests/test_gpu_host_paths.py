"""Host-memory entry points, the calls a real caller makes first (the reference's
encode(&mut [T]) over separately allocated shards, src/reedsolomon.rs:271-351):

* rs8_encode_batch, the pipelined many-stripe path, over more than its 64 MiB chunk
  size, from pinned and from pageable memory, at a shard length that is not a multiple
  of 16 (pitched device rows) and with stripes laid out data-then-parity (strided);
* rs8_encode on one stripe large enough to be cut into column chunks that rotate over
  the pipeline streams (with a ragged last chunk), from pageable and pinned shards.

Parity is checked against the oracle's scalar encode at sampled columns (encoding is
column-wise) and, on every byte, against the device-resident batched encode.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cols(length, rng, count=2048):
    """Sampled byte columns: both ends, 16-byte and chunk edges, and random ones."""
    fixed = {0, 1, 15, 16, length - 1, length - 2}
    for edge in (1 << 18, 2 << 18, 3 << 18, 4 << 18):
        if edge < length:
            fixed |= {edge - 1, edge}
    rest = rng.choice(length, size=min(length, count), replace=False)
    return np.array(sorted(fixed | set(int(c) for c in rest)))


def _oracle_check(O, k, m, data, parity, rng):
    """data: (k, len), parity: (m, len) of one stripe."""
    cols = _cols(data.shape[1], rng)
    d = np.ascontiguousarray(data[:, cols])
    assert np.array_equal(parity[:, cols], O.encode8(k, m, d))


def _device_parity(gpu, k, m, data):
    """Every stripe's parity from the device-resident batched path: (S, m, len)."""
    import torch

    rs = gpu.ReedSolomon(k, m)
    S, _, length = data.shape
    d = torch.from_numpy(np.ascontiguousarray(data)).cuda()
    p = torch.empty((S, m, length), dtype=torch.uint8, device="cuda")
    rs.encode_batch_dev(d, p, length, S)
    torch.cuda.synchronize()
    return p.cpu().numpy()


@pytest.mark.parametrize("pinned", [True, False])
def test_host_batch_over_chunk_boundaries(gpu, O, pinned):
    """RS(10,10), 11 stripes of 1 MiB + 5 bytes (about 110 MiB of data, so the 64 MiB
    chunks split it three ways with a partial last chunk; rows pitched on the device)."""
    import torch

    k, m, length, S = 10, 10, (1 << 20) + 5, 11
    rng = np.random.default_rng(31 + pinned)
    if pinned:
        data = torch.empty((S, k, length), dtype=torch.uint8, pin_memory=True).numpy()
        parity = torch.zeros((S, m, length), dtype=torch.uint8, pin_memory=True).numpy()
    else:
        data = np.empty((S, k, length), np.uint8)
        parity = np.zeros((S, m, length), np.uint8)
    data[:] = rng.integers(0, 256, size=data.shape, dtype=np.uint8)
    rs = gpu.ReedSolomon(k, m)
    rs.encode_batch_host(data, parity, length, S)
    assert np.array_equal(parity, _device_parity(gpu, k, m, data))
    for s in (0, 5, S - 1):
        _oracle_check(O, k, m, data[s], parity[s], rng)


def test_host_batch_strided_stripes(gpu, O):
    """Stripes stored whole (k data rows then m parity rows), 36 stripes of RS(32,32) x
    64 KiB + 16 (144 MiB): data and parity strides of n rows."""
    k, m, length, S = 32, 32, (64 << 10) + 16, 36
    n = k + m
    rng = np.random.default_rng(33)
    stripes = rng.integers(0, 256, size=(S, n, length), dtype=np.uint8)
    want = _device_parity(gpu, k, m, stripes[:, :k])
    stripes[:, k:] = 0
    rs = gpu.ReedSolomon(k, m)
    flat = stripes.reshape(-1)
    rs.encode_batch_host(flat, flat[k * length:], length, S, data_stride=n * length, parity_stride=n * length)
    assert np.array_equal(stripes[:, k:], want)
    _oracle_check(O, k, m, stripes[S - 1, :k], stripes[S - 1, k:], rng)


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("length", [(1 << 20) + 333, (4 << 20) + 333])
def test_single_stripe_host_encode_in_column_chunks(gpu, O, pinned, length):
    """One RS(32,32) stripe of separately allocated shards (the reference's Vec<u8>
    shards): at 1 MiB + 333 bytes the stripe is gathered into pinned memory by host
    threads in 1 MiB pieces (a ragged last piece per shard); at 4 MiB + 333 bytes (more
    than 256 MiB of shards) it goes through the column-chunk pipeline, with a ragged
    last chunk."""
    import torch

    k, m = 32, 32
    rng = np.random.default_rng(35 + pinned)
    shards = []
    for i in range(k + m):
        if pinned:
            a = torch.empty(length, dtype=torch.uint8, pin_memory=True).numpy()
        else:
            a = np.empty(length, np.uint8)
        a[:] = rng.integers(0, 256, size=length, dtype=np.uint8) if i < k else 0xA5
        shards.append(a)
    rs = gpu.ReedSolomon(k, m)
    rs.encode(shards)
    data = np.stack(shards[:k])
    parity = np.stack(shards[k:])
    assert np.array_equal(parity, _device_parity(gpu, k, m, data[None])[0])
    _oracle_check(O, k, m, data, parity, rng)
    assert rs.verify(shards)


@pytest.mark.parametrize("staging", [1, 0])
def test_host_calls_with_and_without_pinned_staging(gpu, O, staging):
    """Host-pointer encode (and encode_rows), verify and reconstruct of both coders, with
    the rows gathered into
    pinned memory (1, the default) or copied shard by shard (0): the oracle's bytes.
    Covers a tower shape with the FFT encode and decoder (k + m > 256) and one on the
    tower matrix kernels."""
    L = gpu.load()
    old = L.rs_set_host_staging(staging)
    try:
        rng = np.random.default_rng(40 + staging)
        for k, m, length in [(32, 32, 4096 + 3), (10, 4, 70000)]:
            data = rng.integers(0, 256, size=(k, length), dtype=np.uint8)
            full = np.concatenate([data, O.encode8(k, m, data)])
            rs = gpu.ReedSolomon(k, m)
            shards = [s.copy() for s in data] + [np.zeros(length, np.uint8) for _ in range(m)]
            rs.encode(shards)
            assert np.array_equal(np.array(shards), full), (k, m)
            rows = rs.encode_rows(np.ascontiguousarray(data).reshape(-1), length)
            assert np.array_equal(np.asarray(rows).reshape(m, length), full[k:]), (k, m)
            assert rs.verify(shards)
            shards[k][-1] ^= 1
            assert not rs.verify(shards)
            shards[k][-1] ^= 1
            erased = set(rng.choice(k + m, size=m, replace=False).tolist())
            for e in erased:
                shards[e][:] = 0
            rs.reconstruct([(s, i not in erased) for i, s in enumerate(shards)])
            assert np.array_equal(np.array(shards), full), (k, m)
        for k, m, length, route in [(300, 200, 66, "fft"), (20, 300, 130, "matrix")]:
            data = rng.integers(0, 256, size=(k, length), dtype=np.uint8)
            full = np.concatenate([data, O.encode16(k, m, data)])
            rs = gpu.ReedSolomon16(k, m)
            rs.set_route(route)
            shards = [s.copy() for s in data] + [np.zeros(length, np.uint8) for _ in range(m)]
            rs.encode(shards)
            assert np.array_equal(np.array(shards), full), (k, m)
            assert rs.verify(shards)
            shards[k][0] ^= 1
            assert not rs.verify(shards)
            shards[k][0] ^= 1
            erased = set(rng.choice(k + m, size=m, replace=False).tolist())
            for e in erased:
                shards[e][:] = 0
            rs.reconstruct([(s, i not in erased) for i, s in enumerate(shards)])
            assert np.array_equal(np.array(shards), full), (k, m)
    finally:
        L.rs_set_host_staging(old)
