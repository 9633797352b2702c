"""GF(2^8) encode on the B200 through the C ABI, byte-identical to the oracle.

Mirrors the reference's tests: encode == fused == scalar over shapes and tail lengths
(src/reedsolomon.rs:944-970), staged/FFT == scalar (:997-1021), encode_sep == encode
(:972-995), encode_rows == encode (:915-942), verify blocks (:1160-1185), the
per-coefficient slice kernels (src/gf/x86.rs tests), plus the reference's own generated
FFT program outputs.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def lcg_data(n, seed):
    """deterministic_data of src/reedsolomon.rs:897-904."""
    out = np.empty(n, np.uint8)
    s = seed
    for i in range(n):
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = (s >> 16) & 0xFF
    return out


def rand_data(k, length, seed):
    return np.random.default_rng(seed).integers(0, 256, size=(k, length), dtype=np.uint8)


def encode_gpu(rs, data, m):
    k, length = data.shape
    shards = [data[i].copy() for i in range(k)] + [np.full(length, 0xA5, np.uint8) for _ in range(m)]
    rs.encode(shards)
    return np.array(shards[k:]) if m else np.zeros((0, length), np.uint8)


SHAPES = [(7, 13), (10, 10), (20, 10), (4, 2), (6, 4), (17, 17), (32, 32), (16, 16), (14, 14),
          (18, 6), (20, 12), (1, 1), (2, 2), (8, 8), (64, 64), (128, 128), (255, 1), (1, 255),
          (6, 3), (8, 4), (10, 4), (12, 4), (16, 4), (17, 3)]
LENGTHS = [1, 15, 16, 17, 31, 32, 33, 63, 64, 65, 100, 987, 1024, 4103, 65536]


@pytest.mark.parametrize("k,m", SHAPES)
def test_encode_matches_oracle(gpu, O, k, m):
    rs = gpu.ReedSolomon(k, m)
    for length in LENGTHS:
        data = rand_data(k, length, k * 1000 + length)
        want = O.encode8(k, m, data)
        for route in ("auto", "matrix", "fft"):
            rs.set_route(route)
            got = encode_gpu(rs, data, m)
            assert np.array_equal(got, want), (k, m, length, route)


@pytest.mark.parametrize("k,m", [(32, 32), (10, 10), (16, 16)])
def test_every_tail_length(gpu, O, k, m):
    rs = gpu.ReedSolomon(k, m)
    for length in range(1, 130):
        data = rand_data(k, length, length)
        want = O.encode8(k, m, data)
        for route in ("matrix", "fft"):
            rs.set_route(route)
            assert np.array_equal(encode_gpu(rs, data, m), want), (k, m, length, route)


def test_reference_program_outputs(gpu, golden):
    """Columns and parity produced by the reference's own generated programs."""
    for p in golden["fft_programs"]:
        k, m = p["k"], p["m"]
        cols = np.array(p["columns"], np.uint8)  # (64, k)
        data = cols.T.copy()
        rs = gpu.ReedSolomon(k, m)
        for route in ("matrix", "fft"):
            rs.set_route(route)
            assert encode_gpu(rs, data, m).T.tolist() == p["parity"], (k, m, route)


def test_deterministic_data_shapes(gpu, O):
    """encode_fused_matches_encode's data generator and shapes."""
    for k, m in [(7, 13), (10, 10), (20, 10), (4, 2), (6, 4), (17, 17)]:
        rs = gpu.ReedSolomon(k, m)
        for length in [1, 15, 16, 17, 31, 32, 63, 100, 1024, 10000]:
            data = lcg_data(k * length, 0x9E3779B9).reshape(k, length)
            assert np.array_equal(encode_gpu(rs, data, m), O.encode8(k, m, data))


def test_encode_sep_matches_encode(gpu):
    for k, m in [(7, 13), (10, 10), (32, 32), (4, 2), (18, 6)]:
        rs = gpu.ReedSolomon(k, m)
        for length in [16, 100, 987, 1024]:
            data = lcg_data(k * length, 0x12345678).reshape(k, length)
            combined = encode_gpu(rs, data, m)
            parity = [np.zeros(length, np.uint8) for _ in range(m)]
            rs.encode_sep([data[i] for i in range(k)], parity)
            assert np.array_equal(np.array(parity), combined)


def test_encode_rows_matches_encode(gpu):
    k, m, row_len = 6, 4, 293
    rs = gpu.ReedSolomon(k, m)
    data = lcg_data(k * row_len, 0x12345678)
    want = encode_gpu(rs, data.reshape(k, row_len), m).reshape(-1)
    assert np.array_equal(rs.encode_rows(data, row_len), want)
    buf = np.zeros(m * row_len, np.uint8)
    rs.encode_rows_into(data, row_len, buf)
    assert np.array_equal(buf, want)
    with pytest.raises(gpu.RsError) as e:
        rs.encode_rows_into(data, row_len, np.zeros(m * row_len + 1, np.uint8))
    assert e.value.name == "IncorrectShardSize"
    with pytest.raises(AssertionError):
        rs.encode_rows(data[:-1], row_len)
    assert rs.encode_rows(np.zeros(0, np.uint8), 0).size == 0


def test_encode_errors(gpu):
    rs = gpu.ReedSolomon(4, 2)
    mk = lambda n, ln: [np.zeros(ln, np.uint8) for _ in range(n)]
    for shards, name in [(mk(5, 8), "TooFewShards"), (mk(7, 8), "TooManyShards"),
                         (mk(6, 0), "EmptyShard")]:
        with pytest.raises(gpu.RsError) as e:
            rs.encode(shards)
        assert e.value.name == name
    bad = mk(6, 8)
    bad[3] = np.zeros(9, np.uint8)
    with pytest.raises(gpu.RsError) as e:
        rs.encode(bad)
    assert e.value.name == "IncorrectShardSize"
    # encode_sep count errors, and its len-0 quirk (no EmptyShard).
    for d, p, name in [(3, 2, "TooFewDataShards"), (5, 2, "TooManyDataShards"),
                       (4, 1, "TooFewParityShards"), (4, 3, "TooManyParityShards")]:
        with pytest.raises(gpu.RsError) as e:
            rs.encode_sep(mk(d, 8), mk(p, 8))
        assert e.value.name == name
    rs.encode_sep(mk(4, 0), mk(2, 0))


def test_verify_blocks(gpu):
    k, m = 4, 3
    rs = gpu.ReedSolomon(k, m)
    for length in [100, 32 * 1024, 32 * 1024 + 17]:
        data = lcg_data(k * length, 0x12345678).reshape(k, length)
        shards = [data[i] for i in range(k)] + list(encode_gpu(rs, data, m))
        assert rs.verify(shards)
        for pos in [0, length // 2, length - 1]:
            bad = [s.copy() for s in shards]
            bad[k][pos] ^= 1
            assert not rs.verify(bad)


def test_mul_slice_all_coefficients(gpu, O):
    table = O.gf8_mul_table()
    rng = np.random.default_rng(9)
    for length in [0, 1, 7, 31, 32, 33, 127, 128, 129, 1000, 65537]:
        x = rng.integers(0, 256, size=length, dtype=np.uint8)
        for c in range(256):
            if length > 1000 and c % 17:
                continue
            out = rng.integers(0, 256, size=length, dtype=np.uint8)
            base = out.copy()
            gpu.mul_slice_xor(out, x, c)
            assert np.array_equal(out, base ^ table[c][x])
            gpu.mul_slice(out, x, c)
            assert np.array_equal(out, table[c][x])
    with pytest.raises(gpu.RsError):
        gpu.mul_slice(np.zeros(3, np.uint8), np.zeros(4, np.uint8), 2)


def test_encode_route_introspection(gpu):
    assert gpu.ReedSolomon(32, 32).encode_route(1 << 20) == "fft-bitsliced"
    assert gpu.ReedSolomon(20, 12).encode_route(1 << 20) == "generator-bitsliced"
    assert gpu.ReedSolomon(10, 10).encode_route(1 << 16) == "generator-bitsliced"
    assert gpu.ReedSolomon(10, 10).encode_route(32) == "matrix"  # under two column groups
    assert gpu.ReedSolomon(20, 10).encode_route(1 << 20) == "matrix"
    for k, m in [(4, 2), (6, 3), (8, 4), (10, 4), (12, 4), (16, 4), (17, 3)]:
        assert gpu.ReedSolomon(k, m).encode_route(4096) == "generator-bitsliced", (k, m)


def test_clone_and_eq(gpu):
    a = gpu.ReedSolomon(10, 10)
    b = a.clone()
    assert a == b and a != gpu.ReedSolomon(10, 9)
    data = rand_data(10, 300, 3)
    assert np.array_equal(encode_gpu(a, data, 10), encode_gpu(b, data, 10))


def test_batch_encode_device(gpu, O):
    import torch

    for k, m, row_len, stripes in [(32, 32, 4096, 33), (16, 16, 1000, 7), (10, 10, 257, 5), (20, 12, 4096, 9)]:
        rs = gpu.ReedSolomon(k, m)
        rng = np.random.default_rng(k + stripes)
        host = rng.integers(0, 256, size=(stripes, k, row_len), dtype=np.uint8)
        d = torch.from_numpy(host).cuda()
        p = torch.full((stripes, m, row_len), 0xA5, dtype=torch.uint8, device="cuda")
        rs.encode_batch_dev(d, p, row_len, stripes)
        torch.cuda.synchronize()
        got = p.cpu().numpy()
        for s in range(stripes):
            assert np.array_equal(got[s], O.encode8(k, m, host[s])), (k, m, s)


def test_encode_dev_pointers(gpu, O):
    import torch

    k, m, length = 32, 32, 5000
    rs = gpu.ReedSolomon(k, m)
    host = rand_data(k, length, 77)
    bufs = [torch.from_numpy(host[i].copy()).cuda() for i in range(k)]
    bufs += [torch.zeros(length, dtype=torch.uint8, device="cuda") for _ in range(m)]
    for route in ("matrix", "fft"):
        rs.set_route(route)
        rs.encode_dev(bufs)
        torch.cuda.synchronize()
        got = np.array([b.cpu().numpy() for b in bufs[k:]])
        assert np.array_equal(got, O.encode8(k, m, host)), route
    assert rs.verify_dev(bufs, length)


@pytest.mark.parametrize("k,m", [(16, 16), (10, 10)])
def test_encode_dev_unaligned_pointers(gpu, O, k, m):
    """Shards at odd byte offsets take the FFT / generator kernel's byte path; same bytes."""
    import torch

    length = 4099
    rs = gpu.ReedSolomon(k, m)
    host = rand_data(k, length, 78)
    pool = torch.zeros((k + m) * (length + 64), dtype=torch.uint8, device="cuda")
    bufs = [pool[i * (length + 64) + 1 + i: i * (length + 64) + 1 + i + length] for i in range(k + m)]
    for i in range(k):
        bufs[i].copy_(torch.from_numpy(host[i]))
    for route in ("matrix", "fft"):
        rs.set_route(route)
        for b in bufs[k:]:
            b.zero_()
        rs.encode_dev(bufs)
        torch.cuda.synchronize()
        got = np.array([b.cpu().numpy() for b in bufs[k:]])
        assert np.array_equal(got, O.encode8(k, m, host)), route


@pytest.mark.parametrize("k,m", [(32, 32), (16, 16), (10, 10), (10, 4), (64, 64), (128, 128), (20, 12)])
def test_encode_batch_packed_unaligned_rows(gpu, O, k, m):
    """Rows packed back to back at odd lengths start at every offset mod 16, so the
    compiled kernels' unaligned paths all run (a row's first group by bytes, interior
    groups through the aligned 48-byte window, the tail by bytes, stores split at the
    group's edges); the bytes equal the oracle's on every route."""
    import torch

    rng = np.random.default_rng(k * 7 + m)
    stripes = 3
    for length in (33, 63, 65, 95, 97, 100, 129, 987, 4099):
        data = rng.integers(0, 256, size=(stripes, k, length), dtype=np.uint8)
        want = np.stack([O.encode8(k, m, data[s]) for s in range(stripes)])
        d = torch.from_numpy(data.reshape(-1)).cuda()
        for route in ("fft", "auto", "matrix"):
            rs = gpu.ReedSolomon(k, m)
            rs.set_route(route)
            par = torch.full((stripes * m * length,), 0xA5, dtype=torch.uint8, device="cuda")
            rs.encode_batch_dev(d, par, length, stripes)
            torch.cuda.synchronize()
            got = par.cpu().numpy().reshape(stripes, m, length)
            assert np.array_equal(got, want), (k, m, length, route)
