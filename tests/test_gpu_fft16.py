"""FFT route of ReedSolomon16: the bitsliced tower LCH transform (src/fft16.rs) must give
the bytes of the symbol-wise oracle and of the matrix route, for power-of-two k and for
k between powers of two (the recursive interpolation of src/fft.rs:198-239), parity
counts below, at and across multiples of the transform size (several cosets), and shard
lengths that are not multiples of the 32-symbol groups.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand(k, length, seed):
    return np.random.default_rng(seed).integers(0, 256, size=(k, length), dtype=np.uint8)


def _encode(rs, data, m):
    k, length = data.shape
    shards = [data[i].copy() for i in range(k)] + [np.full(length, 0xA5, np.uint8) for _ in range(m)]
    rs.encode(shards)
    return np.array(shards[k:])


@pytest.mark.parametrize("k", [2, 3, 4, 5, 6, 7, 8, 11, 16, 17, 24, 32, 33, 63, 64, 100, 128, 200, 256, 300])
def test_fft_route_matches_oracle(gpu, O, k):
    for m in sorted({1, max(1, k // 2), k, k + 1, 2 * k, 3 * k - 1}):
        rs = gpu.ReedSolomon16(k, m)
        rs.set_route("fft")
        assert rs.encode_route() == "fft"
        for length in [2, 64, 66, 130, 2048]:
            if k * m * length > 30_000_000:
                continue
            data = _rand(k, length, 7 * k + m + length)
            assert np.array_equal(_encode(rs, data, m), O.encode16(k, m, data)), (k, m, length)


def test_fft_route_1024x1024(gpu, O):
    import torch

    k = m = 1024
    rs = gpu.ReedSolomon16(k, m)
    assert rs.encode_route() == "fft"  # picked automatically at this shape
    data = _rand(k, 66, 1)  # short shards keep the oracle fast
    assert np.array_equal(_encode(rs, data, m), O.encode16(k, m, data))
    # 2 KiB shards, several stripes: FFT route == matrix route on the device.
    S, stripes = 2048, 3
    g = torch.Generator(device="cuda").manual_seed(5)
    d = torch.randint(0, 256, (stripes, k, S), dtype=torch.uint8, device="cuda", generator=g)
    p_fft = torch.empty((stripes, m, S), dtype=torch.uint8, device="cuda")
    p_mat = torch.empty_like(p_fft)
    rs.encode_batch_dev(d, p_fft, S, stripes)
    rs.set_route("matrix")
    rs.encode_batch_dev(d, p_mat, S, stripes)
    torch.cuda.synchronize()
    assert torch.equal(p_fft, p_mat)


def test_fft_route_4096x12288_cosets(gpu):
    import torch

    k, m, S = 4096, 12288, 2048
    rs = gpu.ReedSolomon16(k, m)
    assert rs.encode_route() == "fft"
    g = torch.Generator(device="cuda").manual_seed(9)
    d = torch.randint(0, 256, (1, k, S), dtype=torch.uint8, device="cuda", generator=g)
    p_fft = torch.empty((1, m, S), dtype=torch.uint8, device="cuda")
    p_mat = torch.empty_like(p_fft)
    rs.encode_batch_dev(d, p_fft, S, 1)
    rs.set_route("matrix")
    rs.encode_batch_dev(d, p_mat, S, 1)
    torch.cuda.synchronize()
    assert torch.equal(p_fft, p_mat)


def test_fft_route_device_pointer_table(gpu, O):
    import torch

    k, m, length = 64, 100, 322
    rs = gpu.ReedSolomon16(k, m)
    rs.set_route("fft")
    data = _rand(k, length, 3)
    shards = [torch.from_numpy(data[i]).cuda() for i in range(k)] + \
             [torch.zeros(length, dtype=torch.uint8, device="cuda") for _ in range(m)]
    rs.encode_dev(shards)
    torch.cuda.synchronize()
    got = np.array([s.cpu().numpy() for s in shards[k:]])
    assert np.array_equal(got, O.encode16(k, m, data))


def test_fft_route_large_odd_k(gpu):
    import torch

    for k, m in [(1000, 3000), (2500, 700), (129, 12000)]:
        S = 1026
        rs = gpu.ReedSolomon16(k, m)
        assert rs.encode_route() == "fft"
        g = torch.Generator(device="cuda").manual_seed(k)
        d = torch.randint(0, 256, (2, k, S), dtype=torch.uint8, device="cuda", generator=g)
        p_fft = torch.empty((2, m, S), dtype=torch.uint8, device="cuda")
        p_mat = torch.empty_like(p_fft)
        rs.encode_batch_dev(d, p_fft, S, 2)
        rs.set_route("matrix")
        rs.encode_batch_dev(d, p_mat, S, 2)
        torch.cuda.synchronize()
        assert torch.equal(p_fft, p_mat), (k, m)


def test_route_choice(gpu):
    assert gpu.ReedSolomon16(3, 2).encode_route() == "matrix"  # too small to pay off
    assert gpu.ReedSolomon16(2, 1).encode_route() == "matrix"
    assert gpu.ReedSolomon16(256, 256).encode_route() == "fft"
    assert gpu.ReedSolomon16(300, 500).encode_route() == "fft"
