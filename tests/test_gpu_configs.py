"""The measured configurations as tests: configuration 1 exactly as specified, and
configuration 2 at its full stripe count (4096 per launch) with the smallest shard
size, through size-independent properties: the two encode routes agree, encoding is
linear over GF(2^8), and every stripe's own erasure pattern is rebuilt exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_config1_rs10x10_64k(gpu, O):
    """One stripe of 10 x 64 KiB seeded bytes: parity equals the oracle's; erasing 10 of
    the 20 shards chosen uniformly (seeded shuffle) and reconstructing gives the stripe
    back byte for byte."""
    k, m, S = 10, 10, 65536
    rng = np.random.default_rng(1)
    data = rng.integers(0, 256, size=(k, S), dtype=np.uint8)
    rs = gpu.ReedSolomon(k, m)
    shards = [data[i].copy() for i in range(k)] + [np.zeros(S, np.uint8) for _ in range(m)]
    rs.encode(shards)
    assert np.array_equal(np.array(shards[k:]), O.encode8(k, m, data))
    full = [s.copy() for s in shards]
    erased = rng.permutation(k + m)[:m]
    for e in erased:
        shards[e][:] = 0
    rs.reconstruct([(s, i not in erased) for i, s in enumerate(shards)])
    for i in range(k + m):
        assert np.array_equal(shards[i], full[i]), i


@pytest.mark.parametrize("k,m", [(32, 32), (16, 16)])
def test_config2_4096_stripes(gpu, k, m):
    import torch

    S, N = 4096, 4096
    n = k + m
    rs = gpu.ReedSolomon(k, m)
    g = torch.Generator(device="cuda").manual_seed(k)
    rows = torch.randint(0, 256, (N, n, S), dtype=torch.uint8, device="cuda", generator=g)
    stride = n * S
    rs.set_route("fft")
    rs.encode_batch_dev(rows, rows[:, k:], S, N, data_stride=stride, parity_stride=stride)
    fft_par = rows[:, k:].clone()
    rs.set_route("matrix")
    rs.encode_batch_dev(rows, rows[:, k:], S, N, data_stride=stride, parity_stride=stride)
    torch.cuda.synchronize()
    assert torch.equal(rows[:, k:], fft_par)
    # Linearity: parity(a ^ b) == parity(a) ^ parity(b), on the FFT route.
    rs.set_route("fft")
    b = torch.randint(0, 256, (N, n, S), dtype=torch.uint8, device="cuda", generator=g)
    rs.encode_batch_dev(b, b[:, k:], S, N, data_stride=stride, parity_stride=stride)
    c = rows ^ b
    rs.encode_batch_dev(c, c[:, k:], S, N, data_stride=stride, parity_stride=stride)
    torch.cuda.synchronize()
    assert torch.equal(c[:, k:], rows[:, k:] ^ b[:, k:])
    del b, c
    # Independent erasure patterns of 1..m shards per stripe, rebuilt in one call.
    rng = np.random.default_rng(2)
    present = np.ones((N, n), np.uint8)
    for s in range(N):
        present[s, rng.choice(n, size=int(rng.integers(1, m + 1)), replace=False)] = 0
    full = rows.clone()
    rows[torch.from_numpy(present == 0).cuda()] = 0
    st = rs.reconstruct_batch_dev(rows, N, S, present)
    torch.cuda.synchronize()
    assert st == [0] * N
    assert torch.equal(rows, full)
