"""The measured configurations as tests: configuration 1 exactly as specified, and
configuration 2 at its full stripe count (4096 per launch) at 4 KiB and 64 KiB shards
and at 1 MiB on a 64-stripe launch: sampled stripes against the oracle, the two
encode routes equal on every byte, encoding linear over GF(2^8) (4 KiB), and every
stripe's own erasure pattern rebuilt exactly.
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


def _check_sampled_stripes(O, rows, k, m, S, n_check, seed):
    """n_check stripes chosen at random (the first and last always) against the oracle's
    encode: whole shards up to 4 KiB, else 4096 sampled byte columns (both shard ends
    included); encoding is column-wise, so the oracle runs on the sampled columns."""
    import torch

    rng = np.random.default_rng(seed)
    N = rows.shape[0]
    picks = sorted({0, N - 1} | set(int(s) for s in rng.choice(N, size=min(N, n_check) - 2, replace=False)))
    cols = np.arange(S) if S <= 4096 else np.array(
        sorted({0, 1, S - 2, S - 1} | set(int(c) for c in rng.choice(S, size=4092, replace=False))))
    idx = torch.from_numpy(cols).to(rows.device)
    for s in picks:
        stripe = rows[s].index_select(1, idx).cpu().numpy()
        assert np.array_equal(stripe[k:], O.encode8(k, m, stripe[:k])), s


@pytest.mark.parametrize("k,m,S", [(32, 32, 4096), (16, 16, 4096), (32, 32, 65536), (16, 16, 65536)])
def test_config2_4096_stripes(gpu, O, k, m, S):
    """Configuration 2 at 4096 stripes per launch: 32 sampled stripes of the FFT route's
    parity against the oracle, the matrix route equal to it on every stripe, linearity
    (4 KiB), and every stripe's own erasure pattern of 1..m shards rebuilt exactly."""
    import torch

    N = 4096
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
    del fft_par
    _check_sampled_stripes(O, rows, k, m, S, 32, seed=S + k)
    rs.set_route("fft")
    if S <= 4096:
        _linearity(rs, rows, k, n, S, N, g)
    _rebuild_every_pattern(rs, rows, m, n, S, N)


def test_config2_rs32x32_1MiB_64_stripes(gpu, O):
    """RS(32,32) with 1 MiB shards, 64 stripes per launch (4 GiB): FFT-route parity of
    every stripe against the oracle at 4096 sampled columns, the matrix route equal on
    every byte, then per-stripe erasure patterns rebuilt exactly."""
    import torch

    k, m, S, N = 32, 32, 1 << 20, 64
    n = k + m
    rs = gpu.ReedSolomon(k, m)
    g = torch.Generator(device="cuda").manual_seed(77)
    rows = torch.randint(0, 256, (N, n, S), dtype=torch.uint8, device="cuda", generator=g)
    stride = n * S
    rs.set_route("fft")
    rs.encode_batch_dev(rows, rows[:, k:], S, N, data_stride=stride, parity_stride=stride)
    torch.cuda.synchronize()
    _check_sampled_stripes(O, rows, k, m, S, N, seed=78)
    fft_par = rows[:, k:].clone()
    rs.set_route("matrix")
    rs.encode_batch_dev(rows, rows[:, k:], S, N, data_stride=stride, parity_stride=stride)
    torch.cuda.synchronize()
    assert torch.equal(rows[:, k:], fft_par)
    del fft_par
    rs.set_route("fft")
    _rebuild_every_pattern(rs, rows, m, n, S, N)


def _linearity(rs, rows, k, n, S, N, g):
    import torch

    stride = n * S
    b = torch.randint(0, 256, (N, n, S), dtype=torch.uint8, device="cuda", generator=g)
    rs.encode_batch_dev(b, b[:, k:], S, N, data_stride=stride, parity_stride=stride)
    c = rows ^ b
    rs.encode_batch_dev(c, c[:, k:], S, N, data_stride=stride, parity_stride=stride)
    torch.cuda.synchronize()
    assert torch.equal(c[:, k:], rows[:, k:] ^ b[:, k:])


def _rebuild_every_pattern(rs, rows, m, n, S, N):
    """Independent erasure patterns of 1..m shards per stripe, rebuilt in one call."""
    import torch

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
