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
    rs.set_route("fft")  # also for the short shards below
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
    # Both routes against the oracle at sampled symbol columns (both planes), every
    # parity shard: the column evaluator is O(k) per point and column.
    cols = _sample_cols(S // 2, 16, seed=11)
    for s in range(stripes):
        data = d[s].cpu().numpy()
        want = O.eval_columns(16, k, data, cols, range(k, k + m))
        assert np.array_equal(O.symbols(16, p_fft[s].cpu().numpy(), cols), want), s


def _sample_cols(n_sym, count, seed):
    """count symbol columns out of n_sym: both ends, the 32-symbol group edges next to
    them, and random ones."""
    rng = np.random.default_rng(seed)
    fixed = [0, 31, 32, n_sym - 33, n_sym - 1]
    rest = rng.choice(n_sym, size=count - len(fixed), replace=False)
    return sorted(set(fixed) | set(int(c) for c in rest))


def test_fft_route_4096x12288_cosets(gpu, O):
    """(4096, 12288) at 2 KiB shards on the FFT route (many forward cosets) and on the
    matrix route: equal to each other and, at 16 sampled symbol columns of both planes,
    to the oracle's Lagrange evaluation for all 12288 parity shards."""
    import torch

    k, m, S = 4096, 12288, 2048
    rs = gpu.ReedSolomon16(k, m)
    assert rs.encode_route() == "fft"
    rs.set_route("fft")
    g = torch.Generator(device="cuda").manual_seed(9)
    d = torch.randint(0, 256, (1, k, S), dtype=torch.uint8, device="cuda", generator=g)
    p_fft = torch.empty((1, m, S), dtype=torch.uint8, device="cuda")
    p_mat = torch.empty_like(p_fft)
    rs.encode_batch_dev(d, p_fft, S, 1)
    rs.set_route("matrix")
    rs.encode_batch_dev(d, p_mat, S, 1)
    torch.cuda.synchronize()
    cols = _sample_cols(S // 2, 16, seed=12)
    want = O.eval_columns(16, k, d[0].cpu().numpy(), cols, range(k, k + m))
    assert np.array_equal(O.symbols(16, p_fft[0].cpu().numpy(), cols), want)
    assert np.array_equal(O.symbols(16, p_mat[0].cpu().numpy(), cols), want)
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
        rs.set_route("fft")
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
    assert gpu.ReedSolomon16(3, 2).encode_route() == "subfield"  # k + m <= 256
    assert gpu.ReedSolomon16(200, 56).encode_route() == "subfield"
    rs = gpu.ReedSolomon16(3, 2)
    rs.set_route("matrix")
    assert rs.encode_route() == "matrix"
    assert gpu.ReedSolomon16(256, 256).encode_route() == "fft"
    assert gpu.ReedSolomon16(300, 500).encode_route() == "fft"


def test_route_choice_per_call(gpu, O):
    """On the automatic route a single short stripe, where the transform's pass
    launches dominate, takes the matrix kernel; many stripes or a large shape take the
    FFT. Every route gives the oracle's bytes."""
    k, m = 64, 300
    rs = gpu.ReedSolomon16(k, m)
    assert rs.encode_route() == "fft"
    assert rs.encode_route(2048, 1) == "matrix"
    assert rs.encode_route(65536, 256) == "fft"
    assert gpu.ReedSolomon16(512, 512).encode_route(2048, 1) == "fft"
    rs.set_route("fft")
    assert rs.encode_route(2048, 1) == "fft"
    rs.set_route("matrix")
    assert rs.encode_route(65536, 256) == "matrix"
    rs.set_route("auto")
    data = _rand(k, 2048, 11)
    assert np.array_equal(_encode(rs, data, m), O.encode16(k, m, data))


@pytest.mark.parametrize("k,m", [(7, 13), (2, 1), (32, 32), (100, 156), (3, 250)])
def test_subfield_route(gpu, O, k, m):
    """k + m <= 256: every coefficient lies in GF(2^8), so the automatic route runs
    the GF(2^8) codec over both byte planes. Encode (host, device pointers, strided
    batch), verify and reconstruct give the tower oracle's bytes and the tower
    kernels' bytes; the tower's own checks (even, non-zero lengths) still apply."""
    import torch

    rs = gpu.ReedSolomon16(k, m)
    assert rs.encode_route() == "subfield" and rs.encode_route(2048, 1) == "subfield"
    if (k, m) == (100, 156):
        # No compiled GF(2^8) kernel for this shape: a large batch is estimated faster
        # on the tower FFT than on the GF(2^8) matrix kernel.
        assert rs.encode_route(16384, 64) == "fft"
    else:
        assert rs.encode_route(2048, 64) == "subfield"
    for length in [2, 66, 130, 2048, 4098]:
        data = _rand(k, length, 3 * k + m + length)
        want = O.encode16(k, m, data)
        assert np.array_equal(_encode(rs, data, m), want), (k, m, length)
        full = [data[i].copy() for i in range(k)] + [want[j].copy() for j in range(m)]
        assert rs.verify(full)
        erased = [int(e) for e in np.random.default_rng(length).choice(k + m, size=m, replace=False)]
        shards = _erase(full, erased)
        rs.reconstruct([(s, i not in erased) for i, s in enumerate(shards)])
        assert np.array_equal(np.array(shards), np.array(full)), (k, m, length, erased)
    with pytest.raises(gpu.RsError):
        _encode(rs, _rand(k, 65, 1), m)  # odd length: the tower's IncorrectShardSize
    # Device-resident: strided batch and pointer table against the forced tower kernels.
    S, stripes = 4098, 3
    g = torch.Generator(device="cuda").manual_seed(k + m)
    d = torch.randint(0, 256, (stripes, k, S), dtype=torch.uint8, device="cuda", generator=g)
    p_sub = torch.empty((stripes, m, S), dtype=torch.uint8, device="cuda")
    p_mat = torch.empty_like(p_sub)
    rs.encode_batch_dev(d, p_sub, S, stripes)
    rs.set_route("matrix")
    rs.encode_batch_dev(d, p_mat, S, stripes)
    rs.set_route("auto")
    ptr_shards = [d[1, i].clone() for i in range(k)] + [torch.zeros(S, dtype=torch.uint8, device="cuda")
                                                        for _ in range(m)]
    rs.encode_dev(ptr_shards)
    torch.cuda.synchronize()
    assert torch.equal(p_sub, p_mat)
    assert all(torch.equal(ptr_shards[k + j], p_mat[1, j]) for j in range(m))


def test_subfield_shape_batch_on_tower_fft(gpu):
    """(100,156) x 64 stripes of 16 KiB takes the tower FFT on the automatic route; its
    bytes equal the tower matrix kernel's."""
    import torch

    k, m, S, stripes = 100, 156, 16384, 64
    rs = gpu.ReedSolomon16(k, m)
    assert rs.encode_route(S, stripes) == "fft"
    g = torch.Generator(device="cuda").manual_seed(17)
    d = torch.randint(0, 256, (stripes, k, S), dtype=torch.uint8, device="cuda", generator=g)
    p_auto = torch.empty((stripes, m, S), dtype=torch.uint8, device="cuda")
    p_mat = torch.empty_like(p_auto)
    rs.encode_batch_dev(d, p_auto, S, stripes)
    rs.set_route("matrix")
    rs.encode_batch_dev(d, p_mat, S, stripes)
    torch.cuda.synchronize()
    assert torch.equal(p_auto, p_mat)


def _erase(full, erased):
    shards = [s.copy() for s in full]
    for e in erased:
        shards[e][:] = 0
    return shards


@pytest.mark.parametrize("k,m", [(2, 1), (3, 2), (4, 4), (7, 13), (16, 16), (33, 31), (100, 50), (17, 200),
                                 (300, 200)])
def test_fft_decode_rebuilds_every_pattern(gpu, O, k, m):
    """Erasure decoding on the FFT route (error locator, formal derivative) gives back
    the original shards for random patterns of 1..m erasures, and data-only leaves the
    absent parity untouched."""
    rs = gpu.ReedSolomon16(k, m)
    rs.set_route("fft")
    rng = np.random.default_rng(k * 7 + m)
    n = k + m
    for length in [2, 66, 1026]:
        if k * m * length > 40_000_000:
            continue
        data = _rand(k, length, length + k)
        full = np.concatenate([data, O.encode16(k, m, data)])
        patterns = [[0], [k - 1], list(range(k, n)), list(range(min(m, k)))]
        patterns += [sorted(rng.choice(n, size=int(rng.integers(1, m + 1)), replace=False).tolist())
                     for _ in range(4)]
        for erased in patterns:
            shards = _erase(full, erased)
            rs.reconstruct([(s, i not in erased) for i, s in enumerate(shards)])
            assert np.array_equal(np.array(shards), full), (k, m, length, erased)
            shards = _erase(full, erased)
            rs.reconstruct_data([(s, i not in erased) for i, s in enumerate(shards)])
            for i in range(n):
                want = full[i] if (i < k or i not in erased) else np.zeros(length, np.uint8)
                assert np.array_equal(shards[i], want), (k, m, length, erased, i)


def test_fft_decode_device_and_large(gpu):
    """Device-resident shards; (1024,1024) and (4096,12288) with m erasures, FFT decode
    against the matrix route."""
    import torch

    for k, m, S in [(1024, 1024, 2048), (4096, 12288, 2048), (1000, 3000, 66)]:
        n = k + m
        rs = gpu.ReedSolomon16(k, m)
        g = torch.Generator(device="cuda").manual_seed(k)
        rows = torch.zeros((n, S), dtype=torch.uint8, device="cuda")
        rows[:k] = torch.randint(0, 256, (k, S), dtype=torch.uint8, device="cuda", generator=g)
        rs.encode_batch_dev(rows[:k], rows[k:], S, 1)
        torch.cuda.synchronize()
        full = rows.clone()
        present = np.ones(n, np.uint8)
        present[np.random.default_rng(k).choice(n, size=m, replace=False)] = 0
        for route in ("fft", "matrix"):
            rs2 = gpu.ReedSolomon16(k, m)
            rs2.set_route(route)
            work = full.clone()
            work[torch.from_numpy(present == 0).cuda()] = 0
            rs2.reconstruct_dev([work[i] for i in range(n)], present.tolist(), S)
            torch.cuda.synchronize()
            assert torch.equal(work, full), (k, m, route)


def test_decode_route_choice(gpu, O):
    """The automatic choice takes the FFT decoder where many shards are rebuilt over
    many survivors, and still rebuilds exactly."""
    k, m, length = 512, 512, 64
    rs = gpu.ReedSolomon16(k, m)
    data = _rand(k, length, 5)
    full = np.concatenate([data, O.encode16(k, m, data)])
    erased = list(range(0, 2 * k, 2))  # every other shard: 512 erasures
    shards = _erase(full, erased)
    rs.reconstruct([(s, i not in erased) for i, s in enumerate(shards)])
    assert np.array_equal(np.array(shards), full)


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_both_pass_kernels_match_the_oracle(gpu, O, variant):
    """The tower FFT pass kernel with constants through shared-memory masks (0), through
    compiled networks selected by the warp-uniform constant (1), and the latter in
    passes of four levels through shared memory, of five for one pass when the level
    count is odd (2; 32 and 128 registers: one five-level pass, 512: five and four): the
    oracle's bytes on shapes with one and several cosets."""
    L = gpu.load()
    old = L.rs_set_fft16_pass(variant)
    try:
        for k, m, length in [(8, 8, 66), (32, 96, 130), (100, 50, 64), (256, 300, 34), (1024, 64, 66)]:
            rs = gpu.ReedSolomon16(k, m)
            rs.set_route("fft")
            data = _rand(k, length, k + m + variant)
            assert np.array_equal(_encode(rs, data, m), O.encode16(k, m, data)), (k, m, length)
        # The erasure decoder's load, derivative and store kernels under the same switch.
        rng = np.random.default_rng(40 + variant)
        for k, m, length in [(7, 13, 66), (100, 50, 130), (300, 200, 34)]:
            rs = gpu.ReedSolomon16(k, m)
            rs.set_route("fft")
            n = k + m
            data = _rand(k, length, 3 * k + variant)
            full = np.concatenate([data, O.encode16(k, m, data)])
            for erased in ([0], list(range(k, n)),
                           sorted(rng.choice(n, size=m, replace=False).tolist())):
                shards = _erase(full, erased)
                rs.reconstruct([(sh, i not in erased) for i, sh in enumerate(shards)])
                assert np.array_equal(np.array(shards), full), (k, m, erased)
    finally:
        L.rs_set_fft16_pass(old)


def test_pass_kernel_variants_agree_on_large_batches(gpu, O):
    """Launches with several items per CTA and more items than one grid stride: pass
    variants 0, 1 and 2 give the same bytes, and stripe 0 equals the oracle (odd and
    even level counts: 512 and 1024 registers)."""
    import torch

    L = gpu.load()
    old = L.rs_set_fft16_pass(1)
    try:
        for k, m, S, stripes in [(256, 256, 8192, 17), (1000, 24, 4098, 5), (500, 40, 4098, 9)]:
            rs = gpu.ReedSolomon16(k, m)
            rs.set_route("fft")
            g = torch.Generator(device="cuda").manual_seed(k)
            d = torch.randint(0, 256, (stripes, k, S), dtype=torch.uint8, device="cuda", generator=g)
            outs = []
            for variant in (1, 2, 0):
                L.rs_set_fft16_pass(variant)
                p = torch.full((stripes, m, S), 0xA5, dtype=torch.uint8, device="cuda")
                rs.encode_batch_dev(d, p, S, stripes)
                torch.cuda.synchronize()
                outs.append(p)
            assert all(torch.equal(outs[0], o) for o in outs[1:]), (k, m)
            host = d[0].cpu().numpy()
            assert np.array_equal(outs[1][0].cpu().numpy(), O.encode16(k, m, host)), (k, m)
    finally:
        L.rs_set_fft16_pass(old)
