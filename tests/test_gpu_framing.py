"""Payload framing on the device (rs*_frame_*_dev): a payload is cut into stripes of k
data shards, every stripe encoded, shards erased, and the payload reassembled from any
k shards per stripe, for

* shred-style FEC sets: RS(32,32) with 987-byte shards, the reference's Agave test
  shape (src/reedsolomon.rs:973), many stripes of rows packed back to back;
* the tape outer coder: ReedSolomon16 with k = ceil(groups / 3), m = groups - k and
  shards of ceil(segment / k) bytes rounded up to 64
  (benches/gf16-bench/src/bin/live.rs:1-16), at the live 20-group shape (7,13) and at
  300 groups (100,200, the tower route).

Parity is checked against the oracle, data rows against the payload's bytes in order.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _payload(length, seed):
    import torch

    rng = np.random.default_rng(seed)
    return torch.from_numpy(rng.integers(0, 256, size=length, dtype=np.uint8)).cuda()


def _check_layout(stripes, payload, k, shard_len):
    """Data rows hold the payload's bytes in order, then zeros."""
    S = stripes.shape[0]
    data = stripes[:, :k].reshape(-1).cpu().numpy()
    want = np.zeros(S * k * shard_len, np.uint8)
    want[: payload.numel()] = payload.cpu().numpy()
    assert np.array_equal(data, want)


def _erase(stripes, n, e_max, rng, overflow=()):
    """Erase 1..e_max random shards per stripe (e_max + 1 in the `overflow` stripes)."""
    S = stripes.shape[0]
    present = np.ones((S, n), np.uint8)
    for s in range(S):
        e = e_max + 1 if s in overflow else int(rng.integers(1, e_max + 1))
        present[s, rng.choice(n, size=e, replace=False)] = 0
    import torch

    stripes[torch.from_numpy(present == 0).cuda()] = 0
    return present


def test_shred_sets_round_trip(gpu, O):
    k, m, shard = 32, 32, 987
    rs = gpu.ReedSolomon(k, m)
    payload = _payload((1 << 20) + 17, 41)
    stripes = rs.frame_encode_dev(payload, shard)
    assert stripes.shape[0] == gpu.frame_stripe_count(payload.numel(), k, shard) == 34
    import torch

    torch.cuda.synchronize()
    _check_layout(stripes, payload, k, shard)
    rng = np.random.default_rng(42)
    for s in sorted({0, 17, stripes.shape[0] - 1} | set(int(x) for x in rng.choice(34, 4, replace=False))):
        st = stripes[s].cpu().numpy()
        assert np.array_equal(st[k:], O.encode8(k, m, st[:k])), s
    present = _erase(stripes, k + m, m, rng)
    out, statuses = rs.frame_decode_dev(stripes, shard, present, payload.numel())
    torch.cuda.synchronize()
    assert statuses == [0] * stripes.shape[0]
    assert torch.equal(out, payload)


def test_shred_sets_report_unrecoverable_stripes(gpu):
    """A stripe with more than m shards lost reports TooFewShardsPresent; the other
    stripes' payload bytes are still rebuilt."""
    import torch

    k, m, shard = 32, 32, 987
    rs = gpu.ReedSolomon(k, m)
    payload = _payload(5 * k * shard + 100, 43)
    stripes = rs.frame_encode_dev(payload, shard)
    rng = np.random.default_rng(44)
    present = _erase(stripes, k + m, m, rng, overflow={2})
    out, statuses = rs.frame_decode_dev(stripes, shard, present, payload.numel())
    torch.cuda.synchronize()
    assert gpu.ERROR_NAMES[statuses[2]] == "TooFewShardsPresent"
    assert [s for i, s in enumerate(statuses) if i != 2] == [0] * 5
    per = k * shard
    for s in (0, 1, 3, 4, 5):
        assert torch.equal(out[s * per: (s + 1) * per], payload[s * per: (s + 1) * per]), s


@pytest.mark.parametrize("length", [0, 1, 32 * 987, 32 * 987 + 1])
def test_shred_payload_edges(gpu, length):
    import torch

    k, m, shard = 32, 32, 987
    rs = gpu.ReedSolomon(k, m)
    payload = _payload(length, 45) if length else torch.empty(0, dtype=torch.uint8, device="cuda")
    stripes = rs.frame_encode_dev(payload, shard)
    assert stripes.shape[0] == gpu.frame_stripe_count(length, k, shard)
    if length:
        _check_layout(stripes, payload, k, shard)
        present = np.ones((stripes.shape[0], k + m), np.uint8)
        present[:, :m] = 0
        stripes[:, :m] = 0
    else:
        present = np.ones((0, k + m), np.uint8)
    out, statuses = rs.frame_decode_dev(stripes, shard, present, length)
    torch.cuda.synchronize()
    assert statuses == [0] * stripes.shape[0]
    assert torch.equal(out, payload)


def test_frame_errors(gpu):
    import torch

    rs = gpu.ReedSolomon(4, 2)
    with pytest.raises(gpu.RsError) as e:
        rs.frame_encode_dev(_payload(100, 1), 0)
    assert e.value.name == "EmptyShard"
    rs16 = gpu.ReedSolomon16(4, 2)
    with pytest.raises(gpu.RsError) as e:
        rs16.frame_encode_dev(_payload(100, 1), 33)
    assert e.value.name == "IncorrectShardSize"
    L = gpu.load()
    stripes = torch.zeros((3, 6, 16), dtype=torch.uint8, device="cuda")
    code = L.rs8_frame_encode_dev(rs._h, _payload(100, 1).data_ptr(), 100, 16, stripes.data_ptr(), 3, None)
    assert gpu.ERROR_NAMES[code] == "IncorrectShardSize"  # 100 bytes at 4 x 16 fill 2 stripes


def _symbol_cols(n_sym, rng, count=24):
    return sorted({0, 31, 32, n_sym - 1} | set(int(c) for c in rng.choice(n_sym, size=count, replace=False)))


@pytest.mark.parametrize("groups,segment", [(20, (1 << 20) + 3), (300, 300_001)])
def test_outer_coder_round_trip(gpu, O, groups, segment):
    import torch

    k, m = gpu.outer_shape(groups)
    shard = gpu.outer_shard_bytes(segment, k)
    assert shard % 64 == 0 and k * shard >= segment > k * (shard - 64)
    rs = gpu.ReedSolomon16(k, m)
    payload = _payload(segment, groups)
    stripes = rs.frame_encode_dev(payload, shard)
    assert stripes.shape[0] == 1
    torch.cuda.synchronize()
    _check_layout(stripes, payload, k, shard)
    rng = np.random.default_rng(groups + 1)
    cols = _symbol_cols(shard // 2, rng)
    full = stripes[0].cpu().numpy()
    want = O.eval_columns(16, k, full[:k], cols, range(k + m))
    assert np.array_equal(O.symbols(16, full, cols), want)
    present = _erase(stripes, k + m, m, rng)
    out, statuses = rs.frame_decode_dev(stripes, shard, present, segment)
    torch.cuda.synchronize()
    assert statuses == [0]
    assert torch.equal(out, payload)
