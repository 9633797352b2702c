"""Mixed batches (rs_batch_*): stripes of the nine config-3 shapes, ragged lengths that
are mostly not multiples of 64, encode and reconstruct mixed in one CUDA graph. Every
encoded stripe must equal the oracle's encode; every reconstructed stripe must equal
the stripe before erasure (decoding is unique)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(7, 13), (10, 10), (14, 14), (16, 16), (18, 6), (32, 32), (20, 12), (64, 64), (128, 128), (10, 4),
          (17, 3)]


def make_batch(gpu, O, n_stripes, seed, max_len=8192):
    import torch

    rng = np.random.default_rng(seed)
    codecs = {s: gpu.ReedSolomon(*s) for s in SHAPES}
    stripes = []
    for _ in range(n_stripes):
        k, m = SHAPES[int(rng.integers(len(SHAPES)))]
        length = int(np.exp(rng.uniform(np.log(33), np.log(max_len))))
        stride = (length + 255) // 256 * 256
        data = rng.integers(0, 256, size=(k, length), dtype=np.uint8)
        full = np.concatenate([data, O.encode8(k, m, data)])
        op = gpu.RECONSTRUCT if rng.random() < 0.25 else gpu.ENCODE
        present = None
        host = np.zeros((k + m, stride), np.uint8)
        if op == gpu.ENCODE:
            host[:k, :length] = data
            host[k:, :length] = 0xA5
        else:
            e = int(rng.integers(1, m + 1))
            present = np.ones(k + m, np.uint8)
            present[rng.choice(k + m, size=e, replace=False)] = 0
            host[:, :length] = full
            host[present == 0, :length] = 0
        dev = torch.from_numpy(host).cuda()
        stripes.append(dict(k=k, m=m, len=length, stride=stride, full=full, op=op, present=present, dev=dev,
                            codec=codecs[(k, m)]))
    return stripes


def check(stripes):
    import torch

    torch.cuda.synchronize()
    for i, s in enumerate(stripes):
        got = s["dev"].cpu().numpy()[:, : s["len"]]
        assert np.array_equal(got, s["full"]), (i, s["k"], s["m"], s["len"], s["op"])


@pytest.mark.parametrize("flags", [0, 1, 2])
def test_mixed_batch_matches_oracle(gpu, O, flags):
    stripes = make_batch(gpu, O, 60, 100 + flags)
    items = [(s["codec"], s["dev"], s["stride"], s["len"], s["op"], s["present"]) for s in stripes]
    b = gpu.Batch(items, flags=flags)
    assert b.statuses == [0] * len(stripes)
    st = b.stats()
    assert st["fft_items"] + st["matrix_items"] == len(stripes)
    if flags & 1:
        assert st["fft_items"] == 0
    b.launch()
    check(stripes)
    # A replay recomputes the same bytes (reconstruct outputs are not read as inputs).
    for s in stripes:
        if s["op"] == gpu.ENCODE:
            s["dev"][s["k"]:, : s["len"]] = 0
    b.launch()
    check(stripes)


def test_batch_statuses(gpu, O):
    import torch

    rs = gpu.ReedSolomon(4, 2)
    rows = torch.zeros((6, 256), dtype=torch.uint8, device="cuda")
    items = [
        (rs, rows, 256, 100, gpu.RECONSTRUCT, [1, 1, 1, 0, 0, 0]),  # 3 < k present
        (rs, rows, 256, 0, gpu.ENCODE, None),                         # empty shard
        (rs, rows, 64, 100, gpu.ENCODE, None),                        # stride < len
        (rs, rows, 256, 100, gpu.RECONSTRUCT, [1] * 6),               # nothing to do
        (rs, rows, 256, 100, gpu.ENCODE, None),                       # fine
    ]
    b = gpu.Batch(items)
    assert [gpu.ERROR_NAMES.get(s, s) for s in b.statuses] == [
        "TooFewShardsPresent", "EmptyShard", "IncorrectShardSize", 0, 0]
    b.launch()
    torch.cuda.synchronize()
