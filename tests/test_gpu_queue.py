"""The persistent work queue (rs_queue_*): one long-running launch coding stripes that
the host pushes while it runs, and its bounded device waits. The stall test makes the
failure on the host (a producer that stops pushing without closing the queue): the
kernel's waits run out, the session ends with RS_ERR_TIMEOUT, work published before is
done, and the device and the queue stay usable. No GPU fault is involved."""
import gc
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _no_frees_during_sessions():
    """Freeing device or pinned memory (cudaFree, cudaFreeHost) synchronizes the device,
    so a codec that the garbage collector destroys while a session runs would hold the
    host until the session's kernel ends at its timeout. Collect first and keep the
    collector off for the test."""
    gc.collect()
    gc.disable()
    try:
        yield
    finally:
        gc.enable()

SHAPES = [(32, 32), (10, 10), (7, 13), (64, 64), (20, 12), (3, 5)]


def _stripes(gpu, O, n, seed):
    """n stripes of mixed shapes and lengths in device memory: (items, want) where want
    holds each stripe's full bytes; encodes start with zeroed parity, reconstructs with
    1..m erased rows zeroed."""
    import torch

    rng = np.random.default_rng(seed)
    codecs = {sh: gpu.ReedSolomon(*sh) for sh in SHAPES}
    items, want, keep = [], [], []
    for i in range(n):
        k, m = SHAPES[i % len(SHAPES)]
        L = int(rng.integers(1, 9000))
        stride = L if i % 3 == 0 else (L + 15) // 16 * 16
        data = rng.integers(0, 256, size=(k, L), dtype=np.uint8)
        full = np.zeros((k + m, stride), np.uint8)
        full[:k, :L] = data
        full[k:, :L] = O.encode8(k, m, data)
        work = full.copy()
        present = None
        if i % 4 == 3:
            present = np.ones(k + m, np.uint8)
            present[rng.choice(k + m, size=int(rng.integers(1, m + 1)), replace=False)] = 0
            work[present == 0] = 0
            op = gpu.RECONSTRUCT
        else:
            work[k:] = 0
            op = gpu.ENCODE
        rows = torch.from_numpy(work.reshape(-1)).cuda()
        keep.append(rows)
        items.append((codecs[(k, m)], rows, stride, L, op, present))
        want.append((full, L))
    return items, want, keep


def _check(items, want):
    import torch

    torch.cuda.synchronize()
    for (codec, rows, stride, L, op, present), (full, L2) in zip(items, want):
        n = full.shape[0]
        got = rows.cpu().numpy().reshape(n, stride)
        assert np.array_equal(got[:, :L], full[:, :L])


def test_queue_codes_stripes_pushed_while_it_runs(gpu, O):
    q = gpu.Queue(max_units=1 << 15, timeout_s=5.0)
    q.start()
    all_items, all_want, keep = [], [], []
    for wave in range(3):
        items, want, k2 = _stripes(gpu, O, 40, seed=wave)
        assert q.push(items) == [0] * len(items)
        all_items += items
        all_want += want
        keep += k2
        time.sleep(0.02)  # the kernel is running meanwhile
    assert q.finish() == 0
    done, published = q.progress()
    assert done == published > 0
    _check(all_items, all_want)
    # A second session on the same queue.
    q.start()
    items, want, k2 = _stripes(gpu, O, 30, seed=9)
    assert q.push(items) == [0] * len(items)
    assert q.finish() == 0
    _check(items, want)


def test_queue_stalled_producer_times_out(gpu, O):
    """The producer stops without closing: every device wait gives up after the timeout,
    the session reports Timeout, the units published before it are finished, and the
    device and the queue keep working."""
    q = gpu.Queue(max_units=4096, timeout_s=0.2)
    items, want, keep = _stripes(gpu, O, 12, seed=21)
    q.start()
    assert q.push(items) == [0] * len(items)
    t0 = time.monotonic()
    code = q.wait()  # nothing more is pushed and the queue is not closed
    elapsed = time.monotonic() - t0
    assert gpu.ERROR_NAMES[code] == "Timeout"
    assert elapsed < 10.0
    done, published = q.progress()
    assert done == published
    _check(items, want)
    # The device is usable: a plain encode, and a new session that closes normally.
    rs = gpu.ReedSolomon(10, 4)
    data = np.random.default_rng(1).integers(0, 256, size=(10, 100), dtype=np.uint8)
    shards = [d.copy() for d in data] + [np.zeros(100, np.uint8) for _ in range(4)]
    rs.encode(shards)
    assert np.array_equal(np.array(shards[10:]), O.encode8(10, 4, data))
    items, want, keep = _stripes(gpu, O, 8, seed=22)  # built first: the timeout is 0.2 s
    q.start()
    assert q.push(items) == [0] * len(items)
    assert q.finish() == 0
    _check(items, want)


def test_queue_validation_and_capacity(gpu, O):
    import torch

    q = gpu.Queue(max_units=4, timeout_s=1.0)
    rs = gpu.ReedSolomon(4, 2)
    rows = torch.zeros(6 * 100, dtype=torch.uint8, device="cuda")
    with pytest.raises(gpu.RsError):
        q.push([(rs, rows, 100, 100, gpu.ENCODE, None)])  # no session
    q.start()
    st = q.push([(rs, rows, 100, 0, gpu.ENCODE, None), (rs, rows, 50, 100, gpu.ENCODE, None),
                 (rs, rows, 100, 100, gpu.RECONSTRUCT, np.array([1, 0, 0, 0, 1, 1], np.uint8))])
    assert [gpu.ERROR_NAMES[c] for c in st] == ["EmptyShard", "IncorrectShardSize", "TooFewShardsPresent"]
    big = torch.zeros(6 * (1 << 20), dtype=torch.uint8, device="cuda")
    with pytest.raises(gpu.RsError) as e:
        q.push([(rs, big, 1 << 20, 1 << 20, gpu.ENCODE, None)])  # 256 tiles: 16 units > 4
    assert e.value.name == "TooLarge"
    assert q.finish() == 0
