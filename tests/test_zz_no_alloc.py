"""rs8_reconstruct_batch_noalloc: the batched reconstruct for callers that cannot
allocate device memory while they run (a latency-critical path that must not stall on
the allocator, a process whose memory budget was fixed at start-up, a host whose
allocator belongs to another framework). It keeps its working memory in a fixed 8 MiB
device array inside the library, so its results must match the allocating entry point
(rs8_reconstruct_batch_dev) byte for byte, call after call, although every call
reuses what the previous one left in that array.

Named to be collected last: if it fails, a run that stops at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stripes(O, k, m, row_len, n_stripes, seed):
    rng = np.random.default_rng(seed)
    full = np.empty((n_stripes, k + m, row_len), np.uint8)
    present = np.ones((n_stripes, k + m), np.uint8)
    for s in range(n_stripes):
        data = rng.integers(0, 256, size=(k, row_len), dtype=np.uint8)
        full[s] = np.concatenate([data, O.encode8(k, m, data)])
        present[s, rng.choice(k + m, size=int(rng.integers(1, m + 1)), replace=False)] = 0
    present[0, :] = 1  # one stripe with nothing to rebuild
    work = full.copy()
    work[present == 0] = 0
    return full, work, present


def _noalloc(gpu, rs, rows, n_stripes, row_len, present, data_only=False):
    L = gpu.load()
    flags = np.ascontiguousarray(present, np.uint8)
    st = (ctypes.c_int * n_stripes)()
    code = L.rs8_reconstruct_batch_noalloc(
        rs._h, rows.data_ptr(), rows.shape[1] * row_len, n_stripes, row_len,
        flags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), int(data_only), st, 0)
    return code, list(st)


@pytest.mark.parametrize("k,m,row_len,n_stripes", [(32, 32, 4096, 24), (10, 10, 333, 40), (7, 13, 64, 60)])
def test_noalloc_matches_allocating_entry_point(gpu, O, k, m, row_len, n_stripes):
    import torch

    rs = gpu.ReedSolomon(k, m)
    for call in range(2):  # two calls in a row share the same working array
        full, work, present = _stripes(O, k, m, row_len, n_stripes, seed=100 * call + k)
        for data_only in (False, True):
            want = torch.from_numpy(work).cuda()
            ref_status = rs.reconstruct_batch_dev(want, n_stripes, row_len, present, data_only=data_only)
            got = torch.from_numpy(work).cuda()
            code, status = _noalloc(gpu, rs, got, n_stripes, row_len, present, data_only)
            torch.cuda.synchronize()
            assert code == 0
            assert status == ref_status
            assert torch.equal(got, want)
            if not data_only:
                assert np.array_equal(got.cpu().numpy(), full)


def test_noalloc_rejects_requests_beyond_its_working_area(gpu):
    import torch

    L = gpu.load()
    k, m, row_len = 128, 128, 64
    rs = gpu.ReedSolomon(k, m)
    n_stripes = 600  # 600 x (128*128 decode rows + index lists) is about 9.9 MB > 8 MiB
    assert L.rs8_reconstruct_batch_noalloc_limit(k, m, n_stripes) > 8 << 20
    rows = torch.zeros((n_stripes, k + m, row_len), dtype=torch.uint8, device="cuda")
    present = np.ones((n_stripes, k + m), np.uint8)
    present[:, 0] = 0
    code, _ = _noalloc(gpu, rs, rows, n_stripes, row_len, present)
    assert gpu.ERROR_NAMES[code] == "TooLarge"


def test_noalloc_warm_calls_take_no_device_memory(gpu, O):
    """After its first call on the device (which loads its device code and, with it,
    the fixed working array), further calls leave the device's free memory as it was."""
    import torch

    k, m, row_len, n_stripes = 16, 16, 2048, 32
    rs = gpu.ReedSolomon(k, m)
    full, work, present = _stripes(O, k, m, row_len, n_stripes, seed=7)
    rows = torch.from_numpy(work).cuda()
    code, _ = _noalloc(gpu, rs, rows, n_stripes, row_len, present)  # warm-up
    torch.cuda.synchronize()
    assert code == 0
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        rows.copy_(torch.from_numpy(work))
        code, _ = _noalloc(gpu, rs, rows, n_stripes, row_len, present)
        assert code == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    assert np.array_equal(rows.cpu().numpy(), full)


def test_noalloc_refuses_a_capturing_stream(gpu, O):
    """The index lists pass through a host buffer that the next call overwrites, so a
    call made while its stream records a graph is refused instead of recorded."""
    import torch

    k, m, row_len, n_stripes = 10, 10, 512, 4
    rs = gpu.ReedSolomon(k, m)
    _, work, present = _stripes(O, k, m, row_len, n_stripes, seed=9)
    rows = torch.from_numpy(work).cuda()
    torch.cuda.synchronize()
    L = gpu.load()
    flags = np.ascontiguousarray(present, np.uint8)
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        graph.capture_begin()
        code = L.rs8_reconstruct_batch_noalloc(
            rs._h, rows.data_ptr(), (k + m) * row_len, n_stripes, row_len,
            flags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), 0, None, side.cuda_stream)
        graph.capture_end()
    assert gpu.ERROR_NAMES[code] == "InvalidArgument"
    assert torch.equal(rows, torch.from_numpy(work).cuda())
