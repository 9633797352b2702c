"""The bitsliced matrix kernel (gf8_bits_kernel: warp-uniform coefficients selecting
compiled XOR networks) against the oracle, in both of its forms and against the SWAR
kernel, on the strided calls it serves: matrix-route batched encode and batched
reconstruct (per-stripe decode rows and row maps), with aligned and unaligned lengths,
partial last groups and stripes too short for one group."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4])
def test_matrix_kernels_match_the_oracle(gpu, O, mode):
    import torch

    L = gpu.load()
    old = L.rs_set_matrix_bits(mode)
    try:
        for k, m, S, N in [(32, 32, 4096, 6), (10, 10, 1000, 5), (20, 30, 77, 7), (3, 5, 5, 3), (64, 64, 4133, 4)]:
            n = k + m
            rs = gpu.ReedSolomon(k, m)
            rs.set_route("matrix")
            rng = np.random.default_rng(k * 100 + S + mode)
            data = rng.integers(0, 256, size=(N, n, S), dtype=np.uint8)
            rows = torch.from_numpy(data).cuda()
            rs.encode_batch_dev(rows, rows[:, k:], S, N, data_stride=n * S, parity_stride=n * S)
            torch.cuda.synchronize()
            got = rows.cpu().numpy()
            for s in range(N):
                assert np.array_equal(got[s, k:], O.encode8(k, m, got[s, :k])), (k, m, S, s)
            full = rows.clone()
            present = np.ones((N, n), np.uint8)
            for s in range(N):
                present[s, rng.choice(n, size=int(rng.integers(1, m + 1)), replace=False)] = 0
            rows[torch.from_numpy(present == 0).cuda()] = 0
            st = rs.reconstruct_batch_dev(rows, N, S, present)
            torch.cuda.synchronize()
            assert st == [0] * N
            assert torch.equal(rows, full), (k, m, S)
    finally:
        L.rs_set_matrix_bits(old)


@pytest.mark.parametrize("mode", [0, 2, 3, 4])
def test_ragged_batches_match_the_oracle(gpu, O, mode):
    """Mixed batches put matrix-route encodes and every reconstruct's rows on one ragged
    launch: under the SWAR (0) and the bitsliced (2) ragged kernels the stripes match the
    oracle, at packed (unaligned) and aligned row strides."""
    import torch

    L = gpu.load()
    old = L.rs_set_matrix_bits(mode)
    try:
        rng = np.random.default_rng(60 + mode)
        shapes = [(20, 30), (5, 3), (32, 32), (100, 60)]
        codecs = {sh: gpu.ReedSolomon(*sh) for sh in shapes}
        items, keep, want = [], [], []
        for i in range(24):
            k, m = shapes[i % len(shapes)]
            S = int(rng.integers(1, 6000))
            stride = S if i % 2 else (S + 15) // 16 * 16
            data = rng.integers(0, 256, size=(k, S), dtype=np.uint8)
            full = np.zeros((k + m, stride), np.uint8)
            full[:k, :S] = data
            full[k:, :S] = O.encode8(k, m, data)
            work = full.copy()
            if i % 3 == 0:
                present = np.ones(k + m, np.uint8)
                present[rng.choice(k + m, size=int(rng.integers(1, m + 1)), replace=False)] = 0
                work[present == 0] = 0
                op = gpu.RECONSTRUCT
            else:
                present = None
                work[k:] = 0
                op = gpu.ENCODE
            rows = torch.from_numpy(work.reshape(-1)).cuda()
            keep.append(rows)
            items.append((codecs[(k, m)], rows, stride, S, op, present))
            want.append((full, S, stride))
        b = gpu.Batch(items, flags=gpu.MATRIX_ONLY)
        assert b.statuses == [0] * len(items)
        b.launch()
        torch.cuda.synchronize()
        for rows, (full, S, stride) in zip(keep, want):
            got = rows.cpu().numpy().reshape(full.shape[0], stride)
            assert np.array_equal(got[:, :S], full[:, :S])
    finally:
        L.rs_set_matrix_bits(old)
