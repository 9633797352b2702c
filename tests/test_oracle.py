"""The CPU oracle against the reference's own golden vectors and known answers.

These pin the oracle before any GPU result is compared with it:
* src/galois.rs:119-163   Backblaze log table, known products, field axioms
* src/galois16.rs:143-233 tower constant, const_matrix, inverses
* src/reedsolomon16.rs:1087-1101 frozen wire vector
* src/fft_programs.rs     the reference's generated programs: digests, counts, outputs
* src/fft.rs:890-1103     FFT/IFFT shape tests, programs == matrix encode, op counts
* src/matrix.rs:205-236   Vandermonde inverse, singular matrix
"""
import numpy as np
import pytest


def test_log_table_same_as_backblaze(O, golden):
    log, _ = O.gf8_tables()
    assert list(log) == golden["backblaze_log_table"]


def test_known_products(O, golden):
    assert golden["known_mul"] and golden["known_exp"]
    for a, b, c in golden["known_mul"]:
        assert O.gf8_mul(a, b) == c
    for a, n, c in golden["known_exp"]:
        assert O.gf8_exp(a, n) == c


def test_field_axioms(O):
    t = O.gf8_mul_table()
    assert np.array_equal(t, t.T)
    for a in range(1, 256):
        assert O.gf8_mul(a, O.gf8_div(1, a)) == 1
    with pytest.raises(ZeroDivisionError):
        O.gf8_div(3, 0)


def _trace(O, x):
    acc = 0
    for _ in range(8):
        acc ^= x
        x = O.gf8_mul(x, x)
    return acc


def test_tower_constant_smallest_trace_one(O, golden):
    L = golden["gf16_tower_l"]
    assert all(_trace(O, c) == 0 for c in range(L))
    assert _trace(O, L) == 1
    assert sum(_trace(O, c) for c in range(256)) == 128


def test_const_matrix(O, golden):
    for c, want in golden["gf16_const_matrix"]:
        assert O.gf16_const_matrix(c) == want
    rng = np.random.default_rng(5)
    for c in list(range(0, 65536, 97)) + [0xFFFF, 0x0100, 32]:
        m = O.gf16_const_matrix(c)
        for a in rng.integers(0, 65536, size=6).tolist() + [0, 1, 0xFFFF]:
            ah, al = a >> 8, a & 0xFF
            hi = O.gf8_mul(m[0], ah) ^ O.gf8_mul(m[1], al)
            lo = O.gf8_mul(m[2], ah) ^ O.gf8_mul(m[3], al)
            assert (hi << 8 | lo) == O.gf16_mul(c, a)


def test_gf16_all_inverses(O):
    for a in range(1, 65536):
        assert O.gf16_mul(a, O.gf16_inv(a)) == 1


def test_gf16_wire_vector(O, golden):
    g = golden["gf16_wire_vector"]
    data = np.array(g["data"], np.uint8)
    assert O.encode16(g["k"], g["m"], data).tolist() == g["parity"]


@pytest.mark.parametrize("idx", range(6))
def test_fft_programs_match_reference(O, golden, idx):
    p = golden["fft_programs"][idx]
    k, m = p["k"], p["m"]
    ops, regs, _, mults = O.fft_flat_program(k, m)
    assert regs == p["registers"]
    assert len(ops) == p["ops_body"] == p["ops_header"]
    assert mults == p["multiplies"]
    assert O.fft_program_digest(k, m) == p["sha256"]
    cols = np.array(p["columns"], np.uint8)
    for col, want in zip(cols, p["parity"]):
        assert O.fft_flat_run(k, m, col).tolist() == want
        assert O.fft_staged_run(k, m, col).tolist() == want
    # The matrix encode equals the reference programs' outputs.
    assert O.encode8(k, m, cols.T.copy()).T.tolist() == p["parity"]


def test_what_tables(O):
    what = O.fft_what().astype(np.int64)
    for level in range(8):
        assert (what[level, : 1 << level] == 0).all()
        assert what[level, 1 << level] == 1
        for a in range(256):
            assert what[level, a ^ 0x5A] == what[level, a] ^ what[level, 0x5A]


# src/fft.rs:963-985 shape list
SHAPES = [(1, 1), (1, 4), (2, 2), (3, 5), (4, 2), (5, 3), (6, 4), (7, 13), (9, 3), (10, 10),
          (10, 7), (11, 5), (13, 7), (14, 14), (16, 4), (17, 17), (18, 6), (20, 10), (24, 8),
          (32, 32), (37, 21)]


@pytest.mark.parametrize("k,m", SHAPES)
def test_programs_match_matrix(O, k, m):
    rng = np.random.default_rng(k * 131 + m)
    data = rng.integers(0, 256, size=(k, 64), dtype=np.uint8)
    want = O.encode8(k, m, data)
    for b in range(64):
        assert O.fft_flat_run(k, m, data[:, b]).tolist() == want[:, b].tolist()
        assert O.fft_staged_run(k, m, data[:, b]).tolist() == want[:, b].tolist()


def test_program_op_counts(O):
    for k, m in [(7, 13), (10, 10), (14, 14), (16, 16), (18, 6)]:
        _, _, _, mults = O.fft_flat_program(k, m)
        assert mults < k * m
        assert O.fft_staged_stats(k, m)["mult_count"] < k * m


@pytest.mark.parametrize("field,size", [(8, 20), (16, 86)])
def test_vandermonde_inverse_is_identity(O, field, size):
    v = O.vandermonde(field, size, size)
    st, inv = O.invert(field, v)
    assert st == 0
    assert np.array_equal(O.matmul(field, v, inv), np.eye(size, dtype=np.uint16))


def test_singular_matrix_errors(O):
    st, _ = O.invert(16, np.ones((2, 2), np.uint16))
    assert st == 14


@pytest.mark.parametrize("field", [8, 16])
def test_oracle_reconstruct_round_trip(O, field):
    rng = np.random.default_rng(field)
    for k, m in [(4, 2), (7, 13), (10, 10)]:
        length = 64
        data = rng.integers(0, 256, size=(k, length), dtype=np.uint8)
        par = O.encode8(k, m, data) if field == 8 else O.encode16(k, m, data)
        full = np.concatenate([data, par])
        for e in range(1, m + 1):
            erased = rng.choice(k + m, size=e, replace=False)
            rows = full.copy()
            rows[erased] = 0
            present = np.ones(k + m, np.uint8)
            present[erased] = 0
            assert O.reconstruct(field, k, m, rows, present) == 0
            assert np.array_equal(rows, full)


def test_tower_subfield_shapes_equal_gf8_code(O):
    """With k + m <= 256 every evaluation point of the tower code has a zero high byte,
    so its generator and decode coefficients lie in GF(2^8), which scales the low and
    the high byte plane alike: the tower code is ReedSolomon(k, m) on the shard bytes.
    The library's automatic tower route relies on this; the oracle shows it on encode,
    the parity matrices and reconstruct. Past 256 shards it no longer holds."""
    rng = np.random.default_rng(256)
    for k, m in [(1, 1), (2, 1), (7, 13), (32, 32), (100, 156), (3, 250), (255, 1)]:
        assert np.array_equal(O.build_matrix(16, k, k + m), O.build_matrix(8, k, k + m).astype(np.uint16))
        data = rng.integers(0, 256, size=(k, 66), dtype=np.uint8)
        par = O.encode16(k, m, data)
        assert np.array_equal(par, O.encode8(k, m, data)), (k, m)
        full = np.concatenate([data, par])
        erased = rng.choice(k + m, size=m, replace=False)
        present = np.ones(k + m, np.uint8)
        present[erased] = 0
        rows8, rows16 = full.copy(), full.copy()
        rows8[erased] = 0
        rows16[erased] = 0
        assert O.reconstruct(8, k, m, rows8, present) == 0
        assert O.reconstruct(16, k, m, rows16, present) == 0
        assert np.array_equal(rows8, full) and np.array_equal(rows16, full)
    assert (O.build_matrix(16, 200, 300)[200:] >> 8).any()  # points >= 256: tower coefficients


@pytest.mark.parametrize("field,k,m,length", [
    (8, 1, 1, 5), (8, 10, 10, 100), (8, 32, 32, 64), (8, 7, 13, 33), (8, 128, 128, 40), (8, 3, 253, 9),
    (16, 2, 1, 2), (16, 4, 2, 30), (16, 17, 33, 66), (16, 100, 200, 20), (16, 300, 20, 6)])
def test_column_evaluator_matches_gauss_jordan_oracle(O, field, k, m, length):
    """The barycentric column evaluator (used to check shapes too large for the O(k^3)
    generator) gives every shard of the stripe the Gauss-Jordan oracle encodes."""
    rng = np.random.default_rng(k * 1000 + m + field)
    data = rng.integers(0, 256, size=(k, length), dtype=np.uint8)
    parity = (O.encode8 if field == 8 else O.encode16)(k, m, data)
    n_sym = length if field == 8 else length // 2
    got = O.eval_columns(field, k, data, range(n_sym), range(k + m))
    assert np.array_equal(got, O.symbols(field, np.concatenate([data, parity]), range(n_sym)))


@pytest.mark.parametrize("k,m", [(7, 13), (10, 10), (14, 14), (16, 16), (18, 6), (32, 32), (20, 12), (4, 2)])
def test_timed_cpu_encoder_matches_oracle(O, k, m):
    """The multi-threaded CPU encoder timed as the baseline (straight-line GFNI code for
    the six generated shapes, program replay or scalar otherwise) writes the oracle's
    parity, for lengths below, at and between strips, with the overlapped last strip."""
    rng = np.random.default_rng(k * 100 + m)
    for length in (1, 31, 63, 64, 65, 127, 255, 256, 257, 1000, 4096 + 17):
        stripes = rng.integers(0, 256, size=(3, k + m, length), dtype=np.uint8)
        O.encode8_batch_mt(k, m, stripes, 2)
        for s in range(3):
            assert np.array_equal(stripes[s, k:], O.encode8(k, m, stripes[s, :k])), (length, s)
        one = rng.integers(0, 256, size=(k + m, length), dtype=np.uint8)
        O.encode8_repeat(k, m, one, 2)
        assert np.array_equal(one[k:], O.encode8(k, m, one[:k])), length


def test_timed_cpu_encoder_takes_straight_line_code_on_gfni_hosts(O):
    if not O.cpu_has_gfni():
        pytest.skip("host without GFNI/AVX-512: the scalar path is timed")
    assert O.cpu_path(32, 32, 1 << 20).startswith("straight-line")
    assert O.cpu_path(20, 12, 1 << 20) == "GFNI/AVX-512 program replay"
