"""The C ABI library without a GPU: it loads, exports every declared symbol, maps the
reference's errors, and its host-side construction matches the oracle.

The host construction (closed-form Lagrange rows) must equal the reference's
vandermonde * inverse(top) generator (src/reedsolomon.rs:155-159) and its decode rows
(src/reedsolomon.rs:539-585 plus the parity rows applied to the recovered data,
:877-889) exactly; the oracle restates those.
"""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "rs_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(\w+)\s*\([^;{]*\)\s*;", text)))


def test_library_exports_every_declared_symbol(rsb):
    names = declared_symbols()
    assert len(names) > 50
    lib = ctypes.CDLL(rsb.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the binding declares each one
    from reed_solomon_b200 import _lib

    assert sorted(_lib.SIGNATURES) == names


def test_error_messages_match_reference(rsb, golden):
    L = rsb.load()
    for code, (name, msg) in enumerate(zip(golden["error_variants"], golden["error_messages"]), start=1):
        assert rsb.ERROR_NAMES[code] == name
        assert L.rs_strerror(code).decode() == msg


def test_new_argument_errors_without_device(rsb):
    # src/reedsolomon.rs:166-176: these checks precede any device work.
    for k, m, name in [(0, 1, "TooFewDataShards"), (1, 0, "TooFewParityShards"),
                       (200, 57, "TooManyShards")]:
        with pytest.raises(rsb.RsError) as e:
            rsb.ReedSolomon(k, m)
        assert e.value.name == name
    with pytest.raises(rsb.RsError) as e:
        rsb.ReedSolomon16(40000, 30000)
    assert e.value.name == "TooManyShards"


def _gen_rows(rsb, field, k, m):
    out = np.zeros(k * m, np.uint16)
    st = rsb.load().rs_generator_rows(field, k, m, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), out.size)
    assert st == 0
    return out.reshape(m, k)


GF8_SHAPES = [(1, 1), (2, 2), (3, 5), (4, 2), (7, 13), (10, 10), (14, 14), (16, 16), (18, 6),
              (20, 12), (32, 32), (1, 255), (255, 1), (64, 64), (128, 128), (17, 200)]


@pytest.mark.parametrize("k,m", GF8_SHAPES)
def test_generator_rows_match_oracle_gf8(rsb, O, k, m):
    want = O.build_matrix(8, k, k + m)
    assert np.array_equal(want[:k], np.eye(k, dtype=np.uint16))
    assert np.array_equal(_gen_rows(rsb, 8, k, m), want[k:])


@pytest.mark.parametrize("k,m", [(3, 2), (4, 2), (17, 33), (86, 170), (100, 200)])
def test_generator_rows_match_oracle_gf16(rsb, O, k, m):
    want = O.build_matrix(16, k, k + m)
    assert np.array_equal(_gen_rows(rsb, 16, k, m), want[k:])


def _decode_rows(rsb, field, k, m, present):
    p = np.ascontiguousarray(np.asarray(present, np.uint8))
    out = np.zeros((k + m) * k, np.uint16)
    n = ctypes.c_size_t(0)
    st = rsb.load().rs_decode_rows(field, k, m, p.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), out.size,
                                   ctypes.byref(n))
    return st, out[: n.value * k].reshape(n.value, k)


@pytest.mark.parametrize("field,k,m", [(8, 4, 2), (8, 7, 13), (8, 10, 10), (8, 32, 32), (8, 20, 12),
                                       (16, 17, 33), (16, 10, 10)])
def test_decode_rows_match_oracle(rsb, O, field, k, m):
    rng = np.random.default_rng(k * 7 + m + field)
    gen = O.build_matrix(field, k, k + m)
    for _ in range(6):
        e = int(rng.integers(1, m + 1))
        present = np.ones(k + m, np.uint8)
        present[rng.choice(k + m, size=e, replace=False)] = 0
        st, rows = _decode_rows(rsb, field, k, m, present)
        assert st == 0
        st2, data_rows = O.decode_rows(field, k, m, present)
        assert st2 == 0
        nd = data_rows.shape[0]
        assert np.array_equal(rows[:nd], data_rows)
        # Missing parity rows: generator row times the inverse (the reference applies
        # the generator row to the recovered data).
        surv = [i for i in range(k + m) if present[i]][:k]
        _, inv = O.invert(field, gen[surv])
        missing_parity = [i for i in range(k, k + m) if not present[i]]
        for t, p in enumerate(missing_parity):
            want = O.matmul(field, gen[p:p + 1], inv)[0]
            assert np.array_equal(rows[nd + t], want)


def test_decode_rows_too_few_present(rsb):
    st, _ = _decode_rows(rsb, 8, 4, 2, [1, 1, 1, 0, 0, 0])
    assert st == 10


def test_fft_tuning_hooks_and_automatic_choice(rsb):
    """rs_set_fft_variant / rs_set_fft_lanes return the previous value, reject shapes
    without an FFT kernel (generator shapes included) and out-of-range values, and -1
    restores the automatic choice (host state only, no device needed)."""
    L = rsb.load()
    n = L.rs_fft_variant_count()
    assert n >= 4
    base = L.rs_set_fft_variant(32, 2)
    assert 0 <= base < n
    assert L.rs_set_fft_variant(32, 1) == 2
    assert L.rs_set_fft_variant(32, -1) == 1
    assert L.rs_set_fft_variant(32, -1) == base  # back to the tuned default
    assert L.rs_set_fft_variant(32, n) == -1
    assert L.rs_set_fft_variant(32, -2) == -1
    assert L.rs_set_fft_variant(10, 0) == -1  # (10,10) is a generator shape
    assert L.rs_set_fft_variant(24, 0) == -1  # no compiled kernel
    wide = L.rs_set_fft_lanes(128, 0)
    assert wide in (0, 1)
    assert L.rs_set_fft_lanes(128, -1) == 0
    assert L.rs_set_fft_lanes(128, -1) == wide
    assert L.rs_set_fft_lanes(128, 2) == -1
    assert L.rs_set_fft_lanes(14, 0) == -1
    # Host-pointer staging switches (host state only).
    t = L.rs_set_host_copy_threads(4)
    assert t >= 1
    assert L.rs_set_host_copy_threads(0) == 4  # out of range: unchanged
    assert L.rs_set_host_copy_threads(t) == 4
    on = L.rs_set_host_staging(0)
    assert on == 1
    assert L.rs_set_host_staging(1) == 0


def test_tuning_configurations_match_the_tuner(rsb):
    """The library's configuration table (the cost model's output order) is the one the
    Python tuner times, and the model reads the six features it computes."""
    from reed_solomon_b200 import tuner

    assert tuner.library_configs() == tuner.CONFIGS
    assert rsb.load().rs_tuning_features() == tuner.N_FEATURES


def test_shipped_cost_model_file(rsb):
    """cost_model.rsmlp: the magic, then 6 inputs, 64 hidden, 13 outputs, then exactly
    the network's float32 parameters, all finite."""
    import struct

    import numpy as np

    from reed_solomon_b200 import tuner

    blob = open(tuner.MODEL_PATH, "rb").read()
    assert blob[:8] == b"RSMLP\x00\x00\x01"
    n_in, hidden, n_out = struct.unpack("<3i", blob[8:20])
    assert (n_in, hidden, n_out) == (tuner.N_FEATURES, 64, len(tuner.CONFIGS))
    n_params = n_in * hidden + hidden + 2 * (hidden * hidden + hidden) + hidden * n_out + n_out
    params = np.frombuffer(blob[20:], dtype="<f4")
    assert params.size == n_params and np.all(np.isfinite(params))


def test_mlp_load_rejects_other_files(rsb, tmp_path):
    import ctypes

    bad = tmp_path / "not_a_model.bin"
    bad.write_bytes(b"RSMLP\x00\x00\x02" + b"\x00" * 64)
    h = ctypes.c_void_p()
    assert rsb.load().rs_mlp_load(str(bad).encode(), ctypes.byref(h)) == 102
    assert rsb.load().rs_mlp_load(str(tmp_path / "missing").encode(), ctypes.byref(h)) == 102
