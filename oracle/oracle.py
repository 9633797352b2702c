"""ctypes binding to the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: a restatement of the reference crate's scalar path used
to check the CUDA library. Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this module; the product package never does.
"""
import ctypes
import hashlib
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u16p = ctypes.POINTER(ctypes.c_uint16)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_szp = ctypes.POINTER(ctypes.c_size_t)
_sz = ctypes.c_size_t

_lib = None


def build():
    """Compile the oracle library with its Makefile (gcc only)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.or_gf8_mul.restype = ctypes.c_uint8
        L.or_gf8_mul.argtypes = [ctypes.c_uint8, ctypes.c_uint8]
        L.or_gf8_exp.restype = ctypes.c_uint8
        L.or_gf8_exp.argtypes = [ctypes.c_uint8, _sz]
        L.or_gf8_div.argtypes = [ctypes.c_uint8, ctypes.c_uint8, _u8p]
        L.or_gf8_tables.argtypes = [_u8p, _u8p]
        L.or_gf16_mul.restype = ctypes.c_uint16
        L.or_gf16_mul.argtypes = [ctypes.c_uint16, ctypes.c_uint16]
        L.or_gf16_inv.restype = ctypes.c_uint16
        L.or_gf16_inv.argtypes = [ctypes.c_uint16]
        L.or_gf16_const_matrix.argtypes = [ctypes.c_uint16, _u8p]
        L.or_invert.argtypes = [ctypes.c_int, _sz, _u16p, _u16p]
        L.or_vandermonde.argtypes = [ctypes.c_int, _sz, _sz, _u16p]
        L.or_matmul.argtypes = [ctypes.c_int, _sz, _sz, _sz, _u16p, _u16p, _u16p]
        L.or_build_matrix.argtypes = [ctypes.c_int, _sz, _sz, _u16p]
        L.or_encode8.argtypes = [_sz, _sz, _u8p, _u8p, _sz]
        L.or_encode16.argtypes = [_sz, _sz, _u8p, _u8p, _sz]
        L.or_reconstruct.argtypes = [ctypes.c_int, _sz, _sz, _u8p, _u8p, _sz, ctypes.c_int]
        L.or_decode_rows.argtypes = [ctypes.c_int, _sz, _sz, _u8p, _u16p, _szp]
        L.or_fft_flat_program.argtypes = [_sz, _sz, _u32p, _sz, _szp, _szp, _u16p, _szp]
        L.or_fft_staged_program.argtypes = [_sz, _sz, _szp, _szp, _szp, _szp, _szp, _szp]
        L.or_fft_flat_run.argtypes = [_sz, _sz, _u8p, _u8p]
        L.or_fft_staged_run.argtypes = [_sz, _sz, _u8p, _u8p]
        L.or_fft_what.argtypes = [_u8p]
        L.or_eval_columns.argtypes = [ctypes.c_int, _sz, _u8p, _sz, _u32p, _sz, _u32p, _sz, _u16p]
        L.or_encode8_batch_mt.restype = ctypes.c_double
        L.or_encode8_batch_mt.argtypes = [_sz, _sz, _u8p, _sz, _sz, ctypes.c_int]
        _lib = L
    return _lib


def _p8(a):
    return a.ctypes.data_as(_u8p)


def _p16(a):
    return a.ctypes.data_as(_u16p)


def gf8_mul(a, b):
    return lib().or_gf8_mul(a, b)


def gf8_exp(a, n):
    return lib().or_gf8_exp(a, n)


def gf8_div(a, b):
    out = ctypes.c_uint8(0)
    if lib().or_gf8_div(a, b, ctypes.byref(out)) != 0:
        raise ZeroDivisionError("Divisor is 0")
    return out.value


def gf8_tables():
    log = np.zeros(256, np.uint8)
    exp = np.zeros(510, np.uint8)
    lib().or_gf8_tables(_p8(log), _p8(exp))
    return log, exp


def gf8_mul_table():
    log, exp = gf8_tables()
    a = np.arange(256)
    t = exp[(log[a][:, None].astype(np.int32) + log[a][None, :].astype(np.int32))]
    t[0, :] = 0
    t[:, 0] = 0
    return t.astype(np.uint8)


def gf16_mul(a, b):
    return lib().or_gf16_mul(a, b)


def gf16_inv(a):
    return lib().or_gf16_inv(a)


def gf16_const_matrix(c):
    out = np.zeros(4, np.uint8)
    lib().or_gf16_const_matrix(c, _p8(out))
    return [int(v) for v in out]


def build_matrix(field, k, n):
    out = np.zeros(n * k, np.uint16)
    st = lib().or_build_matrix(field, k, n, _p16(out))
    if st:
        raise RuntimeError("build_matrix status %d" % st)
    return out.reshape(n, k)


def invert(field, mat):
    mat = np.ascontiguousarray(mat, dtype=np.uint16)
    n = mat.shape[0]
    out = np.zeros_like(mat)
    st = lib().or_invert(field, n, _p16(mat), _p16(out))
    return st, out


def vandermonde(field, rows, cols):
    out = np.zeros(rows * cols, np.uint16)
    lib().or_vandermonde(field, rows, cols, _p16(out))
    return out.reshape(rows, cols)


def matmul(field, a, b):
    a = np.ascontiguousarray(a, dtype=np.uint16)
    b = np.ascontiguousarray(b, dtype=np.uint16)
    out = np.zeros((a.shape[0], b.shape[1]), np.uint16)
    lib().or_matmul(field, a.shape[0], a.shape[1], b.shape[1], _p16(a), _p16(b), _p16(out))
    return out


def encode8(k, m, data):
    """data: (k, len) uint8 -> parity (m, len), src/reedsolomon.rs:402-424."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    par = np.zeros((m, data.shape[1]), np.uint8)
    st = lib().or_encode8(k, m, _p8(data), _p8(par), data.shape[1])
    if st:
        raise RuntimeError("encode8 status %d" % st)
    return par


def encode16(k, m, data):
    """data: (k, len) uint8 split-plane shards -> parity (m, len)."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    par = np.zeros((m, data.shape[1]), np.uint8)
    st = lib().or_encode16(k, m, _p8(data), _p8(par), data.shape[1])
    if st:
        raise RuntimeError("encode16 status %d" % st)
    return par


def reconstruct(field, k, m, rows, present, data_only=False):
    """rows: (k+m, len) uint8, rebuilt in place; returns the status code."""
    assert rows.flags["C_CONTIGUOUS"] and rows.dtype == np.uint8
    pres = np.ascontiguousarray(np.asarray(present, dtype=np.uint8))
    return lib().or_reconstruct(field, k, m, _p8(rows), _p8(pres), rows.shape[1], int(data_only))


def decode_rows(field, k, m, present):
    pres = np.ascontiguousarray(np.asarray(present, dtype=np.uint8))
    out = np.zeros((k + m) * k, np.uint16)
    n = ctypes.c_size_t(0)
    st = lib().or_decode_rows(field, k, m, _p8(pres), _p16(out), ctypes.byref(n))
    return st, out[: n.value * k].reshape(n.value, k)


def eval_columns(field, k, data, cols, points):
    """Shard values of the encoded stripe at the given evaluation points (shard
    indexes) and symbol columns, by barycentric Lagrange evaluation (O(k) per point and
    column; eval_columns.c). data: (k, len) uint8, split-plane for field 16. Returns
    (len(points), len(cols)) uint16 symbols."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    cols = np.ascontiguousarray(np.asarray(cols, dtype=np.uint32))
    points = np.ascontiguousarray(np.asarray(points, dtype=np.uint32))
    out = np.zeros((len(points), len(cols)), np.uint16)
    st = lib().or_eval_columns(field, k, _p8(data), data.shape[1], cols.ctypes.data_as(_u32p), len(cols),
                               points.ctypes.data_as(_u32p), len(points), _p16(out))
    if st:
        raise RuntimeError("eval_columns status %d" % st)
    return out


def symbols(field, shards, cols):
    """The symbols of (rows, len) shards at the given symbol columns, as uint16:
    GF(2^8) bytes, or tower symbols (high << 8) | low from the split-plane wire."""
    shards = np.asarray(shards, dtype=np.uint8)
    cols = np.asarray(cols, dtype=np.int64)
    if field == 8:
        return shards[:, cols].astype(np.uint16)
    half = shards.shape[1] // 2
    return (shards[:, half + cols].astype(np.uint16) << 8) | shards[:, cols]


_KIND = {0: "mx", 1: "xo", 2: "mc", 3: "cp"}


def fft_flat_program(k, m):
    """(ops, register_count, parity_regs, mult_count); ops as (kind, dst, src, c)."""
    cap = 1 << 16
    buf = np.zeros(cap, np.uint32)
    n_ops, regs, mults = ctypes.c_size_t(0), ctypes.c_size_t(0), ctypes.c_size_t(0)
    par = np.zeros(max(m, 1), np.uint16)
    st = lib().or_fft_flat_program(
        k, m, buf.ctypes.data_as(_u32p), cap, ctypes.byref(n_ops), ctypes.byref(regs),
        _p16(par), ctypes.byref(mults))
    if st:
        raise RuntimeError("fft program build failed")
    ops = [(int(v >> 28), int((v >> 18) & 0x3FF), int((v >> 8) & 0x3FF), int(v & 0xFF))
           for v in buf[: n_ops.value]]
    return ops, regs.value, [int(p) for p in par[:m]], mults.value


def fft_program_text(k, m):
    """The program in the reference's generated-list token form (ld/mx/xo/mc/cp/st)."""
    ops, _, par, _ = fft_flat_program(k, m)
    lines = ["ld %d %d" % (i, i) for i in range(k)]
    for kind, dst, src, c in ops:
        name = _KIND[kind]
        lines.append("%s %d %d %d" % (name, dst, src, c) if kind in (0, 2) else "%s %d %d" % (name, dst, src))
    lines += ["st %d %d" % (j, r) for j, r in enumerate(par)]
    return lines


def fft_program_digest(k, m):
    return hashlib.sha256("\n".join(fft_program_text(k, m)).encode()).hexdigest()


def fft_staged_stats(k, m):
    vals = [ctypes.c_size_t(0) for _ in range(6)]
    st = lib().or_fft_staged_program(k, m, *[ctypes.byref(v) for v in vals])
    if st:
        raise RuntimeError("staged build failed")
    keys = ["register_count", "mult_count", "xor_count", "stages", "glue", "zero_regs"]
    return {key: v.value for key, v in zip(keys, vals)}


def fft_flat_run(k, m, column):
    col = np.ascontiguousarray(np.asarray(column, dtype=np.uint8))
    par = np.zeros(m, np.uint8)
    lib().or_fft_flat_run(k, m, _p8(col), _p8(par))
    return par


def fft_staged_run(k, m, column):
    col = np.ascontiguousarray(np.asarray(column, dtype=np.uint8))
    par = np.zeros(m, np.uint8)
    lib().or_fft_staged_run(k, m, _p8(col), _p8(par))
    return par


def fft_what():
    out = np.zeros(8 * 256, np.uint8)
    lib().or_fft_what(_p8(out))
    return out.reshape(8, 256)


def encode8_batch_mt(k, m, stripes, threads):
    """stripes: (S, k+m, len) uint8, parity rows written; returns seconds."""
    assert stripes.flags["C_CONTIGUOUS"] and stripes.dtype == np.uint8
    return lib().or_encode8_batch_mt(k, m, _p8(stripes), stripes.shape[0], stripes.shape[2], threads)


def encode8_repeat(k, m, stripe, reps):
    """stripe: (k+m, len) uint8; one thread encodes it reps times (after one untimed
    pass); returns seconds for the reps."""
    assert stripe.flags["C_CONTIGUOUS"] and stripe.dtype == np.uint8
    L = lib()
    L.or_encode8_repeat.restype = ctypes.c_double
    L.or_encode8_repeat.argtypes = [_sz, _sz, _u8p, _sz, _sz]
    return L.or_encode8_repeat(k, m, _p8(stripe), stripe.shape[1], reps)


def cpu_has_gfni():
    return bool(lib().or_cpu_has_gfni())


_PATHS = {2: "straight-line GFNI/AVX-512 (generated)", 1: "GFNI/AVX-512 program replay", 0: "scalar"}


def cpu_path(k, m, length):
    """Which CPU encoder encode8_batch_mt runs for (k, m) at this shard length."""
    L = lib()
    L.or_cpu_path.argtypes = [_sz, _sz, _sz]
    return _PATHS[L.or_cpu_path(k, m, length)]
