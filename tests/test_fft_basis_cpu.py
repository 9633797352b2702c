"""The bitsliced FFT encode's subspace bases (fftc::fft_basis in kernels_fft.cuh).

The device kernel evaluates the encode polynomial with the additive FFT over a searched
ordered basis of {0..K-1} and a searched representative beta of the parity coset instead
of the reference's powers of two and beta = K (src/fft.rs). These CPU tests check that
(1) the compiled table is what fft_basis_search.c finds, and (2) the transform pair over
each tabled basis, with the kernel's register-to-shard mapping and its C+1 form of the
forward butterfly, reproduces the oracle's parity bytes.
"""
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "reed-solomon_b200", "csrc")


def compiled_table():
    """(K, W) -> (basis vectors, beta) as written in fft_basis()."""
    src = open(os.path.join(CSRC, "kernels_fft.cuh")).read()
    body = src[src.index("constexpr FftBasis fft_basis(int K, int W)"):]
    body = body[:body.index("\n}\n")]
    vec = r"\{\{([\d, ]+)\}, (\d+)\}"
    out = {}

    def put(K, W, v, beta):
        n = K.bit_length() - 1
        vs = [int(x) for x in v.split(",")]
        out[(K, W)] = (vs[:n], int(beta))

    for K, v, beta in re.findall(r"case (\d+): return " + vec + ";", body):
        put(int(K), 1, v, beta)
    pat = r"W == (\d) \? FftBasis" + vec + r" : FftBasis" + vec + ";"
    for K, W, v1, b1, v2, b2 in re.findall(r"case (\d+): return " + pat, body):
        put(int(K), int(W), v1, b1)
        put(int(K), int(W) + 1, v2, b2)
    for W, v1, b1, v2, b2 in re.findall(r"default: return " + pat, body):
        put(128, int(W), v1, b1)
        put(128, int(W) + 1, v2, b2)
    return out


def test_compiled_bases_are_the_search_output():
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "fft_basis_search")
        subprocess.run([gcc, "-O2", "-o", exe, os.path.join(CSRC, "fft_basis_search.c")], check=True)
        text = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    found = {}
    for K, W, std, best, v, beta in re.findall(
            r"K=\s*(\d+) W=(\d) standard=\s*(\d+) best=\s*(\d+)\s+\{\{([\d, ]+)\}, (\d+)\}", text):
        K, W = int(K), int(W)
        n = K.bit_length() - 1
        assert int(best) <= int(std)
        found[(K, W)] = ([int(x) for x in v.split(",")][:n], int(beta))
    table = compiled_table()
    assert set(found) == set(table)
    for key in found:
        assert table[key] == found[key], key


def _mul_cost(MT, c):
    """Three-input XORs of d ^= c*s in the kernel's XOR networks."""
    if c <= 1:
        return 8 * c
    n = 0
    for b in range(8):
        nb = sum((int(MT[c, 1 << p]) >> b) & 1 for p in range(8))
        n += (nb + 1) // 2
    return n


def encode_over_basis(O, MT, K, v, beta, data):
    n = K.bit_length() - 1
    inv = {a: next(c for c in range(1, 256) if MT[a, c] == 1) for a in range(1, 256)}
    raw = [list(range(256))]
    for j in range(n - 1):
        piv = raw[j][v[j]]
        raw.append([int(MT[raw[j][x], raw[j][x] ^ piv]) for x in range(256)])
    W = [[int(MT[raw[j][x], inv[raw[j][v[j]]]]) for x in range(256)] for j in range(n)]
    P = [0] * K
    for i in range(K):
        for j in range(n):
            if (i >> j) & 1:
                P[i] ^= v[j]
    regs = [data[P[i]].copy() for i in range(K)]  # register i holds data point P(i)
    for lev in range(n):  # inverse transform on V
        h = 1 << lev
        for base in range(0, K, 2 * h):
            c = W[lev][P[base]]
            for i in range(base, base + h):
                lo, hi = regs[i], regs[i + h]
                hi = hi ^ lo
                lo = lo ^ MT[c][hi]
                regs[i], regs[i + h] = lo, hi
    for lev in reversed(range(n)):  # forward transform on the coset beta + V
        h = 1 << lev
        for base in range(0, K, 2 * h):
            c = W[lev][beta ^ P[base]]
            flip = c != 0 and _mul_cost(MT, c ^ 1) < _mul_cost(MT, c)
            for i in range(base, base + h):
                lo, hi = regs[i], regs[i + h]
                if flip:
                    hi2 = lo ^ MT[c ^ 1][hi]
                    lo2 = hi2 ^ hi
                else:
                    lo2 = lo ^ MT[c][hi]
                    hi2 = hi ^ lo2
                regs[i], regs[i + h] = lo2, hi2
    parity = np.zeros_like(data)
    for i in range(K):
        parity[(beta ^ P[i]) - K] = regs[i]  # register i holds parity point beta ^ P(i)
    return parity


def test_searched_bases_give_the_oracle_parity(O):
    MT = np.asarray(O.gf8_mul_table(), dtype=np.uint8).reshape(256, 256)
    rng = np.random.default_rng(17)
    for (K, W), (v, beta) in sorted(compiled_table().items()):
        data = rng.integers(0, 256, size=(K, 48), dtype=np.uint8)
        got = encode_over_basis(O, MT, K, v, beta, data)
        assert np.array_equal(got, O.encode8(K, K, data)), (K, W, v, beta)
