/*
 * CPU oracle for the tape-reed-solomon encode/reconstruct path.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates the reference crate's scalar
 * Galois path in plain C so that tests can check the CUDA library byte for byte.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it; the product library never links or calls it.
 *
 * Every function names the reference file:line it follows (paths are relative to
 * the reference crate root, spool-labs/reed-solomon 0.2.2).
 *
 * Status codes follow the reference `Error` enum order (src/errors.rs:7-20),
 * 1-based, 0 = Ok.
 */
#ifndef RS_ORACLE_H
#define RS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  OR_OK = 0,
  OR_TOO_FEW_SHARDS = 1,
  OR_TOO_MANY_SHARDS = 2,
  OR_TOO_FEW_DATA_SHARDS = 3,
  OR_TOO_MANY_DATA_SHARDS = 4,
  OR_TOO_FEW_PARITY_SHARDS = 5,
  OR_TOO_MANY_PARITY_SHARDS = 6,
  OR_TOO_FEW_BUFFER_SHARDS = 7,
  OR_TOO_MANY_BUFFER_SHARDS = 8,
  OR_INCORRECT_SHARD_SIZE = 9,
  OR_TOO_FEW_SHARDS_PRESENT = 10,
  OR_EMPTY_SHARD = 11,
  OR_INVALID_SHARD_FLAGS = 12,
  OR_INVALID_INDEX = 13,
  OR_SINGULAR_MATRIX = 14,
};

/* ---- GF(2^8), src/galois.rs ---- */
void or_gf8_tables(uint8_t log_out[256], uint8_t exp_out[510]);
uint8_t or_gf8_mul(uint8_t a, uint8_t b);
int or_gf8_div(uint8_t a, uint8_t b, uint8_t *out);
uint8_t or_gf8_exp(uint8_t a, size_t n);

/* ---- GF((2^8)^2) tower, src/galois16.rs ---- */
uint16_t or_gf16_mul(uint16_t a, uint16_t b);
uint16_t or_gf16_inv(uint16_t a);
void or_gf16_const_matrix(uint16_t c, uint8_t out[4]);

/* ---- dense matrices, src/matrix.rs. field = 8 or 16; elements stored as u16 ---- */
int or_invert(int field, size_t n, const uint16_t *in, uint16_t *out);
void or_vandermonde(int field, size_t rows, size_t cols, uint16_t *out);
void or_matmul(int field, size_t r, size_t n, size_t c, const uint16_t *a,
               const uint16_t *b, uint16_t *out);
/* Systematic generator vandermonde(n,k) * inv(top k x k), src/reedsolomon.rs:155-159 */
int or_build_matrix(int field, size_t k, size_t n, uint16_t *out);

/* ---- encode, src/reedsolomon.rs:402-424 and src/reedsolomon16.rs:919-936 ---- */
/* data: k rows of len bytes back to back; parity: m rows of len bytes. */
int or_encode8(size_t k, size_t m, const uint8_t *data, uint8_t *parity, size_t len);
/* Same over rows of an arbitrary coefficient matrix (rows x k, u8). */
void or_apply8(size_t k, size_t rows, const uint8_t *coeffs, const uint8_t *const *in,
               uint8_t *const *out, size_t len);
int or_encode16(size_t k, size_t m, const uint8_t *data, uint8_t *parity, size_t len);

/* ---- reconstruct, src/reedsolomon.rs:470-641,801-891 (and the 16-bit twin) ----
 * rows: n = k+m rows of len bytes; present[i] != 0 for valid rows. Missing rows are
 * rebuilt in place (missing parity left untouched when data_only). */
int or_reconstruct(int field, size_t k, size_t m, uint8_t *rows, const uint8_t *present,
                   size_t len, int data_only);
/* The decode rows the reference plan uses (src/reedsolomon.rs:550-585): rows of the
 * inverted survivor matrix at the missing data indexes, in ascending order. */
int or_decode_rows(int field, size_t k, size_t m, const uint8_t *present,
                   uint16_t *rows_out, size_t *n_rows);

/* ---- column-sampled evaluation of the systematic code (eval_columns.c) ----
 * data: k shards of len bytes back to back (split-plane wire for field 16). For each
 * evaluation point x in points and each symbol column s in cols, out[p * n_cols + c] =
 * f(x) where f (degree < k) has f(i) = data symbol i at column s: the shard at index x
 * of the encoded stripe (src/reedsolomon.rs:155-159, src/field.rs:57-61). */
int or_eval_columns(int field, size_t k, const uint8_t *data, size_t len, const uint32_t *cols,
                    size_t n_cols, const uint32_t *points, size_t n_points, uint16_t *out);

/* ---- LCH additive-FFT programs over GF(2^8), src/fft.rs ---- */
/* Op encoding (one u32 per op): kind<<28 | dst<<18 | src<<8 | c, with
 * kind 0 = MulXor, 1 = Xor, 2 = MulCopy, 3 = Copy (src/fft.rs:87-97). */
int or_fft_flat_program(size_t k, size_t m, uint32_t *ops, size_t cap, size_t *n_ops,
                        size_t *register_count, uint16_t *parity_regs, size_t *mult_count);
int or_fft_staged_program(size_t k, size_t m, size_t *register_count, size_t *mult_count,
                          size_t *xor_count, size_t *n_stages, size_t *n_glue,
                          size_t *n_zero);
/* Replay a flat/staged program over one byte column (k bytes in, m bytes out). */
int or_fft_flat_run(size_t k, size_t m, const uint8_t *column, uint8_t *parity);
int or_fft_staged_run(size_t k, size_t m, const uint8_t *column, uint8_t *parity);
/* Normalised subspace-polynomial tables WHAT[8][256] (src/fft.rs:36-79). */
void or_fft_what(uint8_t out[8 * 256]);

/* ---- multi-threaded CPU baseline: one stripe per thread ---- */
/* stripes back to back: each stripe is (k+m) rows of len bytes; data rows read,
 * parity rows written. Returns elapsed seconds. */
double or_encode8_batch_mt(size_t k, size_t m, uint8_t *stripes, size_t n_stripes,
                           size_t len, int threads);
/* One thread, one stripe ((k+m) rows of len bytes) encoded reps times after an
 * untimed pass (a cache-resident stripe, as the reference's benches time it).
 * Returns seconds for the reps. */
double or_encode8_repeat(size_t k, size_t m, uint8_t *stripe, size_t len, size_t reps);
/* 1 when the GFNI/AVX-512 replay runs on this host, 0 for the scalar fallback. */
int or_cpu_has_gfni(void);
/* The path or_encode8_batch_mt takes: 2 straight-line zmm code (the six generated
 * shapes, len >= 64), 1 program replay from memory, 0 scalar. */
int or_cpu_path(size_t k, size_t m, size_t len);

#ifdef __cplusplus
}
#endif
#endif
