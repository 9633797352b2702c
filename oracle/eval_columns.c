/*
 * Column-sampled evaluation of the systematic code (TEST INFRASTRUCTURE ONLY).
 *
 * The reference's systematic generator is vandermonde(n, k) * inverse(top k x k)
 * (src/reedsolomon.rs:155-159, src/reedsolomon16.rs:270-274) with evaluation point
 * i = i (src/field.rs:57-61). Row r of that matrix is the Lagrange basis on the points
 * 0..k-1 evaluated at point r, so at every symbol column the shards of an encoded
 * stripe are the values at 0..n-1 of the unique polynomial f of degree < k with
 * f(i) = data symbol i. The reference's own independent check computes parity symbol
 * by symbol from those rows (symbolwise_parity, src/reedsolomon16.rs:919-936); this
 * file evaluates the same rows in barycentric form,
 *
 *     f(x) = L(x) * sum_i w_i d_i / (x - i),   L(x) = prod_t (x - t),
 *     w_i = 1 / prod_{t != i} (i - t),
 *
 * which needs O(k) field operations per point and column instead of the O(k^3)
 * Gauss-Jordan that or_build_matrix performs. That makes shapes such as
 * ReedSolomon16 (4096, 12288) checkable at sampled columns. Subtraction is XOR in both
 * fields; products go through discrete-log tables of each field's own multiply
 * (or_gf8_mul for GF(2^8) mod 0x11d, or_gf16_mul for the tower y^2 + y + 32), so the
 * arithmetic is the oracle's, only reorganised.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

typedef struct {
  int ready;
  uint32_t q; /* multiplicative group order */
  uint32_t *log;
  uint16_t *exp; /* 2q entries */
} LogTables;

static LogTables g_lt[2];

static uint16_t fmul(int field, uint16_t a, uint16_t b) {
  return field == 8 ? or_gf8_mul((uint8_t)a, (uint8_t)b) : or_gf16_mul(a, b);
}

/* Logs to a generator of the field's multiplicative group, found by search: the
 * smallest element whose powers run through all q nonzero elements. */
static LogTables *tables(int field) {
  LogTables *t = &g_lt[field == 8 ? 0 : 1];
  if (t->ready) return t;
  const uint32_t q = field == 8 ? 255u : 65535u;
  t->q = q;
  t->log = (uint32_t *)calloc(q + 1, sizeof(uint32_t));
  t->exp = (uint16_t *)calloc(2 * (size_t)q, sizeof(uint16_t));
  for (uint32_t g = 2; g <= q; g++) {
    uint16_t x = 1;
    uint32_t order = 0;
    do {
      t->exp[order] = x;
      x = fmul(field, x, (uint16_t)g);
      order++;
    } while (x != 1 && order <= q);
    if (order == q) break;
  }
  for (uint32_t e = 0; e < q; e++) {
    t->log[t->exp[e]] = e;
    t->exp[e + q] = t->exp[e];
  }
  t->ready = 1;
  return t;
}

/* Symbol s of shard i: GF(2^8) byte s; tower symbol (high << 8) | low on the
 * split-plane wire [low N | high N] (src/reedsolomon16.rs:4-7, 143-168). */
static uint16_t symbol(int field, const uint8_t *shard, size_t len, size_t s) {
  if (field == 8) return shard[s];
  const size_t half = len / 2;
  return (uint16_t)(((uint16_t)shard[half + s] << 8) | shard[s]);
}

int or_eval_columns(int field, size_t k, const uint8_t *data, size_t len, const uint32_t *cols,
                    size_t n_cols, const uint32_t *points, size_t n_points, uint16_t *out) {
  if ((field != 8 && field != 16) || k == 0) return OR_INVALID_INDEX;
  const size_t n_sym = field == 8 ? len : len / 2;
  const uint32_t qmax = field == 8 ? 256u : 65536u;
  if (k > qmax) return OR_TOO_MANY_DATA_SHARDS;
  for (size_t c = 0; c < n_cols; c++)
    if (cols[c] >= n_sym) return OR_INVALID_INDEX;
  for (size_t p = 0; p < n_points; p++)
    if (points[p] >= qmax) return OR_INVALID_INDEX;
  LogTables *t = tables(field);
  const uint32_t q = t->q;
  /* log w_i = -(sum_{t != i} log(i ^ t)) mod q */
  uint64_t *logw = (uint64_t *)malloc(k * sizeof(uint64_t));
  uint32_t *logc = (uint32_t *)malloc(k * sizeof(uint32_t));
  uint32_t *logd = (uint32_t *)malloc(k * n_cols * sizeof(uint32_t));
  uint8_t *zero = (uint8_t *)malloc(k * n_cols);
  if (!logw || !logc || !logd || !zero) {
    free(logw);
    free(logc);
    free(logd);
    free(zero);
    return OR_INVALID_INDEX;
  }
  for (size_t i = 0; i < k; i++) {
    uint64_t s = 0;
    for (size_t j = 0; j < k; j++)
      if (j != i) s += t->log[i ^ j];
    logw[i] = (q - s % q) % q;
  }
  for (size_t i = 0; i < k; i++)
    for (size_t c = 0; c < n_cols; c++) {
      const uint16_t d = symbol(field, data + i * len, len, cols[c]);
      zero[i * n_cols + c] = d == 0;
      logd[i * n_cols + c] = d ? t->log[d] : 0;
    }
  for (size_t p = 0; p < n_points; p++) {
    const uint32_t x = points[p];
    uint16_t *row = out + p * n_cols;
    if (x < k) { /* a data point: f(x) is the data symbol itself */
      for (size_t c = 0; c < n_cols; c++) row[c] = symbol(field, data + (size_t)x * len, len, cols[c]);
      continue;
    }
    uint64_t logl = 0;
    for (size_t j = 0; j < k; j++) logl += t->log[x ^ j];
    logl %= q;
    for (size_t i = 0; i < k; i++) logc[i] = (uint32_t)((logw[i] + logl + q - t->log[x ^ i]) % q);
    for (size_t c = 0; c < n_cols; c++) {
      uint16_t acc = 0;
      for (size_t i = 0; i < k; i++)
        if (!zero[i * n_cols + c]) acc ^= t->exp[logc[i] + logd[i * n_cols + c]];
      row[c] = acc;
    }
  }
  free(logw);
  free(logc);
  free(logd);
  free(zero);
  return OR_OK;
}
