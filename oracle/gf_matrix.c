/*
 * CPU oracle: fields, matrices, generator, scalar encode and reconstruct.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h). A plain restatement of the reference's
 * scalar path; no SIMD, no shortcuts. Reference paths are relative to the crate root.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* GF(2^8) mod x^8+x^4+x^3+x^2+1, generator 2: src/galois.rs:3-57             */
/* ------------------------------------------------------------------------- */

static uint8_t LOG[256];
static uint8_t EXP[510];
static uint8_t MUL[256][256];
static int tables_ready = 0;

static void build_tables(void) {
  if (tables_ready) return;
  /* gen_log_table, src/galois.rs:9-22: walk powers of 2, reduce by 0x1d. */
  unsigned b = 1;
  for (unsigned log = 0; log < 255; log++) {
    LOG[b] = (uint8_t)log;
    b <<= 1;
    if (b >= 256) b = (b - 256) ^ 0x1d;
  }
  LOG[0] = 0;
  /* gen_exp_table, src/galois.rs:24-35: doubled so log_a + log_b never wraps. */
  for (unsigned i = 1; i < 256; i++) {
    unsigned l = LOG[i];
    EXP[l] = (uint8_t)i;
    EXP[l + 255] = (uint8_t)i;
  }
  /* gen_mul_table, src/galois.rs:37-57. */
  for (unsigned a = 0; a < 256; a++)
    for (unsigned c = 0; c < 256; c++)
      MUL[a][c] = (a == 0 || c == 0) ? 0 : EXP[LOG[a] + LOG[c]];
  tables_ready = 1;
}

void or_gf8_tables(uint8_t log_out[256], uint8_t exp_out[510]) {
  build_tables();
  memcpy(log_out, LOG, 256);
  memcpy(exp_out, EXP, 510);
}

uint8_t or_gf8_mul(uint8_t a, uint8_t b) {
  build_tables();
  return MUL[a][b];
}

/* src/galois.rs:80-93: div panics on a zero divisor; the oracle reports -1. */
int or_gf8_div(uint8_t a, uint8_t b, uint8_t *out) {
  build_tables();
  if (a == 0) {
    *out = 0;
    return 0;
  }
  if (b == 0) return -1;
  int r = (int)LOG[a] - (int)LOG[b];
  if (r < 0) r += 255;
  *out = EXP[r];
  return 0;
}

/* src/galois.rs:97-111 */
uint8_t or_gf8_exp(uint8_t a, size_t n) {
  build_tables();
  if (n == 0) return 1;
  if (a == 0) return 0;
  size_t r = (size_t)LOG[a] * n;
  while (r >= 255) r -= 255;
  return EXP[r];
}

static uint8_t gf8_inv(uint8_t a) {
  uint8_t out = 0;
  or_gf8_div(1, a, &out);
  return out;
}

/* ------------------------------------------------------------------------- */
/* GF((2^8)^2) tower y^2 + y + 32: src/galois16.rs:19-125                     */
/* ------------------------------------------------------------------------- */

#define TOWER_L 32

/* src/galois16.rs:45-59 */
uint16_t or_gf16_mul(uint16_t a, uint16_t b) {
  build_tables();
  uint8_t ah = a >> 8, al = a & 0xff, bh = b >> 8, bl = b & 0xff;
  uint8_t p2 = MUL[ah][bh];
  uint8_t p1 = MUL[ah][bl] ^ MUL[al][bh];
  uint8_t p0 = MUL[al][bl];
  uint8_t hi = p1 ^ p2;
  uint8_t lo = p0 ^ MUL[p2][TOWER_L];
  return (uint16_t)((hi << 8) | lo);
}

/* src/galois16.rs:76-84: [m00, m01, m10, m11], out_high = m00*a_high + m01*a_low,
 * out_low = m10*a_high + m11*a_low. */
void or_gf16_const_matrix(uint16_t c, uint8_t out[4]) {
  build_tables();
  uint8_t ch = c >> 8, cl = c & 0xff;
  out[0] = ch ^ cl;
  out[1] = ch;
  out[2] = MUL[ch][TOWER_L];
  out[3] = cl;
}

/* src/galois16.rs:110-125: conjugate times inverse norm. Zero maps to zero here
 * (the reference asserts); callers never pass zero. */
uint16_t or_gf16_inv(uint16_t a) {
  build_tables();
  if (a == 0) return 0;
  uint8_t ah = a >> 8, al = a & 0xff;
  uint16_t conj = (uint16_t)((ah << 8) | (uint8_t)(ah ^ al));
  uint16_t norm = or_gf16_mul(a, conj);
  uint8_t ni = gf8_inv((uint8_t)(norm & 0xff));
  return (uint16_t)((MUL[conj >> 8][ni] << 8) | MUL[conj & 0xff][ni]);
}

/* ------------------------------------------------------------------------- */
/* Generic field ops for the matrix layer: src/field.rs:12-88                 */
/* ------------------------------------------------------------------------- */

static inline uint16_t f_mul(int field, uint16_t a, uint16_t b) {
  return field == 8 ? MUL[a & 0xff][b & 0xff] : or_gf16_mul(a, b);
}
static inline uint16_t f_inv(int field, uint16_t a) {
  return field == 8 ? gf8_inv((uint8_t)a) : or_gf16_inv(a);
}

/* Matrix::multiply, src/matrix.rs:51-77 (row-at-a-time accumulation). */
void or_matmul(int field, size_t r, size_t n, size_t c, const uint16_t *a,
               const uint16_t *b, uint16_t *out) {
  build_tables();
  memset(out, 0, r * c * sizeof(uint16_t));
  for (size_t row = 0; row < r; row++) {
    for (size_t i = 0; i < n; i++) {
      uint16_t scale = a[row * n + i];
      if (scale == 0) continue;
      for (size_t col = 0; col < c; col++)
        out[row * c + col] ^= f_mul(field, scale, b[i * c + col]);
    }
  }
}

/* Matrix::vandermonde, src/matrix.rs:183-196 with evaluation_point(r) = r
 * (src/field.rs:57-61, :83-86). */
void or_vandermonde(int field, size_t rows, size_t cols, uint16_t *out) {
  build_tables();
  for (size_t r = 0; r < rows; r++) {
    uint16_t point = field == 8 ? (uint16_t)(uint8_t)r : (uint16_t)r;
    uint16_t power = 1;
    for (size_t c = 0; c < cols; c++) {
      out[r * cols + c] = power;
      power = f_mul(field, power, point);
    }
  }
}

/* Matrix::gaussian_elim, src/matrix.rs:123-168: pivot on the first nonzero entry
 * below, normalise, clear below, then clear above. */
static int gaussian_elim(int field, size_t rows, size_t cols, uint16_t *m) {
  for (size_t r = 0; r < rows; r++) {
    if (m[r * cols + r] == 0) {
      for (size_t rb = r + 1; rb < rows; rb++) {
        if (m[rb * cols + r] != 0) {
          for (size_t c = 0; c < cols; c++) {
            uint16_t t = m[r * cols + c];
            m[r * cols + c] = m[rb * cols + c];
            m[rb * cols + c] = t;
          }
          break;
        }
      }
    }
    if (m[r * cols + r] == 0) return OR_SINGULAR_MATRIX;
    if (m[r * cols + r] != 1) {
      uint16_t scale = f_inv(field, m[r * cols + r]);
      for (size_t c = 0; c < cols; c++) m[r * cols + c] = f_mul(field, scale, m[r * cols + c]);
    }
    for (size_t rb = r + 1; rb < rows; rb++) {
      uint16_t scale = m[rb * cols + r];
      if (scale == 0) continue;
      for (size_t c = 0; c < cols; c++) m[rb * cols + c] ^= f_mul(field, scale, m[r * cols + c]);
    }
  }
  for (size_t d = 0; d < rows; d++) {
    for (size_t ra = 0; ra < d; ra++) {
      uint16_t scale = m[ra * cols + d];
      if (scale == 0) continue;
      for (size_t c = 0; c < cols; c++) m[ra * cols + c] ^= f_mul(field, scale, m[d * cols + c]);
    }
  }
  return OR_OK;
}

/* Matrix::invert, src/matrix.rs:170-181: augment with I, eliminate, keep right half. */
int or_invert(int field, size_t n, const uint16_t *in, uint16_t *out) {
  build_tables();
  size_t cols = 2 * n;
  uint16_t *w = (uint16_t *)calloc(n * cols, sizeof(uint16_t));
  if (!w) return -1;
  for (size_t r = 0; r < n; r++) {
    memcpy(w + r * cols, in + r * n, n * sizeof(uint16_t));
    w[r * cols + n + r] = 1;
  }
  int st = gaussian_elim(field, n, cols, w);
  if (st == OR_OK)
    for (size_t r = 0; r < n; r++) memcpy(out + r * n, w + r * cols + n, n * sizeof(uint16_t));
  free(w);
  return st;
}

/* ReedSolomon::build_matrix, src/reedsolomon.rs:155-159 (and
 * src/reedsolomon16.rs:270-274): vandermonde(n, k) * invert(top k x k). */
int or_build_matrix(int field, size_t k, size_t n, uint16_t *out) {
  build_tables();
  uint16_t *v = (uint16_t *)malloc(n * k * sizeof(uint16_t));
  uint16_t *top_inv = (uint16_t *)malloc(k * k * sizeof(uint16_t));
  if (!v || !top_inv) {
    free(v);
    free(top_inv);
    return -1;
  }
  or_vandermonde(field, n, k, v);
  int st = or_invert(field, k, v, top_inv); /* top block = first k rows of v */
  if (st == OR_OK) or_matmul(field, n, k, k, v, top_inv, out);
  free(v);
  free(top_inv);
  return st;
}

/* ------------------------------------------------------------------------- */
/* Encode                                                                      */
/* ------------------------------------------------------------------------- */

/* gf::scalar::mul_slice(_xor), src/gf/scalar.rs:7-23, folded into the
 * per-input/per-output loop of encode_scalar, src/reedsolomon.rs:402-424. */
void or_apply8(size_t k, size_t rows, const uint8_t *coeffs, const uint8_t *const *in,
               uint8_t *const *out, size_t len) {
  build_tables();
  for (size_t i = 0; i < k; i++) {
    for (size_t j = 0; j < rows; j++) {
      const uint8_t *row = MUL[coeffs[j * k + i]];
      uint8_t *o = out[j];
      const uint8_t *x = in[i];
      if (i == 0)
        for (size_t t = 0; t < len; t++) o[t] = row[x[t]];
      else
        for (size_t t = 0; t < len; t++) o[t] ^= row[x[t]];
    }
  }
}

int or_encode8(size_t k, size_t m, const uint8_t *data, uint8_t *parity, size_t len) {
  if (k == 0) return OR_TOO_FEW_DATA_SHARDS;
  if (m == 0) return OR_TOO_FEW_PARITY_SHARDS;
  if (k + m > 256) return OR_TOO_MANY_SHARDS;
  size_t n = k + m;
  uint16_t *g = (uint16_t *)malloc(n * k * sizeof(uint16_t));
  uint8_t *c = (uint8_t *)malloc(m * k);
  const uint8_t **in = (const uint8_t **)malloc(k * sizeof(void *));
  uint8_t **out = (uint8_t **)malloc(m * sizeof(void *));
  int st = or_build_matrix(8, k, n, g);
  if (st == OR_OK) {
    for (size_t j = 0; j < m; j++)
      for (size_t i = 0; i < k; i++) c[j * k + i] = (uint8_t)g[(k + j) * k + i];
    for (size_t i = 0; i < k; i++) in[i] = data + i * len;
    for (size_t j = 0; j < m; j++) out[j] = parity + j * len;
    if (len) or_apply8(k, m, c, in, out, len);
  }
  free(g);
  free(c);
  free(in);
  free(out);
  return st;
}

/* symbolwise_parity, src/reedsolomon16.rs:919-936: parity symbol by symbol over the
 * split-plane wire [low N | high N] (src/reedsolomon16.rs:4-7). */
static void apply16(size_t k, size_t rows, const uint16_t *coeffs, const uint8_t *const *in,
                    uint8_t *const *out, size_t len) {
  size_t n_sym = len / 2;
  for (size_t j = 0; j < rows; j++) {
    for (size_t s = 0; s < n_sym; s++) {
      uint16_t acc = 0;
      for (size_t i = 0; i < k; i++) {
        uint16_t sym = (uint16_t)((in[i][n_sym + s] << 8) | in[i][s]);
        acc ^= or_gf16_mul(coeffs[j * k + i], sym);
      }
      out[j][s] = (uint8_t)(acc & 0xff);
      out[j][n_sym + s] = (uint8_t)(acc >> 8);
    }
  }
}

int or_encode16(size_t k, size_t m, const uint8_t *data, uint8_t *parity, size_t len) {
  if (k == 0) return OR_TOO_FEW_DATA_SHARDS;
  if (m == 0) return OR_TOO_FEW_PARITY_SHARDS;
  if (k + m > 65536) return OR_TOO_MANY_SHARDS;
  if (len == 0) return OR_EMPTY_SHARD;
  if (len % 2) return OR_INCORRECT_SHARD_SIZE;
  size_t n = k + m;
  uint16_t *g = (uint16_t *)malloc(n * k * sizeof(uint16_t));
  const uint8_t **in = (const uint8_t **)malloc(k * sizeof(void *));
  uint8_t **out = (uint8_t **)malloc(m * sizeof(void *));
  int st = or_build_matrix(16, k, n, g);
  if (st == OR_OK) {
    for (size_t i = 0; i < k; i++) in[i] = data + i * len;
    for (size_t j = 0; j < m; j++) out[j] = parity + j * len;
    apply16(k, m, g + k * k, in, out, len);
  }
  free(g);
  free(in);
  free(out);
  return st;
}

/* ------------------------------------------------------------------------- */
/* Reconstruct                                                                 */
/* ------------------------------------------------------------------------- */

/* build_plan + data_decode_matrix, src/reedsolomon.rs:539-585: survivors are the
 * first k present indexes ascending; data rows are rows of the inverted survivor
 * matrix at the missing data indexes. */
static int build_plan(int field, size_t k, size_t m, const uint16_t *g, const uint8_t *present,
                      size_t *valid, size_t *missing_data, size_t *n_md,
                      size_t *missing_parity, size_t *n_mp, uint16_t *data_rows) {
  size_t n = k + m, nv = 0;
  *n_md = 0;
  *n_mp = 0;
  for (size_t i = 0; i < n; i++) {
    if (present[i]) {
      if (nv < k) valid[nv++] = i;
    } else if (i < k) {
      missing_data[(*n_md)++] = i;
    } else {
      missing_parity[(*n_mp)++] = i;
    }
  }
  if (nv < k) return OR_TOO_FEW_SHARDS_PRESENT;
  uint16_t *sub = (uint16_t *)malloc(k * k * sizeof(uint16_t));
  uint16_t *inv = (uint16_t *)malloc(k * k * sizeof(uint16_t));
  for (size_t r = 0; r < k; r++) memcpy(sub + r * k, g + valid[r] * k, k * sizeof(uint16_t));
  int st = or_invert(field, k, sub, inv);
  if (st == OR_OK)
    for (size_t t = 0; t < *n_md; t++)
      memcpy(data_rows + t * k, inv + missing_data[t] * k, k * sizeof(uint16_t));
  free(sub);
  free(inv);
  return st;
}

int or_decode_rows(int field, size_t k, size_t m, const uint8_t *present, uint16_t *rows_out,
                   size_t *n_rows) {
  build_tables();
  size_t n = k + m;
  uint16_t *g = (uint16_t *)malloc(n * k * sizeof(uint16_t));
  size_t *valid = (size_t *)malloc(n * sizeof(size_t));
  size_t *md = (size_t *)malloc(n * sizeof(size_t));
  size_t *mp = (size_t *)malloc(n * sizeof(size_t));
  size_t n_mp = 0;
  int st = or_build_matrix(field, k, n, g);
  if (st == OR_OK) st = build_plan(field, k, m, g, present, valid, md, n_rows, mp, &n_mp, rows_out);
  free(g);
  free(valid);
  free(md);
  free(mp);
  return st;
}

/* reconstruct_with_plan, src/reedsolomon.rs:829-891 (16-bit twin
 * src/reedsolomon16.rs:806-891; strip-mining there is bit-identical by column
 * independence, so the oracle applies whole rows). */
int or_reconstruct(int field, size_t k, size_t m, uint8_t *rows, const uint8_t *present,
                   size_t len, int data_only) {
  build_tables();
  size_t n = k + m, n_present = 0;
  for (size_t i = 0; i < n; i++) n_present += present[i] ? 1 : 0;
  if (n_present == n) return OR_OK;
  if (n_present < k) return OR_TOO_FEW_SHARDS_PRESENT;
  uint16_t *g = (uint16_t *)malloc(n * k * sizeof(uint16_t));
  size_t *valid = (size_t *)malloc(n * sizeof(size_t));
  size_t *md = (size_t *)malloc(n * sizeof(size_t));
  size_t *mp = (size_t *)malloc(n * sizeof(size_t));
  uint16_t *drows = (uint16_t *)malloc(n * k * sizeof(uint16_t));
  size_t n_md = 0, n_mp = 0;
  int st = or_build_matrix(field, k, n, g);
  if (st == OR_OK) st = build_plan(field, k, m, g, present, valid, md, &n_md, mp, &n_mp, drows);
  if (st == OR_OK) {
    const uint8_t **in = (const uint8_t **)malloc(k * sizeof(void *));
    uint8_t **out = (uint8_t **)malloc(n * sizeof(void *));
    for (size_t t = 0; t < k; t++) in[t] = rows + valid[t] * len;
    for (size_t t = 0; t < n_md; t++) out[t] = rows + md[t] * len;
    if (n_md) {
      if (field == 8) {
        uint8_t *c8 = (uint8_t *)malloc(n_md * k);
        for (size_t t = 0; t < n_md * k; t++) c8[t] = (uint8_t)drows[t];
        or_apply8(k, n_md, c8, in, out, len);
        free(c8);
      } else {
        apply16(k, n_md, drows, in, out, len);
      }
    }
    if (!data_only && n_mp) {
      /* Missing parity from the completed data rows 0..k-1. */
      for (size_t i = 0; i < k; i++) in[i] = rows + i * len;
      for (size_t t = 0; t < n_mp; t++) out[t] = rows + mp[t] * len;
      uint16_t *prow = (uint16_t *)malloc(n_mp * k * sizeof(uint16_t));
      for (size_t t = 0; t < n_mp; t++) memcpy(prow + t * k, g + mp[t] * k, k * sizeof(uint16_t));
      if (field == 8) {
        uint8_t *c8 = (uint8_t *)malloc(n_mp * k);
        for (size_t t = 0; t < n_mp * k; t++) c8[t] = (uint8_t)prow[t];
        or_apply8(k, n_mp, c8, in, out, len);
        free(c8);
      } else {
        apply16(k, n_mp, prow, in, out, len);
      }
      free(prow);
    }
    free(in);
    free(out);
  }
  free(g);
  free(valid);
  free(md);
  free(mp);
  free(drows);
  return st;
}
