/*
 * CPU oracle: multi-threaded encode used as the timed CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h). A C restatement of the reference's x86
 * encode fast path, one stripe per thread:
 *
 * - the six generated shapes (7,13), (10,10), (14,14), (16,16), (18,6), (32,32) run
 *   straight-line code with every program register in a zmm register and one
 *   gf2p8affineqb per multiply, over 64-byte strips with an overlapped last strip,
 *   as the reference's macro-expanded zmm cores do (src/macros.rs:1-45,
 *   src/gf/fft_x86.rs:60-99, 149-211); that code is generated from the oracle's
 *   LCH builder by gen_straight.c into _build/cpu_straight.c;
 * - other shapes replay the same builder's flat program (src/fft.rs
 *   build_encode_program) from memory, 4 strips per op;
 * - shards shorter than one strip, or hosts without GFNI/AVX-512, take the scalar
 *   table path.
 */
#include <immintrin.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "lch_fft.h"
#include "oracle.h"

/* Affine matrix of multiply-by-c: output bit i is the parity of row i with the
 * input byte; row i (stored in byte 7-i) has bit j set when bit i of c*2^j is set. */
static uint64_t gfni_matrix(uint8_t c) {
  uint64_t mat = 0;
  for (int i = 0; i < 8; i++) {
    uint8_t row = 0;
    for (int j = 0; j < 8; j++) {
      uint8_t p = or_gf8_mul(c, (uint8_t)(1u << j));
      if (p & (1u << i)) row |= (uint8_t)(1u << j);
    }
    mat |= (uint64_t)row << (8 * (7 - i));
  }
  return mat;
}

typedef void (*or_straight_fn)(const uint8_t *const *, uint8_t *const *, size_t);
or_straight_fn or_straight_lookup(size_t k, size_t m); /* _build/cpu_straight.c */

typedef struct {
  size_t k, m, len, n_stripes;
  or_straight_fn straight;
  uint8_t *stripes;
  const lch_flat *prog;
  const uint64_t *mats; /* per op */
  int use_gfni;
  size_t next;
  pthread_mutex_t lock;
} job_t;

#define STRIPS 4

__attribute__((target("avx512f,avx512bw,gfni"))) static void run_block_gfni(
    const lch_flat *prog, const uint64_t *mats, const uint8_t *const *in, uint8_t *const *out,
    size_t off, __m512i *r) {
  for (size_t i = 0; i < prog->k; i++)
    for (int s = 0; s < STRIPS; s++)
      r[i * STRIPS + s] = _mm512_loadu_si512((const void *)(in[i] + off + 64 * s));
  for (size_t p = 0; p < prog->n_ops; p++) {
    lch_op op = prog->ops[p];
    __m512i *d = r + (size_t)op.dst * STRIPS;
    const __m512i *x = r + (size_t)op.src * STRIPS;
    __m512i a = _mm512_set1_epi64((long long)mats[p]);
    switch (op.kind) {
      case LCH_MULXOR:
        for (int s = 0; s < STRIPS; s++)
          d[s] = _mm512_xor_si512(d[s], _mm512_gf2p8affine_epi64_epi8(x[s], a, 0));
        break;
      case LCH_XOR:
        for (int s = 0; s < STRIPS; s++) d[s] = _mm512_xor_si512(d[s], x[s]);
        break;
      case LCH_MULCOPY:
        for (int s = 0; s < STRIPS; s++) d[s] = _mm512_gf2p8affine_epi64_epi8(x[s], a, 0);
        break;
      default:
        for (int s = 0; s < STRIPS; s++) d[s] = x[s];
        break;
    }
  }
  for (size_t j = 0; j < prog->m; j++)
    for (int s = 0; s < STRIPS; s++)
      _mm512_storeu_si512((void *)(out[j] + off + 64 * s), r[(size_t)prog->parity_regs[j] * STRIPS + s]);
}

static void encode_stripe(job_t *jb, uint8_t *stripe, __m512i *regs) {
  size_t k = jb->k, m = jb->m, len = jb->len;
  const uint8_t *in[256];
  uint8_t *out[256];
  for (size_t i = 0; i < k; i++) in[i] = stripe + i * len;
  for (size_t j = 0; j < m; j++) out[j] = stripe + (k + j) * len;
  if (jb->straight && len >= 64) {
    jb->straight(in, out, len);
    return;
  }
  const size_t block = 64 * STRIPS;
  size_t off = 0;
  if (jb->use_gfni && len >= block) {
    for (; off + block <= len; off += block) run_block_gfni(jb->prog, jb->mats, in, out, off, regs);
    if (off < len) run_block_gfni(jb->prog, jb->mats, in, out, len - block, regs); /* overlapped tail */
    return;
  }
  uint8_t col[256], par[256];
  for (size_t t = 0; t < len; t++) {
    for (size_t i = 0; i < k; i++) col[i] = in[i][t];
    lch_run_flat(jb->prog, col, par);
    for (size_t j = 0; j < m; j++) out[j][t] = par[j];
  }
}

static void *worker(void *arg) {
  job_t *jb = (job_t *)arg;
  __m512i *regs = (__m512i *)aligned_alloc(64, (jb->prog->register_count + 1) * STRIPS * 64);
  for (;;) {
    pthread_mutex_lock(&jb->lock);
    size_t s = jb->next++;
    pthread_mutex_unlock(&jb->lock);
    if (s >= jb->n_stripes) break;
    encode_stripe(jb, jb->stripes + s * (jb->k + jb->m) * jb->len, regs);
  }
  free(regs);
  return NULL;
}

double or_encode8_batch_mt(size_t k, size_t m, uint8_t *stripes, size_t n_stripes, size_t len,
                           int threads) {
  lch_flat prog;
  if (lch_build_flat(k, m, &prog)) return -1.0;
  uint64_t *mats = (uint64_t *)malloc((prog.n_ops + 1) * sizeof(uint64_t));
  for (size_t p = 0; p < prog.n_ops; p++) mats[p] = gfni_matrix(prog.ops[p].c);
  job_t jb;
  memset(&jb, 0, sizeof(jb));
  jb.k = k;
  jb.m = m;
  jb.len = len;
  jb.n_stripes = n_stripes;
  jb.stripes = stripes;
  jb.prog = &prog;
  jb.mats = mats;
  __builtin_cpu_init();
  jb.use_gfni = __builtin_cpu_supports("gfni") && __builtin_cpu_supports("avx512bw");
  jb.straight = jb.use_gfni ? or_straight_lookup(k, m) : NULL;
  pthread_mutex_init(&jb.lock, NULL);
  if (threads < 1) threads = 1;
  pthread_t *tid = (pthread_t *)malloc(threads * sizeof(pthread_t));
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (int t = 0; t < threads; t++) pthread_create(&tid[t], NULL, worker, &jb);
  for (int t = 0; t < threads; t++) pthread_join(tid[t], NULL);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  pthread_mutex_destroy(&jb.lock);
  free(tid);
  free(mats);
  lch_free_flat(&prog);
  return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

/* One thread encodes one stripe reps times after one untimed pass, as the
 * reference's criterion benches time a stripe that stays in cache
 * (benches/bench-harness/src/main.rs:100-117). Returns seconds for the reps. */
double or_encode8_repeat(size_t k, size_t m, uint8_t *stripe, size_t len, size_t reps) {
  lch_flat prog;
  if (lch_build_flat(k, m, &prog)) return -1.0;
  uint64_t *mats = (uint64_t *)malloc((prog.n_ops + 1) * sizeof(uint64_t));
  for (size_t p = 0; p < prog.n_ops; p++) mats[p] = gfni_matrix(prog.ops[p].c);
  job_t jb;
  memset(&jb, 0, sizeof(jb));
  jb.k = k;
  jb.m = m;
  jb.len = len;
  jb.prog = &prog;
  jb.mats = mats;
  __builtin_cpu_init();
  jb.use_gfni = __builtin_cpu_supports("gfni") && __builtin_cpu_supports("avx512bw");
  jb.straight = jb.use_gfni ? or_straight_lookup(k, m) : NULL;
  __m512i *regs = (__m512i *)aligned_alloc(64, (prog.register_count + 1) * STRIPS * 64);
  encode_stripe(&jb, stripe, regs);
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (size_t r = 0; r < reps; r++) encode_stripe(&jb, stripe, regs);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  free(regs);
  free(mats);
  lch_free_flat(&prog);
  return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

/* Reports whether the GFNI path is used on this host (1) or the scalar one (0). */
int or_cpu_has_gfni(void) {
  __builtin_cpu_init();
  return __builtin_cpu_supports("gfni") && __builtin_cpu_supports("avx512bw");
}

/* Path or_encode8_batch_mt takes for (k, m) at shard length len: 2 straight-line
 * zmm code, 1 the program replayed from memory, 0 scalar. */
int or_cpu_path(size_t k, size_t m, size_t len) {
  if (!or_cpu_has_gfni()) return 0;
  if (or_straight_lookup(k, m) && len >= 64) return 2;
  return len >= 64 * STRIPS ? 1 : 0;
}
