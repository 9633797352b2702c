/*
 * Emits oracle/_build/cpu_straight.c: straight-line AVX-512 + GFNI encoders for the
 * reference's six generated FFT shapes. TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference runs each generated encode program (src/fft_programs.rs) expanded
 * into straight-line code by its fft_run macro (src/macros.rs:1-45): every register
 * index is a literal, so the register array becomes SSA values held in machine
 * registers, and each 64-byte strip is one pass of that code with one
 * gf2p8affineqb per program multiply (the zmm cores of src/gf/fft_x86.rs:60-99,
 * 149-167, 205-211). This generator writes the same kind of code: it takes the op
 * list from this oracle's LCH builder (lch_fft.c, which reproduces the reference's
 * generated lists op for op; the fixture tests pin that by SHA-256) and prints one C
 * function per shape whose registers are local __m512i variables, plus the strip
 * loop with the overlapped last strip (src/gf/fft_x86.rs:149-167).
 *
 *     gen_straight > _build/cpu_straight.c
 */
#include <stdio.h>

#include "lch_fft.h"
#include "oracle.h"

static const int kShapes[][2] = {{7, 13}, {10, 10}, {14, 14}, {16, 16}, {18, 6}, {32, 32}};

/* Affine matrix of multiply-by-c for gf2p8affineqb: row i (byte 7 - i) has bit j set
 * when bit i of c * 2^j is set (src/gf/gfni.rs:12-64). */
static unsigned long long affine(uint8_t c) {
  unsigned long long mat = 0;
  for (int i = 0; i < 8; i++) {
    unsigned row = 0;
    for (int j = 0; j < 8; j++)
      if (or_gf8_mul(c, (uint8_t)(1u << j)) & (1u << i)) row |= 1u << j;
    mat |= (unsigned long long)row << (8 * (7 - i));
  }
  return mat;
}

static int emit(int k, int m) {
  lch_flat p;
  if (lch_build_flat((size_t)k, (size_t)m, &p)) return 1;
  printf("\n/* RS(%d,%d): %zu registers, %zu ops, %zu multiplies. */\n", k, m, p.register_count, p.n_ops,
         p.mult_count);
  printf("ZMM static void strip_%d_%d(const uint8_t *const *in, uint8_t *const *out, size_t off) {\n", k, m);
  for (size_t r = 0; r < p.register_count; r++) printf("  __m512i r%zu = _mm512_setzero_si512();\n", r);
  for (int i = 0; i < k; i++) printf("  r%d = _mm512_loadu_si512((const void *)(in[%d] + off));\n", i, i);
  for (size_t i = 0; i < p.n_ops; i++) {
    const lch_op o = p.ops[i];
    switch (o.kind) {
      case LCH_MULXOR:
        printf("  r%u = _mm512_xor_si512(r%u, _mm512_gf2p8affine_epi64_epi8(r%u, _mm512_set1_epi64(0x%016llxLL), 0));\n",
               o.dst, o.dst, o.src, affine(o.c));
        break;
      case LCH_XOR:
        printf("  r%u = _mm512_xor_si512(r%u, r%u);\n", o.dst, o.dst, o.src);
        break;
      case LCH_MULCOPY:
        printf("  r%u = _mm512_gf2p8affine_epi64_epi8(r%u, _mm512_set1_epi64(0x%016llxLL), 0);\n", o.dst, o.src,
               affine(o.c));
        break;
      default:
        printf("  r%u = r%u;\n", o.dst, o.src);
        break;
    }
  }
  for (int j = 0; j < m; j++) printf("  _mm512_storeu_si512((void *)(out[%d] + off), r%u);\n", j, p.parity_regs[j]);
  printf("}\n\n");
  printf("ZMM static void encode_%d_%d(const uint8_t *const *in, uint8_t *const *out, size_t len) {\n", k, m);
  printf("  size_t pos = 0;\n");
  printf("  for (;;) {\n");
  printf("    const size_t off = pos + 64 <= len ? pos : len - 64;\n");
  printf("    strip_%d_%d(in, out, off);\n", k, m);
  printf("    if (off + 64 >= len) break;\n");
  printf("    pos += 64;\n");
  printf("  }\n}\n");
  lch_free_flat(&p);
  return 0;
}

int main(void) {
  printf("/* Generated by oracle/gen_straight.c from the oracle's LCH program builder; do not edit.\n"
         " * TEST INFRASTRUCTURE ONLY: the timed CPU baseline's straight-line encoders. */\n");
  printf("#include <immintrin.h>\n#include <stddef.h>\n#include <stdint.h>\n\n");
  printf("#define ZMM __attribute__((target(\"avx512f,avx512bw,gfni\")))\n");
  printf("typedef void (*or_straight_fn)(const uint8_t *const *, uint8_t *const *, size_t);\n");
  const int n = (int)(sizeof(kShapes) / sizeof(kShapes[0]));
  for (int i = 0; i < n; i++)
    if (emit(kShapes[i][0], kShapes[i][1])) return 1;
  printf("\n/* The straight-line encoder of (k, m), or NULL. Needs len >= 64. */\n");
  printf("or_straight_fn or_straight_lookup(size_t k, size_t m) {\n");
  for (int i = 0; i < n; i++)
    printf("  if (k == %d && m == %d) return encode_%d_%d;\n", kShapes[i][0], kShapes[i][1], kShapes[i][0],
           kShapes[i][1]);
  printf("  return NULL;\n}\n");
  return 0;
}
