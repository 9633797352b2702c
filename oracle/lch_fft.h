/*
 * CPU oracle: LCH additive-FFT program types (restating src/fft.rs:87-154).
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#ifndef RS_ORACLE_LCH_FFT_H
#define RS_ORACLE_LCH_FFT_H

#include <stddef.h>
#include <stdint.h>

enum { LCH_MULXOR = 0, LCH_XOR = 1, LCH_MULCOPY = 2, LCH_COPY = 3 };

typedef struct {
  int kind;
  uint16_t dst, src;
  uint8_t c;
} lch_op;

typedef struct {
  lch_op *ops;
  size_t n_ops;
  size_t register_count;
  uint16_t *parity_regs;
  size_t k, m;
  size_t mult_count;
} lch_flat;

typedef struct {
  int is_transform, inverse;
  uint32_t start, size, len, consts_start;
} lch_stage;

typedef struct {
  lch_stage *stages;
  size_t n_stages;
  uint8_t *consts;
  size_t n_consts;
  lch_op *glue;
  size_t n_glue;
  uint16_t *zero_regs;
  size_t n_zero;
  uint16_t *parity_regs;
  size_t register_count, k, m;
  size_t mult_count, xor_count, boundary_count;
} lch_staged;

int lch_build_flat(size_t k, size_t m, lch_flat *prog);
void lch_free_flat(lch_flat *prog);
int lch_build_staged(size_t k, size_t m, lch_staged *prog);
void lch_free_staged(lch_staged *prog);
void lch_run_flat(const lch_flat *prog, const uint8_t *column, uint8_t *parity);
void lch_run_staged(const lch_staged *prog, const uint8_t *column, uint8_t *parity);

#endif
