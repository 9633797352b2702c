/*
 * CPU oracle: Lin-Chung-Han novel-basis additive FFT encode programs over GF(2^8).
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h). Restates src/fft.rs of the reference:
 * the subspace-polynomial tables, the interpolation builder, the flat lowering
 * (flatten, zero-read normalisation, dead-code elimination, register remap) and
 * the staged lowering, plus byte interpreters for both. A flat program built here
 * must equal the reference's generated op lists (src/fft_programs.rs) op for op;
 * tests pin that through digests recorded from the reference file.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "lch_fft.h"

static uint8_t WHAT[8][256];
static int what_ready = 0;

/* gen_what_tables, src/fft.rs:36-79: W_0(x) = x, W_{j+1} = W_j (W_j + W_j(2^j)),
 * then each level scaled so WHAT[j][2^j] = 1. */
static void build_what(void) {
  if (what_ready) return;
  uint8_t w[8][256];
  for (int x = 0; x < 256; x++) w[0][x] = (uint8_t)x;
  for (int j = 0; j + 1 < 8; j++) {
    uint8_t pivot = w[j][1 << j];
    for (int x = 0; x < 256; x++) w[j + 1][x] = or_gf8_mul(w[j][x], w[j][x] ^ pivot);
  }
  for (int j = 0; j < 8; j++) {
    uint8_t pivot = w[j][1 << j], inverse = 0;
    for (int cand = 1; cand < 256; cand++)
      if (or_gf8_mul(pivot, (uint8_t)cand) == 1) {
        inverse = (uint8_t)cand;
        break;
      }
    for (int x = 0; x < 256; x++) WHAT[j][x] = or_gf8_mul(w[j][x], inverse);
  }
  what_ready = 1;
}

void or_fft_what(uint8_t out[8 * 256]) {
  build_what();
  memcpy(out, WHAT, sizeof(WHAT));
}

/* ---- builder (src/fft.rs:156-240) ---- */

typedef struct {
  int is_transform;
  int inverse;
  uint16_t start, size;
  size_t beta;
  lch_op op;
} item_t;

typedef struct {
  item_t *items;
  size_t n, cap;
  uint16_t next_register;
} builder_t;

static void push_item(builder_t *b, item_t it) {
  if (b->n == b->cap) {
    b->cap = b->cap ? 2 * b->cap : 256;
    b->items = (item_t *)realloc(b->items, b->cap * sizeof(item_t));
  }
  b->items[b->n++] = it;
}

static void glue(builder_t *b, int kind, uint16_t dst, uint16_t src, uint8_t c) {
  item_t it;
  memset(&it, 0, sizeof(it));
  it.op.kind = kind;
  it.op.dst = dst;
  it.op.src = src;
  it.op.c = c;
  push_item(b, it);
}

static uint16_t alloc_regs(builder_t *b, size_t count) {
  uint16_t start = b->next_register;
  b->next_register = (uint16_t)(b->next_register + count);
  return start;
}

static void transform(builder_t *b, int inverse, uint16_t start, size_t size, size_t beta) {
  if (size <= 1) return; /* fft()/ifft() skip single registers, src/fft.rs:181-193 */
  item_t it;
  memset(&it, 0, sizeof(it));
  it.is_transform = 1;
  it.inverse = inverse;
  it.start = start;
  it.size = (uint16_t)size;
  it.beta = beta;
  push_item(b, it);
}

static int ctz(size_t x) {
  int n = 0;
  while (!(x & 1)) {
    x >>= 1;
    n++;
  }
  return n;
}

static size_t next_pow2(size_t x) {
  size_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

/* Builder::interpolate, src/fft.rs:198-239 */
static void interpolate(builder_t *b, uint16_t start, size_t n, size_t beta, size_t k) {
  if (k == n) {
    transform(b, 1, start, n, beta);
    return;
  }
  size_t half = n / 2;
  if (k <= half) {
    interpolate(b, start, half, beta, k);
    return;
  }
  transform(b, 1, start, half, beta);
  int level = ctz(n) - 1;
  uint8_t c = WHAT[level][beta];
  uint16_t scratch = alloc_regs(b, half);
  for (size_t j = 0; j < half; j++) glue(b, LCH_XOR, (uint16_t)(scratch + j), (uint16_t)(start + j), 0);
  transform(b, 0, scratch, half, beta ^ half);
  for (size_t i = 0; i < k - half; i++)
    glue(b, LCH_XOR, (uint16_t)(start + half + i), (uint16_t)(scratch + i), 0);
  interpolate(b, (uint16_t)(start + half), half, beta ^ half, k - half);
  for (size_t j = 0; j < k - half; j++) {
    if (c == 1)
      glue(b, LCH_XOR, (uint16_t)(start + j), (uint16_t)(start + half + j), 0);
    else if (c != 0)
      glue(b, LCH_MULXOR, (uint16_t)(start + j), (uint16_t)(start + half + j), c);
  }
}

/* build_interpolation, src/fft.rs:291-296 */
static uint16_t build_interpolation(builder_t *b, size_t k) {
  size_t t = next_pow2(k);
  uint16_t base = alloc_regs(b, t);
  interpolate(b, base, t, 0, k);
  return base;
}

/* ---- op vectors ---- */

typedef struct {
  lch_op *v;
  size_t n, cap;
} opvec_t;

static void opv_push(opvec_t *o, lch_op op) {
  if (o->n == o->cap) {
    o->cap = o->cap ? 2 * o->cap : 1024;
    o->v = (lch_op *)realloc(o->v, o->cap * sizeof(lch_op));
  }
  o->v[o->n++] = op;
}

static lch_op mk(int kind, uint16_t dst, uint16_t src, uint8_t c) {
  lch_op op;
  op.kind = kind;
  op.dst = dst;
  op.src = src;
  op.c = c;
  return op;
}

/* flatten_items, src/fft.rs:244-288: forward walks levels high to low, inverse low
 * to high; one constant per block, butterflies ascending. */
static void flatten(const builder_t *b, opvec_t *out) {
  for (size_t t = 0; t < b->n; t++) {
    const item_t *it = &b->items[t];
    if (!it->is_transform) {
      opv_push(out, it->op);
      continue;
    }
    size_t n = it->size;
    int levels = ctz(n);
    for (int li = 0; li < levels; li++) {
      int level = it->inverse ? li : levels - 1 - li;
      size_t stride = (size_t)1 << level;
      for (size_t base = 0; base < n; base += 2 * stride) {
        uint8_t c = WHAT[level][it->beta ^ base];
        for (size_t i = base; i < base + stride; i++) {
          uint16_t lo = (uint16_t)(it->start + i), hi = (uint16_t)(it->start + i + stride);
          if (it->inverse) {
            opv_push(out, mk(LCH_XOR, hi, lo, 0));
            if (c == 1)
              opv_push(out, mk(LCH_XOR, lo, hi, 0));
            else if (c != 0)
              opv_push(out, mk(LCH_MULXOR, lo, hi, c));
          } else {
            if (c == 1)
              opv_push(out, mk(LCH_XOR, lo, hi, 0));
            else if (c != 0)
              opv_push(out, mk(LCH_MULXOR, lo, hi, c));
            opv_push(out, mk(LCH_XOR, hi, lo, 0));
          }
        }
      }
    }
  }
}

/* normalize_zero_reads, src/fft.rs:596-631 */
static void normalize(const opvec_t *in, size_t reg_count, size_t k, opvec_t *out) {
  char *is_zero = (char *)malloc(reg_count);
  memset(is_zero, 1, reg_count);
  memset(is_zero, 0, k < reg_count ? k : reg_count);
  for (size_t t = 0; t < in->n; t++) {
    lch_op op = in->v[t];
    if (is_zero[op.src]) continue;
    if (is_zero[op.dst]) {
      op.kind = op.kind == LCH_MULXOR ? LCH_MULCOPY : LCH_COPY;
      is_zero[op.dst] = 0;
    }
    opv_push(out, op);
  }
  free(is_zero);
}

/* remap_registers, src/fft.rs:640-716: data registers keep 0..k-1, every other
 * register takes a slot from a free stack on first touch (src before dst) and
 * returns it after its last read. */
static size_t remap(opvec_t *ops, uint16_t *parity_regs, size_t m, size_t reg_count, size_t k) {
  size_t nops = ops->n;
  size_t *last_use = (size_t *)calloc(reg_count, sizeof(size_t));
  for (size_t p = 0; p < nops; p++) {
    last_use[ops->v[p].dst] = p;
    last_use[ops->v[p].src] = p;
  }
  for (size_t j = 0; j < m; j++) last_use[parity_regs[j]] = nops;
  int *mapping = (int *)malloc(reg_count * sizeof(int));
  for (size_t r = 0; r < reg_count; r++) mapping[r] = r < k ? (int)r : -1;
  /* expires[position] lists, built in the reference's order. */
  size_t *exp_count = (size_t *)calloc(nops + 1, sizeof(size_t));
  for (size_t r = 0; r < reg_count; r++)
    if (mapping[r] < 0) exp_count[last_use[r]]++;
  for (size_t r = 0; r < k && r < reg_count; r++)
    if (last_use[r] < nops) exp_count[last_use[r]]++;
  size_t *exp_off = (size_t *)calloc(nops + 2, sizeof(size_t));
  for (size_t p = 0; p <= nops; p++) exp_off[p + 1] = exp_off[p] + exp_count[p];
  size_t *exp_list = (size_t *)malloc((exp_off[nops + 1] + 1) * sizeof(size_t));
  size_t *fill = (size_t *)calloc(nops + 1, sizeof(size_t));
  for (size_t r = 0; r < reg_count; r++)
    if (mapping[r] < 0) exp_list[exp_off[last_use[r]] + fill[last_use[r]]++] = r;
  for (size_t r = 0; r < k && r < reg_count; r++)
    if (last_use[r] < nops) exp_list[exp_off[last_use[r]] + fill[last_use[r]]++] = r;

  uint16_t *free_stack = (uint16_t *)malloc((reg_count + 1) * sizeof(uint16_t));
  size_t n_free = 0;
  uint16_t next_fresh = (uint16_t)k;
  for (size_t p = 0; p < nops; p++) {
    uint16_t regs2[2] = {ops->v[p].src, ops->v[p].dst};
    for (int q = 0; q < 2; q++) {
      uint16_t vr = regs2[q];
      if (mapping[vr] < 0) mapping[vr] = n_free ? free_stack[--n_free] : next_fresh++;
    }
    ops->v[p].dst = (uint16_t)mapping[ops->v[p].dst];
    ops->v[p].src = (uint16_t)mapping[ops->v[p].src];
    for (size_t e = exp_off[p]; e < exp_off[p + 1]; e++)
      if (mapping[exp_list[e]] >= 0) free_stack[n_free++] = (uint16_t)mapping[exp_list[e]];
  }
  for (size_t j = 0; j < m; j++) parity_regs[j] = (uint16_t)mapping[parity_regs[j]];
  free(last_use);
  free(mapping);
  free(exp_count);
  free(exp_off);
  free(exp_list);
  free(fill);
  free(free_stack);
  return next_fresh;
}

/* build_encode_program, src/fft.rs:303-385 */
int lch_build_flat(size_t k, size_t m, lch_flat *prog) {
  build_what();
  memset(prog, 0, sizeof(*prog));
  if (k == 0 || m == 0 || k + m > 256) return -1;
  size_t n = k + m, t = next_pow2(k);
  builder_t b;
  memset(&b, 0, sizeof(b));
  uint16_t base = build_interpolation(&b, k);
  uint16_t *parity = (uint16_t *)calloc(m, sizeof(uint16_t));
  for (size_t bb = t; bb < n; bb += t) {
    uint16_t block = alloc_regs(&b, t);
    for (size_t j = 0; j < (k < t ? k : t); j++)
      glue(&b, LCH_XOR, (uint16_t)(block + j), (uint16_t)(base + j), 0);
    transform(&b, 0, block, t, bb);
    for (size_t point = bb; point < bb + t; point++)
      if (point >= k && point < n) parity[point - k] = (uint16_t)(block + point - bb);
  }
  transform(&b, 0, base, t, 0);
  size_t top = n < t ? n : t;
  size_t in_base = top > k ? top - k : 0;
  for (size_t j = 0; j < in_base; j++) parity[j] = (uint16_t)(base + k + j);

  opvec_t flat = {0}, norm = {0}, kept = {0};
  flatten(&b, &flat);
  size_t reg_count = b.next_register;
  normalize(&flat, reg_count, k, &norm);
  /* Backward liveness from the parity registers; full writes kill. */
  char *needed = (char *)calloc(reg_count, 1);
  for (size_t j = 0; j < m; j++) needed[parity[j]] = 1;
  for (size_t p = norm.n; p-- > 0;) {
    lch_op op = norm.v[p];
    if (!needed[op.dst]) continue;
    if (op.kind == LCH_MULCOPY || op.kind == LCH_COPY) needed[op.dst] = 0;
    needed[op.src] = 1;
    opv_push(&kept, op);
  }
  for (size_t i = 0, j = kept.n ? kept.n - 1 : 0; i < j; i++, j--) {
    lch_op tmp = kept.v[i];
    kept.v[i] = kept.v[j];
    kept.v[j] = tmp;
  }
  size_t mults = 0;
  for (size_t p = 0; p < kept.n; p++)
    if (kept.v[p].kind == LCH_MULXOR || kept.v[p].kind == LCH_MULCOPY) mults++;
  prog->register_count = remap(&kept, parity, m, reg_count, k);
  prog->ops = kept.v;
  prog->n_ops = kept.n;
  prog->parity_regs = parity;
  prog->k = k;
  prog->m = m;
  prog->mult_count = mults;
  free(needed);
  free(flat.v);
  free(norm.v);
  free(b.items);
  return 0;
}

void lch_free_flat(lch_flat *prog) {
  free(prog->ops);
  free(prog->parity_regs);
  memset(prog, 0, sizeof(*prog));
}

/* build_staged_program, src/fft.rs:393-467 */
int lch_build_staged(size_t k, size_t m, lch_staged *prog) {
  build_what();
  memset(prog, 0, sizeof(*prog));
  if (k == 0 || m == 0 || k + m > 256) return -1;
  size_t n = k + m, t = next_pow2(k);
  int t_levels = ctz(t);
  builder_t b;
  memset(&b, 0, sizeof(b));
  uint16_t base = build_interpolation(&b, k);
  uint16_t *parity = (uint16_t *)calloc(m, sizeof(uint16_t));
  for (size_t position = t; position < n;) {
    int tz = ctz(position);
    size_t alignment = (size_t)1 << (tz < 30 ? tz : 30);
    size_t size = next_pow2(n - position);
    if (alignment < size) size = alignment;
    if (t < size) size = t;
    uint16_t chunk = alloc_regs(&b, size);
    int shift = ctz(size);
    for (size_t j = 0; j < size; j++) {
      for (size_t h = 0; h < t / size; h++) {
        size_t index = h * size + j;
        if (index >= k) continue;
        uint8_t factor = 1;
        for (int level = shift; level < t_levels; level++)
          if (index & ((size_t)1 << level)) factor = or_gf8_mul(factor, WHAT[level][position]);
        if (factor == 0) continue;
        if (factor == 1)
          glue(&b, LCH_XOR, (uint16_t)(chunk + j), (uint16_t)(base + index), 0);
        else
          glue(&b, LCH_MULXOR, (uint16_t)(chunk + j), (uint16_t)(base + index), factor);
      }
    }
    transform(&b, 0, chunk, size, position);
    for (size_t off = 0; off < size; off++) {
      size_t point = position + off;
      if (point >= k && point < n) parity[point - k] = (uint16_t)(chunk + off);
    }
    position += size;
  }
  transform(&b, 0, base, t, 0);
  size_t top = n < t ? n : t;
  size_t in_base = top > k ? top - k : 0;
  for (size_t j = 0; j < in_base; j++) parity[j] = (uint16_t)(base + k + j);

  /* lower_staged, src/fft.rs:472-592 */
  size_t reg_count = b.next_register;
  char *is_zero = (char *)malloc(reg_count);
  char *needs_zero = (char *)calloc(reg_count, 1);
  memset(is_zero, 1, reg_count);
  memset(is_zero, 0, k);
  prog->stages = (lch_stage *)calloc(b.n + 1, sizeof(lch_stage));
  prog->glue = (lch_op *)calloc(b.n + 1, sizeof(lch_op));
  size_t const_cap = 1024;
  prog->consts = (uint8_t *)malloc(const_cap);
  long open_glue = -1;
  for (size_t it = 0; it < b.n; it++) {
    item_t *x = &b.items[it];
    if (!x->is_transform) {
      lch_op op = x->op;
      if (is_zero[op.src]) continue;
      if (is_zero[op.dst]) {
        is_zero[op.dst] = 0;
        op.kind = op.kind == LCH_MULXOR ? LCH_MULCOPY : LCH_COPY;
      }
      if (op.kind == LCH_MULXOR || op.kind == LCH_MULCOPY) prog->mult_count++;
      if (open_glue < 0) open_glue = (long)prog->n_glue;
      prog->glue[prog->n_glue++] = op;
      continue;
    }
    if (open_glue >= 0) {
      lch_stage *s = &prog->stages[prog->n_stages++];
      s->is_transform = 0;
      s->start = (uint32_t)open_glue;
      s->len = (uint32_t)(prog->n_glue - (size_t)open_glue);
      open_glue = -1;
    }
    for (size_t r = x->start; r < (size_t)x->start + x->size; r++) {
      if (is_zero[r]) needs_zero[r] = 1;
      is_zero[r] = 0;
    }
    lch_stage *s = &prog->stages[prog->n_stages++];
    s->is_transform = 1;
    s->inverse = x->inverse;
    s->start = x->start;
    s->size = x->size;
    s->consts_start = (uint32_t)prog->n_consts;
    size_t nn = x->size;
    int levels = ctz(nn);
    prog->boundary_count += 2 * nn;
    for (int li = 0; li < levels; li++) {
      int level = x->inverse ? li : levels - 1 - li;
      size_t stride = (size_t)1 << level;
      for (size_t bb = 0; bb < nn; bb += 2 * stride) {
        uint8_t c = WHAT[level][x->beta ^ bb];
        if (prog->n_consts == const_cap) {
          const_cap *= 2;
          prog->consts = (uint8_t *)realloc(prog->consts, const_cap);
        }
        prog->consts[prog->n_consts++] = c;
        if (c != 0) prog->mult_count += stride;
        prog->xor_count += stride;
      }
    }
  }
  if (open_glue >= 0) {
    lch_stage *s = &prog->stages[prog->n_stages++];
    s->is_transform = 0;
    s->start = (uint32_t)open_glue;
    s->len = (uint32_t)(prog->n_glue - (size_t)open_glue);
  }
  prog->zero_regs = (uint16_t *)calloc(reg_count + 1, sizeof(uint16_t));
  for (size_t r = 0; r < reg_count; r++)
    if (needs_zero[r]) prog->zero_regs[prog->n_zero++] = (uint16_t)r;
  prog->parity_regs = parity;
  prog->register_count = reg_count;
  prog->k = k;
  prog->m = m;
  free(is_zero);
  free(needs_zero);
  free(b.items);
  return 0;
}

void lch_free_staged(lch_staged *prog) {
  free(prog->stages);
  free(prog->glue);
  free(prog->consts);
  free(prog->zero_regs);
  free(prog->parity_regs);
  memset(prog, 0, sizeof(*prog));
}

/* ---- byte interpreters, src/fft.rs:719-817 ---- */

static void run_ops(const lch_op *ops, size_t n, uint8_t *r) {
  for (size_t p = 0; p < n; p++) {
    lch_op op = ops[p];
    switch (op.kind) {
      case LCH_MULXOR: r[op.dst] ^= or_gf8_mul(op.c, r[op.src]); break;
      case LCH_XOR: r[op.dst] ^= r[op.src]; break;
      case LCH_MULCOPY: r[op.dst] = or_gf8_mul(op.c, r[op.src]); break;
      default: r[op.dst] = r[op.src]; break;
    }
  }
}

void lch_run_flat(const lch_flat *prog, const uint8_t *column, uint8_t *parity) {
  uint8_t *r = (uint8_t *)calloc(prog->register_count + 1, 1);
  memcpy(r, column, prog->k);
  run_ops(prog->ops, prog->n_ops, r);
  for (size_t j = 0; j < prog->m; j++) parity[j] = r[prog->parity_regs[j]];
  free(r);
}

/* run_staged_bytes, src/fft.rs:758-817: deliberately stale registers (0xA5) so the
 * zero list is exercised. */
void lch_run_staged(const lch_staged *prog, const uint8_t *column, uint8_t *parity) {
  uint8_t *r = (uint8_t *)malloc(prog->register_count + 1);
  memset(r, 0xA5, prog->register_count + 1);
  memcpy(r, column, prog->k);
  for (size_t z = 0; z < prog->n_zero; z++) r[prog->zero_regs[z]] = 0;
  for (size_t s = 0; s < prog->n_stages; s++) {
    const lch_stage *st = &prog->stages[s];
    if (!st->is_transform) {
      run_ops(prog->glue + st->start, st->len, r);
      continue;
    }
    size_t n = st->size;
    int levels = ctz(n);
    size_t ci = st->consts_start;
    for (int li = 0; li < levels; li++) {
      int level = st->inverse ? li : levels - 1 - li;
      size_t stride = (size_t)1 << level;
      for (size_t bb = 0; bb < n; bb += 2 * stride) {
        uint8_t c = prog->consts[ci++];
        for (size_t i = bb; i < bb + stride; i++) {
          size_t lo = st->start + i, hi = lo + stride;
          if (st->inverse) {
            r[hi] ^= r[lo];
            r[lo] ^= or_gf8_mul(c, r[hi]);
          } else {
            r[lo] ^= or_gf8_mul(c, r[hi]);
            r[hi] ^= r[lo];
          }
        }
      }
    }
  }
  for (size_t j = 0; j < prog->m; j++) parity[j] = r[prog->parity_regs[j]];
  free(r);
}

/* ---- exported wrappers (oracle.h) ---- */

int or_fft_flat_program(size_t k, size_t m, uint32_t *ops, size_t cap, size_t *n_ops,
                        size_t *register_count, uint16_t *parity_regs, size_t *mult_count) {
  lch_flat p;
  if (lch_build_flat(k, m, &p)) return -1;
  *n_ops = p.n_ops;
  *register_count = p.register_count;
  *mult_count = p.mult_count;
  for (size_t j = 0; j < m; j++) parity_regs[j] = p.parity_regs[j];
  size_t lim = p.n_ops < cap ? p.n_ops : cap;
  for (size_t i = 0; i < lim; i++)
    ops[i] = ((uint32_t)p.ops[i].kind << 28) | ((uint32_t)p.ops[i].dst << 18) |
             ((uint32_t)p.ops[i].src << 8) | p.ops[i].c;
  lch_free_flat(&p);
  return 0;
}

int or_fft_staged_program(size_t k, size_t m, size_t *register_count, size_t *mult_count,
                          size_t *xor_count, size_t *n_stages, size_t *n_glue, size_t *n_zero) {
  lch_staged p;
  if (lch_build_staged(k, m, &p)) return -1;
  *register_count = p.register_count;
  *mult_count = p.mult_count;
  *xor_count = p.xor_count;
  *n_stages = p.n_stages;
  *n_glue = p.n_glue;
  *n_zero = p.n_zero;
  lch_free_staged(&p);
  return 0;
}

int or_fft_flat_run(size_t k, size_t m, const uint8_t *column, uint8_t *parity) {
  lch_flat p;
  if (lch_build_flat(k, m, &p)) return -1;
  lch_run_flat(&p, column, parity);
  lch_free_flat(&p);
  return 0;
}

int or_fft_staged_run(size_t k, size_t m, const uint8_t *column, uint8_t *parity) {
  lch_staged p;
  if (lch_build_staged(k, m, &p)) return -1;
  lch_run_staged(&p, column, parity);
  lch_free_staged(&p);
  return 0;
}
