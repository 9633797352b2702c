// Decode-plan construction on the device for the GF(2^8) coder.
//
// One CTA per erasure pattern inverts the k x k survivor matrix (generator rows of
// the first k present shards, src/reedsolomon.rs:539-566) by Gauss-Jordan in shared
// memory, pivoting on the first nonzero entry at or below the diagonal as
// src/matrix.rs:123-168 does. The inverse of a nonsingular matrix is unique, so
// clearing above and below each pivot in one sweep yields the reference's bytes.
// It then writes the composed plan rows, one per missing shard, in the order the
// kernels apply them: missing data rows are inverse rows (src/reedsolomon.rs:568-573);
// a missing parity row is its generator row times the inverse, which maps survivors
// straight to that parity (the reference's second apply over recovered data,
// src/reedsolomon.rs:877-889, composed into one linear map).
#pragma once

#include <cstdint>

namespace rsb {

struct PlanArgs {
  const uint8_t *gen;          // m x k parity rows of the systematic generator
  uint32_t k, m;
  const uint16_t *survivors;   // [p * k] survivor shard indexes, ascending
  const uint16_t *targets;     // [p * max_rows] missing indexes: data asc, then parity asc
  const uint16_t *n_targets;   // [p]
  uint32_t max_rows;
  uint8_t *out;                // [p * max_rows * k]
  int *status;                 // [p]: 0, or 14 (SingularMatrix)
};

__device__ __forceinline__ uint8_t gmul_tab(const uint8_t *lg, const uint8_t *ex, uint8_t a,
                                            uint8_t b) {
  return (a && b) ? ex[lg[a] + lg[b]] : 0;
}

// Dynamic shared memory layout, each region on a 16-byte boundary: 768 B of log/exp
// tables; the e x 2e matrix [M | I] (e <= k); the e x (k - e) product R; the missing
// data indexes md, the parity survivors par and the data-survivor flags (k each); e
// pivot factors; the pivot slot and e.
struct PlanSmem {
  uint32_t a_off, r_off, md_off, par_off, mark_off, f_off, piv_off, total;
};
__host__ __device__ inline PlanSmem plan_smem(uint32_t k) {
  auto up = [](uint32_t x) { return (x + 15u) & ~15u; };
  PlanSmem s;
  s.a_off = 768;
  s.r_off = up(s.a_off + 2 * k * k);
  s.md_off = up(s.r_off + (k / 2) * ((k + 1) / 2));  // e (k - e) <= k^2 / 4
  s.par_off = up(s.md_off + k);
  s.mark_off = up(s.par_off + k);
  s.f_off = up(s.mark_off + k);
  s.piv_off = up(s.f_off + k);
  s.total = s.piv_off + 16;
  return s;
}

// Bitwise GF(2^8) product (0x11d), for the table set-up.
__device__ __forceinline__ uint32_t gf8_mul_bits(uint32_t a, uint32_t b) {
  uint32_t r = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    if (b & 1) r ^= a;
    a = (a << 1) ^ ((a & 0x80) ? 0x11d : 0);
    b >>= 1;
  }
  return r & 0xff;
}

// The survivor matrix S (k x k) is systematic: its rows for the k - e present data
// shards dp are unit vectors, the other e rows are the generator rows g_j of the first
// e present parity shards par. With md the e missing data indexes, M = g_par[md] (e x e)
// and N = g_par[dp] (e x (k - e)), the survivors' values v satisfy
// M x_md = v_par + N v_dp, so x_md = M^-1 v_par + (M^-1 N) v_dp: the rows of S^-1 for
// the missing data are [R = M^-1 N | M^-1] over the survivor positions (data survivors
// first, ascending, then the parity survivors), and a missing parity row g_y gives
// g_y[dp] + g_y[md] R on the data positions and g_y[md] M^-1 on the parity positions.
// Only the e x e block is inverted (Gauss-Jordan in shared memory, as src/matrix.rs
// does for the whole matrix; the inverse is unique, so the bytes equal the full
// inversion's), and M is singular exactly when S is.
static __global__ void __launch_bounds__(256) gf8_plan_kernel(const PlanArgs a) {
  extern __shared__ __align__(16) uint8_t sm[];
  uint8_t *lg = sm;          // 256
  uint8_t *ex = sm + 256;    // 512
  const uint32_t k = a.k;
  const PlanSmem lay = plan_smem(k);
  uint8_t *A = sm + lay.a_off;
  uint8_t *R = sm + lay.r_off;
  uint8_t *md = sm + lay.md_off;
  uint8_t *par = sm + lay.par_off;
  uint8_t *mark = sm + lay.mark_off;
  uint8_t *f = sm + lay.f_off;
  int *piv = reinterpret_cast<int *>(sm + lay.piv_off);
  const uint32_t p = blockIdx.x;
  const uint16_t *surv = a.survivors + (uint64_t)p * k;
  // Tables: ex[i] = 2^i (i < 510, period 255), lg[2^i] = i; one entry per thread.
  for (uint32_t i = threadIdx.x; i < 255; i += blockDim.x) {
    uint32_t x = 1, base = 2, e = i;
    while (e) {
      if (e & 1) x = gf8_mul_bits(x, base);
      base = gf8_mul_bits(base, base);
      e >>= 1;
    }
    ex[i] = ex[i + 255] = (uint8_t)x;
    lg[x] = (uint8_t)i;
  }
  if (threadIdx.x == 0) {
    ex[510] = ex[0];
    ex[511] = ex[1];
    lg[0] = 0;
  }
  for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) mark[i] = 0;
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < k; t += blockDim.x)
    if (surv[t] < k) mark[surv[t]] = 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t e = 0;
    for (uint32_t i = 0; i < k; i++)
      if (!mark[i]) md[e++] = (uint8_t)i;
    // The last e survivors are parity shards (survivors ascend); anything else is an
    // invalid list, reported like a singular matrix rather than read past the generator.
    int ok = 1;
    for (uint32_t t = k - e; t < k; t++) {
      const uint32_t j = (uint32_t)surv[t] - k;
      if (surv[t] < k || j >= a.m) ok = 0;
      par[t - (k - e)] = (uint8_t)(ok ? j : 0);
    }
    piv[1] = ok ? (int)e : -1;
  }
  __syncthreads();
  if (piv[1] < 0) {
    if (threadIdx.x == 0) a.status[p] = 14;
    return;  // uniform
  }
  const uint32_t e = (uint32_t)piv[1], d = k - e, w = 2 * e;
  // [M | I]
  for (uint32_t t = threadIdx.x; t < e * w; t += blockDim.x) {
    const uint32_t r = t / w, c = t % w;
    A[t] = c < e ? a.gen[(uint64_t)par[r] * k + md[c]] : (uint8_t)(c - e == r);
  }
  __syncthreads();
  for (uint32_t r = 0; r < e; r++) {
    if (threadIdx.x == 0) {
      int found = -1;
      for (uint32_t q = r; q < e; q++)
        if (A[q * w + r]) {
          found = (int)q;
          break;
        }
      *piv = found;
    }
    __syncthreads();
    const int pr = *piv;
    if (pr < 0) {
      if (threadIdx.x == 0) a.status[p] = 14;
      return;  // uniform: every thread read the same pivot slot
    }
    if ((uint32_t)pr != r)
      for (uint32_t c = threadIdx.x; c < w; c += blockDim.x) {
        uint8_t t0 = A[r * w + c];
        A[r * w + c] = A[pr * w + c];
        A[pr * w + c] = t0;
      }
    __syncthreads();
    const uint8_t inv = ex[255 - lg[A[r * w + r]]];
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < w; c += blockDim.x) A[r * w + c] = gmul_tab(lg, ex, A[r * w + c], inv);
    for (uint32_t q = threadIdx.x; q < e; q += blockDim.x) f[q] = 0;
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < e; q += blockDim.x)
      if (q != r) f[q] = A[q * w + r];
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < e * w; t += blockDim.x) {
      uint32_t q = t / w, c = t % w;
      if (f[q]) A[t] ^= gmul_tab(lg, ex, f[q], A[r * w + c]);
    }
    __syncthreads();
  }
  // R = M^-1 N (e x d); N[b][i] = g_par[b][dp_i], dp_i = surv[i] for i < d.
  for (uint32_t t = threadIdx.x; t < e * d; t += blockDim.x) {
    const uint32_t x = t / d, i = t % d, col = surv[i];
    uint8_t v = 0;
    for (uint32_t b = 0; b < e; b++) v ^= gmul_tab(lg, ex, A[x * w + e + b], a.gen[(uint64_t)par[b] * k + col]);
    R[t] = v;
  }
  __syncthreads();
  // Composed rows over the survivor positions u (data survivors, then parity survivors).
  const uint32_t nt = a.n_targets[p];
  const uint16_t *tg = a.targets + (uint64_t)p * a.max_rows;
  uint8_t *out = a.out + (uint64_t)p * a.max_rows * k;
  for (uint32_t t = threadIdx.x; t < nt * k; t += blockDim.x) {
    const uint32_t j = t / k, u = t % k, x = tg[j];
    uint8_t v;
    if (x < k) {
      uint32_t xi = 0;  // position of x in md
      while (xi < e && md[xi] != x) xi++;
      if (xi == e)  // x is a data survivor: its row picks its own position
        v = (uint8_t)(u < d && surv[u] == x);
      else
        v = u < d ? R[xi * d + u] : A[xi * w + e + (u - d)];
    } else {
      const uint8_t *g = a.gen + (uint64_t)(x - k) * k;
      v = u < d ? g[surv[u]] : 0;
      for (uint32_t b = 0; b < e; b++)
        v ^= gmul_tab(lg, ex, g[md[b]], u < d ? R[b * d + u] : A[b * w + e + (u - d)]);
    }
    out[t] = v;
  }
  if (threadIdx.x == 0) a.status[p] = 0;
}

}  // namespace rsb
