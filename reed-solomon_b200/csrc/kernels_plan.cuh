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

// Dynamic shared memory layout: 768 B of log/exp tables, the k x 2k matrix, k pivot
// factors and the pivot slot, each region starting on a 16-byte boundary.
struct PlanSmem {
  uint32_t f_off, piv_off, total;
};
__host__ __device__ inline PlanSmem plan_smem(uint32_t k) {
  auto up = [](uint32_t x) { return (x + 15u) & ~15u; };
  PlanSmem s;
  s.f_off = up(768 + 2 * k * k);
  s.piv_off = up(s.f_off + k);
  s.total = s.piv_off + 16;
  return s;
}

static __global__ void __launch_bounds__(256) gf8_plan_kernel(const PlanArgs a) {
  extern __shared__ __align__(16) uint8_t sm[];
  uint8_t *lg = sm;          // 256
  uint8_t *ex = sm + 256;    // 512
  const uint32_t k = a.k, w = 2 * k;
  const PlanSmem lay = plan_smem(k);
  uint8_t *A = sm + 768;     // k x 2k
  uint8_t *f = sm + lay.f_off;  // k factors
  int *piv = reinterpret_cast<int *>(sm + lay.piv_off);
  const uint32_t p = blockIdx.x;
  if (threadIdx.x == 0) {
    unsigned x = 1;
    for (unsigned i = 0; i < 255; i++) {
      ex[i] = (uint8_t)x;
      ex[i + 255] = (uint8_t)x;
      lg[x] = (uint8_t)i;
      x <<= 1;
      if (x & 0x100) x ^= 0x11d;
    }
    ex[510] = ex[0];
    ex[511] = ex[1];
    lg[0] = 0;
  }
  const uint16_t *surv = a.survivors + (uint64_t)p * k;
  for (uint32_t t = threadIdx.x; t < k * w; t += blockDim.x) {
    uint32_t r = t / w, c = t % w;
    uint32_t row = surv[r];
    uint8_t v;
    if (c < k)
      v = row < k ? (uint8_t)(row == c) : a.gen[(uint64_t)(row - k) * k + c];
    else
      v = (uint8_t)(c - k == r);
    A[t] = v;
  }
  __syncthreads();
  for (uint32_t r = 0; r < k; r++) {
    if (threadIdx.x == 0) {
      int found = -1;
      for (uint32_t q = r; q < k; q++)
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
    for (uint32_t q = threadIdx.x; q < k; q += blockDim.x) f[q] = 0;
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < k; q += blockDim.x)
      if (q != r) f[q] = A[q * w + r];
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < k * w; t += blockDim.x) {
      uint32_t q = t / w, c = t % w;
      if (f[q]) A[t] ^= gmul_tab(lg, ex, f[q], A[r * w + c]);
    }
    __syncthreads();
  }
  // Composed rows.
  const uint32_t nt = a.n_targets[p];
  const uint16_t *tg = a.targets + (uint64_t)p * a.max_rows;
  uint8_t *out = a.out + (uint64_t)p * a.max_rows * k;
  for (uint32_t t = threadIdx.x; t < nt * k; t += blockDim.x) {
    uint32_t j = t / k, u = t % k;
    uint32_t x = tg[j];
    uint8_t v;
    if (x < k) {
      v = A[x * w + k + u];
    } else {
      const uint8_t *g = a.gen + (uint64_t)(x - k) * k;
      v = 0;
      for (uint32_t i = 0; i < k; i++) v ^= gmul_tab(lg, ex, g[i], A[i * w + k + u]);
    }
    out[t] = v;
  }
  if (threadIdx.x == 0) a.status[p] = 0;
}

}  // namespace rsb
