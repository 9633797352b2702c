// Closed-form Lagrange rows over GF((2^8)^2), built on the device.
//
// rows[t][u] = L_u(x_{targets[t]}) for the Lagrange basis on the points x_{nodes[u]},
// with evaluation point x_i = i (src/field.rs:83-86): the systematic generator's parity
// rows (nodes 0..k-1, targets k..n-1) and every decode plan's rows (nodes = survivors,
// targets = missing shards) are this one map (see gf_host.hpp). Three passes:
//   w[u]   = 1 / prod_{v != u} (x_u - x_v)            (one thread per node)
//   ell[t] = prod_v (x_t - x_v)                         (one thread per target)
//   rows   = w[u] * ell[t] / (x_t - x_u), written as the Karatsuba split constants the
//            tower kernel reads (c_lo, c_hi ^ c_lo, c_hi * 32).
// A target that is itself a node yields the unit row.
#pragma once

#include <cstdint>

namespace rsb {

struct Gf8Smem {
  uint8_t lg[256];
  uint8_t ex[512];
};

__device__ __forceinline__ void gf8_smem_init(Gf8Smem &t) {
  if (threadIdx.x == 0) {
    unsigned x = 1;
    for (unsigned i = 0; i < 255; i++) {
      t.ex[i] = (uint8_t)x;
      t.ex[i + 255] = (uint8_t)x;
      t.lg[x] = (uint8_t)i;
      x <<= 1;
      if (x & 0x100) x ^= 0x11d;
    }
    t.ex[510] = t.ex[0];
    t.ex[511] = t.ex[1];
    t.lg[0] = 0;
  }
  __syncthreads();
}

__device__ __forceinline__ uint8_t d_mul8(const Gf8Smem &t, uint8_t a, uint8_t b) {
  return (a && b) ? t.ex[t.lg[a] + t.lg[b]] : 0;
}

// (high*y + low)(high'*y + low') with y^2 = y + 32.
__device__ __forceinline__ uint16_t d_mul16(const Gf8Smem &t, uint16_t a, uint16_t b) {
  uint8_t ah = a >> 8, al = a & 0xff, bh = b >> 8, bl = b & 0xff;
  uint8_t p2 = d_mul8(t, ah, bh);
  uint8_t p1 = d_mul8(t, ah, bl) ^ d_mul8(t, al, bh);
  uint8_t p0 = d_mul8(t, al, bl);
  return (uint16_t)(((p1 ^ p2) << 8) | (uint8_t)(p0 ^ d_mul8(t, p2, 32)));
}

// Inverse through the norm (a != 0).
__device__ __forceinline__ uint16_t d_inv16(const Gf8Smem &t, uint16_t a) {
  uint8_t ah = a >> 8, al = a & 0xff;
  uint16_t conj = (uint16_t)((ah << 8) | (uint8_t)(ah ^ al));
  uint8_t n = (uint8_t)(d_mul16(t, a, conj) & 0xff);
  uint8_t ni = t.ex[255 - t.lg[n]];
  return (uint16_t)((d_mul8(t, conj >> 8, ni) << 8) | d_mul8(t, conj & 0xff, ni));
}

static __global__ void lagrange16_weights(const uint16_t *nodes, uint32_t k, uint16_t *w) {
  __shared__ Gf8Smem t;
  gf8_smem_init(t);
  uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= k) return;
  uint16_t xu = nodes[u], prod = 1;
  for (uint32_t v = 0; v < k; v++)
    if (v != u) prod = d_mul16(t, prod, (uint16_t)(xu ^ nodes[v]));
  w[u] = d_inv16(t, prod);
}

// ell[t] = prod_v (x_t - x_v); hit[t] = index of the node equal to x_t, or k.
static __global__ void lagrange16_ell(const uint16_t *nodes, uint32_t k, const uint16_t *targets, uint32_t n_t,
                                      uint16_t *ell, uint32_t *hit) {
  __shared__ Gf8Smem t;
  gf8_smem_init(t);
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_t) return;
  uint16_t xt = targets[j], prod = 1;
  uint32_t h = k;
  for (uint32_t v = 0; v < k; v++) {
    uint16_t d = (uint16_t)(xt ^ nodes[v]);
    if (!d) h = v;
    prod = d_mul16(t, prod, d);
  }
  ell[j] = prod;
  hit[j] = h;
}

__device__ __forceinline__ uint32_t split16_dev(const Gf8Smem &t, uint16_t c) {
  uint8_t hi = c >> 8, lo = c & 0xff;
  return (uint32_t)lo | ((uint32_t)(uint8_t)(hi ^ lo) << 8) | ((uint32_t)d_mul8(t, hi, 32) << 16);
}

// One thread per (target, node) entry; out as split constants, plain rows optional.
static __global__ void lagrange16_rows(const uint16_t *nodes, uint32_t k, const uint16_t *targets, uint32_t n_t,
                                       const uint16_t *w, const uint16_t *ell, const uint32_t *hit, uint32_t *split,
                                       uint16_t *plain) {
  __shared__ Gf8Smem t;
  gf8_smem_init(t);
  uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (uint64_t)n_t * k) return;
  uint32_t j = (uint32_t)(e / k), u = (uint32_t)(e % k);
  uint16_t v;
  if (hit[j] < k) {
    v = (uint16_t)(hit[j] == u);
  } else {
    uint16_t d = (uint16_t)(targets[j] ^ nodes[u]);
    v = d_mul16(t, d_mul16(t, w[u], ell[j]), d_inv16(t, d));
  }
  split[e] = split16_dev(t, v);
  if (plain) plain[e] = v;
}

}  // namespace rsb
