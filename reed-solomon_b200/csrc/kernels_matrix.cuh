// Matrix-route kernels: out[j] = sum_i coeff[j][i] * in[i] over byte columns.
//
// GF(2^8) multiply-by-constant is GF(2)-linear in the input byte:
//   c * x = XOR_b  bit_b(x) * (c * 2^b).
// Each 32-bit word carries 4 byte columns. For every input word the kernel expands
// bit b of each byte into a 0x00/0xFF byte mask (one shift + one sign-replicating
// PRMT); a product is then 8 AND-XOR (LOP3) operations against the constants
// c * 2^b replicated into all four bytes. The masks are computed once per input and
// reused by every output row in the register tile, and every output row of the tile
// accumulates in registers, so each input byte is read once per tile of OUT_TILE
// outputs. This is the kernel behind RowTables::apply
// (src/gf/tables.rs:162-191 -> src/gf/x86_fused.rs:598-681) and the reconstruct
// applies (src/reedsolomon.rs:829-891).
#pragma once

#include <cstdint>

#include "runtime.hpp"

namespace rsb {

constexpr int kThreads = 256;
constexpr int kBytesPerThread = 16;
constexpr int kTileBytes = kThreads * kBytesPerThread;  // 4 KiB of columns per CTA
constexpr uint32_t kRowChunk = 32;    // GF(2^8) output rows per CTA (grid.z), default tile
// Tile shapes of the matrix kernel: parity rows accumulated per thread (registers) and
// output rows per CTA (grid.z chunk). Chosen per call by the autotuner.
struct MatrixVariant {
  int out_tile, row_chunk;
};
constexpr MatrixVariant kMatrixVariants[] = {{8, 32}, {4, 16}, {8, 64}, {16, 64}};
constexpr int kMatrixVariantCount = sizeof(kMatrixVariants) / sizeof(kMatrixVariants[0]);
inline int &matrix_variant() {
  static int v = 0;
  return v;
}
constexpr uint32_t kRowChunk16 = 64;  // tower output rows per CTA (grid.z)

// Addressing of one launch: either pointer tables passed by value as a kernel
// parameter (one stripe, at most 256 inputs and outputs) or strided rows (many
// stripes laid out alike).
template <bool PTRS>
struct PtrTableT {
  const uint8_t *in[256];
  uint8_t *out[256];
};
template <>
struct PtrTableT<false> {
  uint8_t unused;
};
using PtrTable = PtrTableT<true>;

struct ApplyArgs {
  // Strided form (used when ptrs == nullptr): stripe s, row i.
  const uint8_t *in_base;
  uint64_t in_row_stride, in_stripe_stride;
  uint8_t *out_base;
  uint64_t out_row_stride, out_stripe_stride;
  // Coefficients, rows x k row-major per stripe (stride 0 = shared by all stripes).
  const uint8_t *coeffs;
  uint64_t coeff_stripe_stride;
  // Per-stripe row count override (reconstruct batches); nullptr = `rows`.
  const uint16_t *rows_per_stripe;
  // Per-stripe input / output row index maps for strided reconstruct batches:
  // in_map[s*k + t] = stripe row read as input t, out_map[s*rows + j] = row written.
  const uint16_t *in_map, *out_map;
  uint32_t k, rows;
  uint64_t len;
  uint32_t n_stripes;
  uint32_t *mismatch;  // verify mode: set to 1 on any difference
};

__device__ __forceinline__ uint32_t sign_bytes(uint32_t x) {
  uint32_t r;
  asm("prmt.b32 %0, %1, 0, 0xBA98;" : "=r"(r) : "r"(x));
  return r;
}

// Byte masks of bit b of each byte of x, b = 0..7.
__device__ __forceinline__ void bit_masks(uint32_t x, uint32_t m[8]) {
#pragma unroll
  for (int b = 0; b < 7; b++) m[b] = sign_bytes(x << (7 - b));
  m[7] = sign_bytes(x);
}

__device__ __forceinline__ uint8_t xtime8(uint8_t v) {
  return (uint8_t)((v << 1) ^ ((v & 0x80) ? 0x1d : 0));
}

// R[c*8 + b] = (c * 2^b) replicated into 4 bytes, for all 256 constants.
__device__ __forceinline__ void fill_rtab(uint32_t *R) {
  for (int c = threadIdx.x; c < 256; c += blockDim.x) {
    uint8_t v = (uint8_t)c;
#pragma unroll
    for (int b = 0; b < 8; b++) {
      R[c * 8 + b] = 0x01010101u * v;
      v = xtime8(v);
    }
  }
}

__device__ __forceinline__ bool aligned16(const void *p) {
  return ((uintptr_t)p & 15u) == 0;
}

__device__ __forceinline__ uint4 load_cols(const uint8_t *p, uint64_t remain) {
  if (remain >= 16 && aligned16(p)) return __ldg(reinterpret_cast<const uint4 *>(p));
  uint32_t w[4] = {0, 0, 0, 0};
  int n = remain < 16 ? (int)remain : 16;
  for (int t = 0; t < n; t++) w[t >> 2] |= (uint32_t)p[t] << (8 * (t & 3));
  return make_uint4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ void store_cols(uint8_t *p, uint64_t remain, uint4 v) {
  if (remain >= 16 && aligned16(p)) {
    *reinterpret_cast<uint4 *>(p) = v;
    return;
  }
  uint32_t w[4] = {v.x, v.y, v.z, v.w};
  int n = remain < 16 ? (int)remain : 16;
  for (int t = 0; t < n; t++) p[t] = (uint8_t)(w[t >> 2] >> (8 * (t & 3)));
}

__device__ __forceinline__ bool equal_cols(const uint8_t *p, uint64_t remain, uint4 v) {
  uint4 have = load_cols(p, remain);
  if (remain < 16) {
    // Compare only the bytes in range: load_cols zero-fills the rest, so zero the
    // same bytes of v.
    uint32_t w[4] = {v.x, v.y, v.z, v.w};
    for (int t = (int)remain; t < 16; t++) w[t >> 2] &= ~(0xffu << (8 * (t & 3)));
    v = make_uint4(w[0], w[1], w[2], w[3]);
  }
  return have.x == v.x && have.y == v.y && have.z == v.z && have.w == v.w;
}

template <bool PTRS>
__device__ __forceinline__ const uint8_t *in_row(const ApplyArgs &a, const PtrTableT<PTRS> &pt,
                                                 uint32_t s, uint32_t i) {
  if constexpr (PTRS) return pt.in[i];
  uint32_t r = a.in_map ? a.in_map[(uint64_t)s * a.k + i] : i;
  return a.in_base + s * a.in_stripe_stride + r * a.in_row_stride;
}

template <bool PTRS>
__device__ __forceinline__ uint8_t *out_row(const ApplyArgs &a, const PtrTableT<PTRS> &pt, uint32_t s,
                                            uint32_t j) {
  if constexpr (PTRS) return pt.out[j];
  uint32_t r = a.out_map ? a.out_map[(uint64_t)s * a.rows + j] : j;
  return a.out_base + s * a.out_stripe_stride + r * a.out_row_stride;
}

// grid.x: column tiles of kTileBytes; grid.y: stripes (looped when more than grid.y).
// Dynamic shared memory: 8 KiB constant table + rows*k coefficient bytes.
template <int OUT_TILE, int ROW_CHUNK, bool PTRS, bool VERIFY>
__global__ void __launch_bounds__(kThreads)
    gf8_matrix_kernel(const ApplyArgs a, const __grid_constant__ PtrTableT<PTRS> pt) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t *R = smem;                                    // 2048 words
  uint8_t *C = reinterpret_cast<uint8_t *>(smem + 2048);  // rows * k bytes
  fill_rtab(R);
  const uint64_t col = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) * kBytesPerThread;
  const uint32_t k = a.k;
  for (uint32_t s = blockIdx.y; s < a.n_stripes; s += gridDim.y) {
    const uint32_t rows = a.rows_per_stripe ? a.rows_per_stripe[s] : a.rows;
    const uint8_t *cs = a.coeffs + s * a.coeff_stripe_stride;
    for (uint32_t t = threadIdx.x; t < rows * k; t += kThreads) C[t] = cs[t];
    __syncthreads();
    if (col < a.len) {
      const uint64_t remain = a.len - col;
      // grid.z splits the output rows into chunks of ROW_CHUNK.
      const uint32_t g_end = min(rows, (blockIdx.z + 1) * ROW_CHUNK);
      for (uint32_t g = blockIdx.z * ROW_CHUNK; g < g_end; g += OUT_TILE) {
        const uint32_t live = g_end - g;
        uint32_t acc[OUT_TILE][4];
#pragma unroll
        for (int o = 0; o < OUT_TILE; o++) acc[o][0] = acc[o][1] = acc[o][2] = acc[o][3] = 0;
        for (uint32_t i = 0; i < k; i++) {
          uint4 x = load_cols(in_row<PTRS>(a, pt, s, i) + col, remain);
          uint32_t m[4][8];
          bit_masks(x.x, m[0]);
          bit_masks(x.y, m[1]);
          bit_masks(x.z, m[2]);
          bit_masks(x.w, m[3]);
#pragma unroll
          for (int o = 0; o < OUT_TILE; o++) {
            if (o < (int)live) {
              const uint4 *r4 = reinterpret_cast<const uint4 *>(R + 8 * C[(g + o) * k + i]);
              uint4 r0 = r4[0], r1 = r4[1];
              uint32_t r[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
#pragma unroll
              for (int w = 0; w < 4; w++)
#pragma unroll
                for (int b = 0; b < 8; b++) acc[o][w] ^= m[w][b] & r[b];
            }
          }
        }
#pragma unroll
        for (int o = 0; o < OUT_TILE; o++) {
          if (o < (int)live) {
            uint4 v = make_uint4(acc[o][0], acc[o][1], acc[o][2], acc[o][3]);
            uint8_t *dst = out_row<PTRS>(a, pt, s, g + o) + col;
            if (VERIFY) {
              if (!equal_cols(dst, remain, v)) atomicOr(a.mismatch, 1u);
            } else {
              store_cols(dst, remain, v);
            }
          }
        }
      }
    }
    __syncthreads();
  }
}

// gf::mul_slice(_xor), src/gf/mod.rs:69-85: out (^)= c * in over n bytes.
static __global__ void __launch_bounds__(kThreads)
    gf8_mul_slice_kernel(uint8_t *out, const uint8_t *in, uint64_t n, uint8_t c, int xor_into) {
  uint32_t r[8];
  uint8_t v = c;
#pragma unroll
  for (int b = 0; b < 8; b++) {
    r[b] = 0x01010101u * v;
    v = xtime8(v);
  }
  for (uint64_t col = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) * 16; col < n;
       col += (uint64_t)gridDim.x * kThreads * 16) {
    uint64_t remain = n - col;
    uint4 x = load_cols(in + col, remain);
    uint32_t xs[4] = {x.x, x.y, x.z, x.w}, y[4];
#pragma unroll
    for (int w = 0; w < 4; w++) {
      uint32_t m[8];
      bit_masks(xs[w], m);
      y[w] = 0;
#pragma unroll
      for (int b = 0; b < 8; b++) y[w] ^= m[b] & r[b];
    }
    if (xor_into) {
      uint4 o = load_cols(out + col, remain);
      y[0] ^= o.x;
      y[1] ^= o.y;
      y[2] ^= o.z;
      y[3] ^= o.w;
    }
    store_cols(out + col, remain, make_uint4(y[0], y[1], y[2], y[3]));
  }
}

// ---------------------------------------------------------------------------
// GF((2^8)^2) tower, split-plane wire. Multiply-by-c on (high, low) in Karatsuba
// form (src/reedsolomon16.rs:61-94, src/gf/tower_x86.rs:10-16):
//   t0 = c_lo * lo, t1 = (c_hi ^ c_lo) * (lo ^ hi), t2 = (c_hi * 32) * hi,
//   out_lo ^= t0 ^ t2, out_hi ^= t0 ^ t1.
// Coefficients arrive pre-split as u32 (k0 | k1 << 8 | k2 << 16).
// A thread owns 8 symbols: 8 low-plane bytes and the matching 8 high-plane bytes.
// ---------------------------------------------------------------------------
struct Apply16Args {
  const uint8_t *const *in_ptrs;  // device table [s * k + i] (nullptr: strided)
  uint8_t *const *out_ptrs;       // device table [s * rows + j]
  const uint8_t *in_base;
  uint64_t in_row_stride, in_stripe_stride;
  uint8_t *out_base;
  uint64_t out_row_stride, out_stripe_stride;
  const uint32_t *coeffs;  // rows x k split constants
  uint32_t k, rows;
  uint64_t n_sym;  // symbols per shard (shard bytes / 2)
  uint32_t n_stripes;
  uint32_t *mismatch;
  uint32_t row_chunk;  // output rows per CTA (grid.z), set by gf16_launch_shape
};

// Launch shape of gf16_matrix_kernel: CTAs as wide as the shard needs (8 symbols per
// thread, 32..256 threads), and output-row chunks halved from 64 down to 4 until the
// grid has two CTAs per SM, so single stripes of short shards still fill the GPU.
inline void gf16_launch_shape(Apply16Args &a, int sms, dim3 &grid, unsigned &threads) {
  const uint64_t need = (a.n_sym + 7) / 8;
  threads = (unsigned)std::min<uint64_t>(kThreads, std::max<uint64_t>(32, (need + 31) / 32 * 32));
  const uint64_t tiles = (a.n_sym + threads * 8ull - 1) / (threads * 8ull);
  const uint32_t stripes = std::min<uint32_t>(a.n_stripes, 65535);
  uint32_t chunk = kRowChunk16;
  while (chunk > 4 && tiles * stripes * ((a.rows + chunk - 1) / chunk) < 2ull * sms) chunk /= 2;
  a.row_chunk = chunk;
  grid = dim3((unsigned)tiles, stripes, (a.rows + chunk - 1) / chunk);
}

__device__ __forceinline__ uint2 load_sym8(const uint8_t *p, uint64_t remain) {
  if (remain >= 8 && (((uintptr_t)p & 7u) == 0)) return *reinterpret_cast<const uint2 *>(p);
  uint32_t w[2] = {0, 0};
  int n = remain < 8 ? (int)remain : 8;
  for (int t = 0; t < n; t++) w[t >> 2] |= (uint32_t)p[t] << (8 * (t & 3));
  return make_uint2(w[0], w[1]);
}

__device__ __forceinline__ void store_sym8(uint8_t *p, uint64_t remain, uint32_t w0, uint32_t w1) {
  if (remain >= 8 && (((uintptr_t)p & 7u) == 0)) {
    *reinterpret_cast<uint2 *>(p) = make_uint2(w0, w1);
    return;
  }
  uint32_t w[2] = {w0, w1};
  int n = remain < 8 ? (int)remain : 8;
  for (int t = 0; t < n; t++) p[t] = (uint8_t)(w[t >> 2] >> (8 * (t & 3)));
}

__device__ __forceinline__ bool equal_sym8(const uint8_t *p, uint64_t remain, uint32_t w0,
                                           uint32_t w1) {
  uint2 h = load_sym8(p, remain);
  if (remain < 8) {
    uint32_t w[2] = {w0, w1};
    for (int t = (int)remain; t < 8; t++) w[t >> 2] &= ~(0xffu << (8 * (t & 3)));
    w0 = w[0];
    w1 = w[1];
  }
  return h.x == w0 && h.y == w1;
}

template <int OUT_TILE, bool VERIFY>
__global__ void __launch_bounds__(kThreads) gf16_matrix_kernel(const Apply16Args a) {
  __shared__ __align__(16) uint32_t R[2048];
  fill_rtab(R);
  __syncthreads();
  const uint64_t sym = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 8;
  const uint32_t k = a.k, chunk = a.row_chunk;
  for (uint32_t s = blockIdx.y; s < a.n_stripes; s += gridDim.y) {
    if (sym >= a.n_sym) continue;
    const uint64_t remain = a.n_sym - sym;
    const uint32_t g_end = min(a.rows, (blockIdx.z + 1) * chunk);
    for (uint32_t g = blockIdx.z * chunk; g < g_end; g += OUT_TILE) {
      const uint32_t live = g_end - g;
      uint32_t lo_acc[OUT_TILE][2], hi_acc[OUT_TILE][2];
#pragma unroll
      for (int o = 0; o < OUT_TILE; o++) lo_acc[o][0] = lo_acc[o][1] = hi_acc[o][0] = hi_acc[o][1] = 0;
      for (uint32_t i = 0; i < k; i++) {
        const uint8_t *row = a.in_ptrs ? a.in_ptrs[(uint64_t)s * k + i]
                                       : a.in_base + s * a.in_stripe_stride + i * a.in_row_stride;
        uint2 lo = load_sym8(row + sym, remain);
        uint2 hi = load_sym8(row + a.n_sym + sym, remain);
        uint32_t ml[2][8], mh[2][8], mm[2][8];
        bit_masks(lo.x, ml[0]);
        bit_masks(lo.y, ml[1]);
        bit_masks(hi.x, mh[0]);
        bit_masks(hi.y, mh[1]);
        bit_masks(lo.x ^ hi.x, mm[0]);
        bit_masks(lo.y ^ hi.y, mm[1]);
#pragma unroll
        for (int o = 0; o < OUT_TILE; o++) {
          if (o < (int)live) {
            uint32_t cc = a.coeffs[(uint64_t)(g + o) * k + i];
            const uint32_t *r0 = R + 8 * (cc & 0xff);
            const uint32_t *r1 = R + 8 * ((cc >> 8) & 0xff);
            const uint32_t *r2 = R + 8 * ((cc >> 16) & 0xff);
#pragma unroll
            for (int w = 0; w < 2; w++) {
              uint32_t t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
              for (int b = 0; b < 8; b++) {
                t0 ^= ml[w][b] & r0[b];
                t1 ^= mm[w][b] & r1[b];
                t2 ^= mh[w][b] & r2[b];
              }
              lo_acc[o][w] ^= t0 ^ t2;
              hi_acc[o][w] ^= t0 ^ t1;
            }
          }
        }
      }
#pragma unroll
      for (int o = 0; o < OUT_TILE; o++) {
        if (o < (int)live) {
          uint8_t *dst = a.out_ptrs ? a.out_ptrs[(uint64_t)s * a.rows + g + o]
                                    : a.out_base + s * a.out_stripe_stride + (g + o) * a.out_row_stride;
          if (VERIFY) {
            if (!equal_sym8(dst + sym, remain, lo_acc[o][0], lo_acc[o][1]) ||
                !equal_sym8(dst + a.n_sym + sym, remain, hi_acc[o][0], hi_acc[o][1]))
              atomicOr(a.mismatch, 1u);
          } else {
            store_sym8(dst + sym, remain, lo_acc[o][0], lo_acc[o][1]);
            store_sym8(dst + a.n_sym + sym, remain, hi_acc[o][0], hi_acc[o][1]);
          }
        }
      }
    }
  }
}

}  // namespace rsb
