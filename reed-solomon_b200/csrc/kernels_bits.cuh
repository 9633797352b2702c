// Bitsliced GF(2^8) products by constants known only at run time but the same for every
// lane of a warp (a butterfly's constant, a stripe's decode coefficient), and the
// bitsliced matrix kernel built on them.
#pragma once

#include <cstdint>

#include "kernels_batch.cuh"
#include "kernels_fft.cuh"

namespace rsb {

// ---- runtime constants through compile-time networks ----
// A butterfly constant is known only at run time, but it is the same for every lane of
// the warp, so each of its three GF(2^8) Karatsuba factors k can select a compiled XOR
// network instead of being applied as 64 masked XORs: k * x = (k & 15) * x + (k & 0xF0) * x,
// and (k & 0xF0) = (k >> 4) * alpha^4 needs no reduction, so both halves are one of 16
// compile-time constants applied to x itself (kernels_fft.cuh mul_set / mul_acc, about
// 10 LOP3 each against 64 masked LOP3 and 16 mask loads). The two switches live in one
// out-of-line function with its operands in registers, so the networks exist once.
struct Planes8 {
  uint32_t v[8];
};

template <int J>
__device__ __forceinline__ void nib_lo(Planes8 &t, const Planes8 &x) {
  fftc::mul_set<(uint8_t)J>(*reinterpret_cast<fftc::Reg *>(t.v), *reinterpret_cast<const fftc::Reg *>(x.v));
}
template <int J>
__device__ __forceinline__ void nib_hi(Planes8 &t, const Planes8 &x) {
  fftc::mul_acc<(uint8_t)(J << 4)>(*reinterpret_cast<fftc::Reg *>(t.v), *reinterpret_cast<const fftc::Reg *>(x.v));
}

// k * x for a warp-uniform byte k, inlined at each use.
__device__ __forceinline__ Planes8 mul8_rt_inl(const Planes8 &x, uint32_t k) {
  Planes8 t;
  switch (k & 15) {
#define RSB_NIB(j)   \
  case j:            \
    nib_lo<j>(t, x); \
    break;
    RSB_NIB(0) RSB_NIB(1) RSB_NIB(2) RSB_NIB(3) RSB_NIB(4) RSB_NIB(5) RSB_NIB(6) RSB_NIB(7)
    RSB_NIB(8) RSB_NIB(9) RSB_NIB(10) RSB_NIB(11) RSB_NIB(12) RSB_NIB(13) RSB_NIB(14) RSB_NIB(15)
#undef RSB_NIB
  }
  switch ((k >> 4) & 15) {
#define RSB_NIB(j)   \
  case j:            \
    nib_hi<j>(t, x); \
    break;
    RSB_NIB(0) RSB_NIB(1) RSB_NIB(2) RSB_NIB(3) RSB_NIB(4) RSB_NIB(5) RSB_NIB(6) RSB_NIB(7)
    RSB_NIB(8) RSB_NIB(9) RSB_NIB(10) RSB_NIB(11) RSB_NIB(12) RSB_NIB(13) RSB_NIB(14) RSB_NIB(15)
#undef RSB_NIB
  }
  return t;
}

// The same out of line: one copy of the networks for every caller.
static __device__ __noinline__ Planes8 mul8_rt(Planes8 x, uint32_t k) { return mul8_rt_inl(x, k); }

struct Planes16 {
  Planes8 a, b;
};

// k0 * x and k1 * x in one out-of-line call.
static __device__ __noinline__ Planes16 mul8x2_rt(Planes8 x, uint32_t k0, uint32_t k1) {
  return Planes16{mul8_rt_inl(x, k0), mul8_rt_inl(x, k1)};
}

// 32 bytes at p (remain of them valid, zeros after) and their store, out of line for the
// partial and unaligned cases so the callers' register arrays are never indexed at run
// time.
static __device__ __noinline__ Planes8 load32_any(const uint8_t *p, uint64_t remain) {
  Planes8 x;
  load32(p, remain, x.v);
  return x;
}
static __device__ __noinline__ void store32_rows(uint8_t *p, uint64_t remain, Planes8 v) { store32(p, remain, v.v); }

__device__ __forceinline__ Planes8 load32_fast(const uint8_t *p, uint64_t remain) {
  if (remain >= 32 && (((uintptr_t)p & 15u) == 0)) {
    const uint4 a = __ldg(reinterpret_cast<const uint4 *>(p)), b = __ldg(reinterpret_cast<const uint4 *>(p + 16));
    return Planes8{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
  }
  return load32_any(p, remain);
}

__device__ __forceinline__ void store32_fast(uint8_t *p, uint64_t remain, const Planes8 &v) {
  if (remain >= 32 && (((uintptr_t)p & 15u) == 0)) {
    *reinterpret_cast<uint4 *>(p) = make_uint4(v.v[0], v.v[1], v.v[2], v.v[3]);
    *reinterpret_cast<uint4 *>(p + 16) = make_uint4(v.v[4], v.v[5], v.v[6], v.v[7]);
    return;
  }
  store32_rows(p, remain, v);
}

// Bitsliced matrix apply (the strided ApplyArgs form of gf8_matrix_kernel, no pointer
// tables, no verify): a thread owns one 32-column group of one stripe; each input row is
// loaded and transposed into 8 bit planes once per tile of OT output rows, and every
// coefficient, read as a warp-uniform byte, selects compiled XOR networks (mul8_rt)
// instead of the SWAR form's 8 masked XORs per 4 columns. grid.x: 32-column group tiles
// of kBitsThreads threads; grid.y: stripes (looped); grid.z: tiles of OT output rows.
constexpr int kBitsThreads = 128;

// FORM: 1 one out-of-line call per coefficient, 2 one call per two output rows.
template <int OT, int FORM>
__global__ void __launch_bounds__(kBitsThreads) gf8_bits_kernel(const ApplyArgs a) {
  const uint64_t col = ((uint64_t)blockIdx.x * kBitsThreads + threadIdx.x) * 32;
  const uint32_t k = a.k;
  for (uint32_t s = blockIdx.y; s < a.n_stripes; s += gridDim.y) {
    const uint32_t rows = a.rows_per_stripe ? a.rows_per_stripe[s] : a.rows;
    const uint32_t g0 = blockIdx.z * OT;
    if (g0 >= rows || col >= a.len) continue;
    const uint32_t live = min(rows - g0, (uint32_t)OT);
    const uint64_t remain = a.len - col;
    const uint8_t *cs = a.coeffs + s * a.coeff_stripe_stride + (uint64_t)g0 * k;
    Planes8 acc[OT];
#pragma unroll
    for (int o = 0; o < OT; o++)
#pragma unroll
      for (int b = 0; b < 8; b++) acc[o].v[b] = 0;
    const PtrTableT<false> none{};
    for (uint32_t i = 0; i < k; i++) {
      Planes8 x = load32_fast(in_row<false>(a, none, s, i) + col, remain);
      bit_transpose(x.v);
      if constexpr (FORM == 2) {
#pragma unroll
        for (int o = 0; o < OT; o += 2) {
          if (o < (int)live) {
            const uint32_t c0 = __ldg(cs + (uint64_t)o * k + i);
            const uint32_t c1 = o + 1 < (int)live ? __ldg(cs + (uint64_t)(o + 1) * k + i) : 0u;
            const Planes16 t = mul8x2_rt(x, c0, c1);
#pragma unroll
            for (int b = 0; b < 8; b++) {
              acc[o].v[b] ^= t.a.v[b];
              acc[o + 1].v[b] ^= t.b.v[b];
            }
          }
        }
      } else {
#pragma unroll
        for (int o = 0; o < OT; o++) {
          if (o < (int)live) {
            const uint32_t c = __ldg(cs + (uint64_t)o * k + i);
            const Planes8 t = mul8_rt(x, c);
#pragma unroll
            for (int b = 0; b < 8; b++) acc[o].v[b] ^= t.v[b];
          }
        }
      }
    }
#pragma unroll
    for (int o = 0; o < OT; o++) {
      if (o < (int)live) {
        bit_transpose(acc[o].v);
        store32_fast(out_row<false>(a, none, s, g0 + o) + col, remain, acc[o]);
      }
    }
  }
}

// The ragged launch's block (kernels_batch.cuh ragged_block) on the bitsliced kernel:
// the same (row chunk, 4 KiB column tile) blocks, 128 threads of 32 columns each.
template <int OT>
__device__ __forceinline__ void ragged_block_bits(const RaggedItem &w, uint32_t local) {
  static_assert(kBitsThreads * 32 == kTileBytes, "block tiles of the ragged launch");
  const uint32_t chunk = local / w.col_tiles, tile = local % w.col_tiles;
  const uint32_t k = w.k;
  const uint32_t g0 = chunk * kRowChunk, g_end = min(w.rows, g0 + kRowChunk);
  const uint64_t col = ((uint64_t)tile * kBitsThreads + threadIdx.x) * 32;
  if (col >= w.len) return;
  const uint64_t remain = w.len - col;
  for (uint32_t g = g0; g < g_end; g += OT) {
    const uint32_t live = min(g_end - g, (uint32_t)OT);
    Planes8 acc[OT];
#pragma unroll
    for (int o = 0; o < OT; o++)
#pragma unroll
      for (int b = 0; b < 8; b++) acc[o].v[b] = 0;
    for (uint32_t i = 0; i < k; i++) {
      const uint32_t row = w.in_rows ? w.in_rows[i] : i;
      Planes8 x = load32_fast(w.base + row * w.row_stride + col, remain);
      bit_transpose(x.v);
#pragma unroll
      for (int o = 0; o < OT; o += 2) {
        if (o < (int)live) {
          const uint32_t c0 = __ldg(w.coeffs + (uint64_t)(g + o) * k + i);
          const uint32_t c1 = o + 1 < (int)live ? __ldg(w.coeffs + (uint64_t)(g + o + 1) * k + i) : 0u;
          const Planes16 t = mul8x2_rt(x, c0, c1);
#pragma unroll
          for (int b = 0; b < 8; b++) {
            acc[o].v[b] ^= t.a.v[b];
            acc[o + 1].v[b] ^= t.b.v[b];
          }
        }
      }
    }
#pragma unroll
    for (int o = 0; o < OT; o++) {
      if (o < (int)live) {
        const uint32_t row = w.out_rows ? w.out_rows[g + o] : k + g + o;
        bit_transpose(acc[o].v);
        store32_fast(w.base + row * w.row_stride + col, remain, acc[o]);
      }
    }
  }
}

template <int OT>
__global__ void __launch_bounds__(kBitsThreads) gf8_ragged_bits_kernel(const RaggedItem *__restrict__ items,
                                                                       uint32_t n_items) {
  const uint32_t it = find_item(items, n_items, blockIdx.x);
  const RaggedItem &w = items[it];
  ragged_block_bits<OT>(w, blockIdx.x - w.block_begin);
}

// Whether launch_gf8 runs gf8_bits_kernel for strided calls (rs_set_matrix_bits): 0 no
// (the SWAR kernel), 1 one out-of-line call per coefficient, 2 (default) one call per
// two output rows. Measured on B200, matrix-route batched calls (RS(32,32), RS(16,16),
// RS(64,64); 64 KiB and 1 MiB shards): form 2 encodes 20-22% and reconstructs 22-26%
// faster than the SWAR kernel, form 1 15-18%; the networks inlined at every use cost
// 220 registers and ran at 0.5-0.6x the SWAR kernel.
inline int &matrix_bits() {
  static int v = 2;
  return v;
}

template <int OT, int FORM>
inline cudaError_t launch_gf8_bits_t(const ApplyArgs &a, cudaStream_t st) {
  const uint64_t groups = (a.len + 31) / 32;
  dim3 grid((unsigned)((groups + kBitsThreads - 1) / kBitsThreads), std::min<uint32_t>(a.n_stripes, 65535),
            (a.rows + OT - 1) / OT);
  gf8_bits_kernel<OT, FORM><<<grid, kBitsThreads, 0, st>>>(a);
  return cudaGetLastError();
}

// The ragged matrix launch (batches, the request server): the bitsliced kernel unless
// matrix_bits() is 0. Measured on the 10,000-stripe mixed batch it runs at the SWAR
// kernel's speed (830 GB/s batched, 148 GB/s matrix-only, both kernels). smem: the SWAR kernel's dynamic shared memory (its attribute is set
// by the caller, outside any stream capture).
inline cudaError_t launch_ragged(const RaggedItem *items, uint32_t n_items, uint64_t blocks, size_t smem,
                                 cudaStream_t st) {
  if (matrix_bits())
    gf8_ragged_bits_kernel<8><<<(unsigned)blocks, kBitsThreads, 0, st>>>(items, n_items);
  else
    gf8_ragged_kernel<8><<<(unsigned)blocks, kThreads, smem, st>>>(items, n_items);
  return cudaGetLastError();
}

inline cudaError_t launch_gf8_bits(const ApplyArgs &a, cudaStream_t st) {
  if (matrix_bits() == 1) return launch_gf8_bits_t<8, 1>(a, st);
  return launch_gf8_bits_t<8, 2>(a, st);
}

}  // namespace rsb
