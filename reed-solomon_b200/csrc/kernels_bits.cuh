// Bitsliced GF(2^8) products by constants known only at run time but the same for every
// lane of a warp (a butterfly's constant, a stripe's decode coefficient), and the
// bitsliced matrix kernel built on them.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

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

// ---- runtime coefficients through shared-memory XOR tables (four Russians) ----
// Plane b of c * x is the XOR of the planes p of x for which bit b of c * 2^p is set.
// Split the 8 input planes into two nibbles: every XOR of a subset of planes 0..3 (16
// words) and of planes 4..7 (16 words) is formed once per input row (11 + 11 XORs) and
// stored in shared memory, one column of words per thread; then plane b of c * x is
// lo[m_lo(c, b)] ^ hi[m_hi(c, b)]: two loads whose row indexes are the same for every
// lane of the warp (one coefficient per warp), so each load is one conflict-free
// wavefront. A coefficient costs 16 loads, 16 PRMT and 8 LOP3 (plus its share of the
// row's 22 XORs and 30 stores) instead of two compiled XOR networks behind two indirect
// branches.
//
// Addressing. The CTA's 128 threads form two halves of 64, each with its own subset
// rows of 64 words (256 bytes), so a thread's word in row j sits at (j << 8) | 4 * lane
// of its half, and each address is one PRMT of two bytes: the thread's and the row
// index. A coefficient's 16 row indexes are one 16-byte table entry (bytes j_lo, j_hi
// for planes 2q and 2q + 1 in word q), read as one broadcast load; the CTA stages its
// output rows' coefficients for every input row as table offsets, 16 to a 64-byte line.
constexpr int kLutThreads = 128;
constexpr int kLutHalf = 64;
constexpr int kLutOT = 16;  // output rows per pass over the inputs (staging is sized for it)
constexpr int kLutMaxK = 255;

struct LutShared {
  uint4 tab[256];                          // [coefficient] -> row index bytes
  uint32_t rows[2][32][kLutHalf];          // [half][subset row: lo 0..15, hi 16..31][lane of half]
  uint32_t cidx[kLutMaxK][kLutOT];         // [input row][output row] -> 16 * coefficient
};

// Table entry of coefficient c: word q holds the lo and hi row indexes of planes 2q and
// 2q + 1 (hi rows are 16 + subset).
__device__ __forceinline__ uint4 lut_entry(uint32_t c) {
  uint32_t col[8];
  col[0] = c;
#pragma unroll
  for (int p = 1; p < 8; p++) col[p] = fftc::xt((uint8_t)col[p - 1]);
  uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
  for (int b = 0; b < 8; b++) {
    uint32_t lo = 0, hi = 16;
#pragma unroll
    for (int p = 0; p < 4; p++) {
      lo |= ((col[p] >> b) & 1u) << p;
      hi |= ((col[p + 4] >> b) & 1u) << p;
    }
    w[b >> 1] |= (lo | hi << 8) << (16 * (b & 1));
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// The table and the zero rows (subset 0 of each nibble, both halves); the caller meets
// at a barrier before the first lookup.
__device__ __forceinline__ void lut_init(LutShared &sh) {
  for (uint32_t c = threadIdx.x; c < 256; c += blockDim.x) sh.tab[c] = lut_entry(c);
  const uint32_t h = threadIdx.x / kLutHalf, l = threadIdx.x % kLutHalf;
  sh.rows[h][0][l] = 0;
  sh.rows[h][16][l] = 0;
}

// The 15 non-empty subsets of planes x0..x3 into rows B + 1 .. B + 15 of this thread's
// column (stride kLutHalf words).
template <int B>
__device__ __forceinline__ void lut_store_nibble(uint32_t *col, uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3) {
  const uint32_t c3 = x0 ^ x1, c5 = x2 ^ x0, c6 = x2 ^ x1, c7 = x2 ^ c3;
  const uint32_t v[16] = {0, x0, x1, c3, x2, c5, c6, c7, x3, x3 ^ x0, x3 ^ x1, x3 ^ c3, x3 ^ x2, x3 ^ c5, x3 ^ c6, x3 ^ c7};
#pragma unroll
  for (int j = 1; j < 16; j++) col[(B + j) * kLutHalf] = v[j];
}

__device__ __forceinline__ uint32_t lut_addr(uint32_t tb, uint32_t w, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(tb), "r"(w), "r"(sel));
  return r;
}

// acc ^= c * x for the coefficient whose table offset is ci; rows: this half's subset
// rows (x's already stored); tb = 4 * lane of the half.
__device__ __forceinline__ void lut_mul_acc(Planes8 &acc, const LutShared &sh, const char *rows, uint32_t tb,
                                            uint32_t ci) {
  const uint4 e = *reinterpret_cast<const uint4 *>(reinterpret_cast<const char *>(sh.tab) + ci);
  const uint32_t w[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
  for (int b = 0; b < 8; b++) {
    // bytes: [tb, row index, 0, 0]; tb < 256, so its bytes 1..3 are zero
    const uint32_t lo = lut_addr(tb, w[b >> 1], 0x1140u + 0x20u * (b & 1));
    const uint32_t hi = lut_addr(tb, w[b >> 1], 0x1150u + 0x20u * (b & 1));
    acc.v[b] ^= *reinterpret_cast<const uint32_t *>(rows + lo) ^ *reinterpret_cast<const uint32_t *>(rows + hi);
  }
}

// One input row's subset rows from its 8 planes.
__device__ __forceinline__ void lut_store_row(uint32_t *col, const Planes8 &x) {
  lut_store_nibble<0>(col, x.v[0], x.v[1], x.v[2], x.v[3]);
  lut_store_nibble<16>(col, x.v[4], x.v[5], x.v[6], x.v[7]);
}

// Stages output rows [g, g + live) of a row-major coefficient matrix (k per row) as
// table offsets; all threads take part, between barriers.
__device__ __forceinline__ void lut_stage(LutShared &sh, const uint8_t *coeffs, uint32_t k, uint32_t live) {
  for (uint32_t t = threadIdx.x; t < live * k; t += blockDim.x) {
    const uint32_t o = t / k, i = t - o * k;
    sh.cidx[i][o] = 16u * __ldg(coeffs + (uint64_t)o * k + i);
  }
}

// The pass over the inputs of one output tile for one half H of the CTA (H a template
// parameter, so its subset rows sit at a compile-time offset). in(i): input row i's
// address at this thread's column; out(o): output row o's.
template <int OT, int H, typename In, typename Out>
__device__ __forceinline__ void lut_tile(LutShared &sh, uint32_t k, uint32_t live, uint64_t remain, In in, Out out) {
  const uint32_t lane = threadIdx.x % kLutHalf, tb = lane * 4;
  uint32_t *col = &sh.rows[H][0][lane];
  const char *rows = reinterpret_cast<const char *>(&sh.rows[H][0][0]);
  Planes8 acc[OT];
#pragma unroll
  for (int o = 0; o < OT; o++)
#pragma unroll
    for (int b = 0; b < 8; b++) acc[o].v[b] = 0;
  for (uint32_t i = 0; i < k; i++) {
    Planes8 x = load32_fast(in(i), remain);
    bit_transpose(x.v);
    lut_store_row(col, x);
    const uint4 *ci = reinterpret_cast<const uint4 *>(sh.cidx[i]);
#pragma unroll
    for (int q = 0; q < OT / 4; q++) {
      const uint4 c4 = ci[q];
      const uint32_t c[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (4 * q + u < (int)live) lut_mul_acc(acc[4 * q + u], sh, rows, tb, c[u]);
    }
  }
#pragma unroll
  for (int o = 0; o < OT; o++) {
    if (o < (int)live) {
      bit_transpose(acc[o].v);
      store32_fast(out(o), remain, acc[o]);
    }
  }
}

// Strided matrix apply on the lookup tables: one 32-column group per thread, tiles of
// OT output rows in grid.z, stripes in grid.y (looped).
template <int OT>
__global__ void __launch_bounds__(kLutThreads) gf8_lut_kernel(const ApplyArgs a) {
  static_assert(OT % 4 == 0 && OT <= kLutOT, "output tile");
  __shared__ __align__(16) LutShared sh;
  lut_init(sh);
  const uint64_t col = ((uint64_t)blockIdx.x * kLutThreads + threadIdx.x) * 32;
  const uint32_t k = a.k;
  const PtrTableT<false> none{};
  for (uint32_t s = blockIdx.y; s < a.n_stripes; s += gridDim.y) {
    const uint32_t rows = a.rows_per_stripe ? a.rows_per_stripe[s] : a.rows;
    const uint32_t g0 = blockIdx.z * OT;
    if (g0 >= rows) continue;  // the same for the whole CTA
    const uint32_t live = min(rows - g0, (uint32_t)OT);
    __syncthreads();  // the previous stripe's offsets are no longer read
    lut_stage(sh, a.coeffs + s * a.coeff_stripe_stride + (uint64_t)g0 * k, k, live);
    __syncthreads();
    if (col >= a.len) continue;
    const uint64_t remain = a.len - col;
    auto in = [&](uint32_t i) { return in_row<false>(a, none, s, i) + col; };
    auto out = [&](uint32_t o) { return out_row<false>(a, none, s, g0 + o) + col; };
    if (threadIdx.x < kLutHalf)
      lut_tile<OT, 0>(sh, k, live, remain, in, out);
    else
      lut_tile<OT, 1>(sh, k, live, remain, in, out);
  }
}

// The ragged launch's block on the lookup tables: the (row chunk, 4 KiB column tile)
// blocks of the other ragged kernels, OT output rows per pass over the inputs.
template <int OT>
__device__ __forceinline__ void ragged_block_lut(const RaggedItem &w, uint32_t local, LutShared &sh) {
  static_assert(kLutThreads * 32 == kTileBytes, "block tiles of the ragged launch");
  const uint32_t chunk = local / w.col_tiles, tile = local % w.col_tiles;
  const uint32_t k = w.k;
  const uint32_t g0 = chunk * kRowChunk, g_end = min(w.rows, g0 + kRowChunk);
  const uint64_t col = ((uint64_t)tile * kLutThreads + threadIdx.x) * 32;
  for (uint32_t g = g0; g < g_end; g += OT) {
    const uint32_t live = min(g_end - g, (uint32_t)OT);
    __syncthreads();
    lut_stage(sh, w.coeffs + (uint64_t)g * k, k, live);
    __syncthreads();
    if (col >= w.len) continue;
    const uint64_t remain = w.len - col;
    auto in = [&](uint32_t i) {
      const uint32_t row = w.in_rows ? w.in_rows[i] : i;
      return w.base + row * w.row_stride + col;
    };
    auto out = [&](uint32_t o) {
      const uint32_t row = w.out_rows ? w.out_rows[g + o] : k + g + o;
      return w.base + row * w.row_stride + col;
    };
    if (threadIdx.x < kLutHalf)
      lut_tile<OT, 0>(sh, k, live, remain, in, out);
    else
      lut_tile<OT, 1>(sh, k, live, remain, in, out);
  }
}

template <int OT>
__global__ void __launch_bounds__(kLutThreads) gf8_ragged_lut_kernel(const RaggedItem *__restrict__ items,
                                                                     uint32_t n_items) {
  __shared__ __align__(16) LutShared sh;
  lut_init(sh);
  const uint32_t it = find_item(items, n_items, blockIdx.x);
  const RaggedItem &w = items[it];
  ragged_block_lut<OT>(w, blockIdx.x - w.block_begin, sh);
}

// The kernel of strided matrix-route calls and of the ragged launches
// (rs_set_matrix_bits): 3 (default) the lookup kernel (gf8_lut_kernel, shared-memory
// subset tables, 8- or 16-row tiles by size), 4 the same with 8-row tiles only, 2 the
// bitsliced kernel whose coefficients select compiled XOR networks (one call per two
// output rows), 1 the same with one call per coefficient, 0 the SWAR kernel. Measured
// on B200 (matrix-route batched calls, one process): the lookup kernel encodes RS(32,32)
// 1.63x and RS(128,128) 1.74x faster than form 2, which was 20-22% faster than the SWAR
// kernel; on the 10,000-stripe mixed batch it takes the (128,128) reconstructs from 43
// to 24 ms.
inline int &matrix_bits() {
  static int v = 3;
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

template <int OT>
inline cudaError_t launch_gf8_lut_t(const ApplyArgs &a, cudaStream_t st) {
  const uint64_t groups = (a.len + 31) / 32;
  dim3 grid((unsigned)((groups + kLutThreads - 1) / kLutThreads), std::min<uint32_t>(a.n_stripes, 65535),
            (a.rows + OT - 1) / OT);
  gf8_lut_kernel<OT><<<grid, kLutThreads, 0, st>>>(a);
  return cudaGetLastError();
}

// Ragged items in launch order: items with at most 8 output rows first, then the rest,
// each part numbered from block 0, so that the lookup kernel runs its 8-row tile (114
// registers, 16 warps per SM) on the short reconstructs and its 16-row tile (168
// registers, 12 warps) on the rest. Measured on the 10,000-stripe mixed batch: the
// 8-row tile rebuilds (10,10) and (16,16) stripes 1.4-1.5x faster than the 16-row tile,
// which is 4% faster at (128,128). Returns the first part's item count; blocks[p] is
// part p's grid size.
inline uint32_t ragged_split(std::vector<RaggedItem> &items, uint64_t blocks[2]) {
  std::stable_partition(items.begin(), items.end(), [](const RaggedItem &r) { return r.rows <= 8; });
  uint32_t n0 = 0;
  blocks[0] = blocks[1] = 0;
  for (RaggedItem &r : items) {
    const int part = r.rows <= 8 ? 0 : 1;
    n0 += part == 0;
    r.col_tiles = (uint32_t)((r.len + kTileBytes - 1) / kTileBytes);
    r.block_begin = (uint32_t)blocks[part];
    blocks[part] += (uint64_t)r.col_tiles * ((r.rows + kRowChunk - 1) / kRowChunk);
  }
  return n0;
}

inline int ragged_launches(const uint64_t blocks[2]) { return (blocks[0] > 0) + (blocks[1] > 0); }

// The ragged matrix launch (batches, the request server) over the two parts that
// ragged_split made: the lookup kernel by default (matrix_bits() 3 or 4), else the
// bitsliced network kernel (1, 2) or the SWAR kernel (0) on both parts. smem: the SWAR
// kernel's dynamic shared memory (its attribute is set by the caller, outside any
// stream capture).
inline cudaError_t launch_ragged(const RaggedItem *items, uint32_t n0, uint32_t n_items, const uint64_t blocks[2],
                                 size_t smem, cudaStream_t st) {
  for (int part = 0; part < 2; part++) {
    const RaggedItem *it = part ? items + n0 : items;
    const uint32_t n = part ? n_items - n0 : n0;
    const unsigned grid = (unsigned)blocks[part];
    if (!n || !grid) continue;
    if (matrix_bits() == 3 && part == 1)
      gf8_ragged_lut_kernel<16><<<grid, kLutThreads, 0, st>>>(it, n);
    else if (matrix_bits() >= 3)
      gf8_ragged_lut_kernel<8><<<grid, kLutThreads, 0, st>>>(it, n);
    else if (matrix_bits())
      gf8_ragged_bits_kernel<8><<<grid, kBitsThreads, 0, st>>>(it, n);
    else
      gf8_ragged_kernel<8><<<grid, kThreads, smem, st>>>(it, n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

inline cudaError_t launch_gf8_bits(const ApplyArgs &a, cudaStream_t st) {
  if (matrix_bits() == 1) return launch_gf8_bits_t<8, 1>(a, st);
  if (matrix_bits() == 3 && a.k <= (uint32_t)kLutMaxK) {
    // The 16-row tile pays where most stripes fill it: encodes of more than 8 parity
    // rows, reconstructs whose largest stripe rebuilds more than 32 rows (measured:
    // RS(32,32) encode 664 vs 610 GB/s, RS(128,128) reconstruct 273 vs 260; RS(32,32)
    // reconstruct 820 vs 888 the other way).
    const bool wide = a.rows_per_stripe ? a.rows > 32 : a.rows > 8;
    return wide ? launch_gf8_lut_t<16>(a, st) : launch_gf8_lut_t<8>(a, st);
  }
  if (matrix_bits() == 4 && a.k <= (uint32_t)kLutMaxK) return launch_gf8_lut_t<8>(a, st);
  return launch_gf8_bits_t<8, 2>(a, st);
}

}  // namespace rsb
