// Ragged batches: one launch over stripes of different shapes, shard lengths and
// erasure patterns. Each work item is one stripe's apply (encode or reconstruct):
// out[j] = sum_t coeff[j][t] * in[t] over `len` byte columns, with rows addressed by
// index into the stripe's row array. The grid is the concatenation of every item's
// (row chunk, column tile) blocks; a CTA finds its item by binary search over the
// items' first-block prefix sums.
#pragma once

#include <cstdint>

#include "kernels_matrix.cuh"

namespace rsb {

struct RaggedItem {
  uint8_t *base;             // row 0 of the stripe
  uint64_t row_stride;       // bytes between rows
  uint64_t len;              // shard bytes
  const uint8_t *coeffs;     // rows x k, row-major
  const uint16_t *in_rows;   // k input row indexes; nullptr = 0..k-1
  const uint16_t *out_rows;  // `rows` output row indexes; nullptr = k..k+rows-1
  uint32_t k, rows;
  uint32_t block_begin;      // first grid block of this item
  uint32_t col_tiles;        // column tiles (kTileBytes each)
};

__device__ __forceinline__ uint32_t find_item(const RaggedItem *items, uint32_t n, uint32_t block) {
  uint32_t lo = 0, hi = n;  // last item with block_begin <= block
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (items[mid].block_begin <= block)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// One block of work of an item: row chunk `local / col_tiles`, column tile
// `local % col_tiles`. R is the 8 KiB constant table (fill_rtab, filled once), C room
// for kRowChunk x k coefficients. Every thread of the CTA calls it (it meets at
// barriers around the coefficient table).
template <int OUT_TILE>
__device__ __forceinline__ void ragged_block(const RaggedItem &w, uint32_t local, const uint32_t *R, uint8_t *C) {
  const uint32_t chunk = local / w.col_tiles, tile = local % w.col_tiles;
  const uint32_t k = w.k;
  const uint32_t g0 = chunk * kRowChunk, g_end = min(w.rows, g0 + kRowChunk);
  __syncthreads();  // the previous block's readers of C are done
  for (uint32_t t = threadIdx.x; t < (g_end - g0) * k; t += kThreads) C[t] = w.coeffs[g0 * k + t];
  __syncthreads();
  const uint64_t col = ((uint64_t)tile * kThreads + threadIdx.x) * kBytesPerThread;
  if (col >= w.len) return;
  const uint64_t remain = w.len - col;
  for (uint32_t g = g0; g < g_end; g += OUT_TILE) {
    const uint32_t live = g_end - g;
    uint32_t acc[OUT_TILE][4];
#pragma unroll
    for (int o = 0; o < OUT_TILE; o++) acc[o][0] = acc[o][1] = acc[o][2] = acc[o][3] = 0;
    for (uint32_t i = 0; i < k; i++) {
      const uint32_t row = w.in_rows ? w.in_rows[i] : i;
      uint4 x = load_cols(w.base + row * w.row_stride + col, remain);
      uint32_t m[4][8];
      bit_masks(x.x, m[0]);
      bit_masks(x.y, m[1]);
      bit_masks(x.z, m[2]);
      bit_masks(x.w, m[3]);
#pragma unroll
      for (int o = 0; o < OUT_TILE; o++) {
        if (o < (int)live) {
          const uint4 *r4 = reinterpret_cast<const uint4 *>(R + 8 * C[(g - g0 + o) * k + i]);
          uint4 r0 = r4[0], r1 = r4[1];
          uint32_t r[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
#pragma unroll
          for (int q = 0; q < 4; q++)
#pragma unroll
            for (int b = 0; b < 8; b++) acc[o][q] ^= m[q][b] & r[b];
        }
      }
    }
#pragma unroll
    for (int o = 0; o < OUT_TILE; o++) {
      if (o < (int)live) {
        const uint32_t row = w.out_rows ? w.out_rows[g + o] : k + g + o;
        store_cols(w.base + row * w.row_stride + col, remain,
                   make_uint4(acc[o][0], acc[o][1], acc[o][2], acc[o][3]));
      }
    }
  }
}

// Dynamic shared memory: 8 KiB constant table + up to max_rows*max_k coefficients.
template <int OUT_TILE>
__global__ void __launch_bounds__(kThreads)
    gf8_ragged_kernel(const RaggedItem *__restrict__ items, uint32_t n_items) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t *R = smem;
  uint8_t *C = reinterpret_cast<uint8_t *>(smem + 2048);
  fill_rtab(R);
  const uint32_t it = find_item(items, n_items, blockIdx.x);
  const RaggedItem &w = items[it];
  ragged_block<OUT_TILE>(w, blockIdx.x - w.block_begin, R, C);
}

}  // namespace rsb
