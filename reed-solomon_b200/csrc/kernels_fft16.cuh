// FFT-route encode for ReedSolomon16: the Lin-Chung-Han additive FFT over the tower
// field GF((2^8)^2) (src/fft16.rs), bitsliced for CUDA cores.
//
// For k = K a power of two, encode is an inverse transform of the K data rows on the
// points {0..K-1} (interpolation into the novel basis, src/fft16.rs:223-) followed,
// for every coset {cK .. cK+K-1} that holds parity points, by a forward transform of
// those coefficients with beta = cK; the outputs are the parity rows in point order.
// Butterflies follow the reference's order and constants: at level l a block of
// 2^(l+1) registers at `base` uses c = WHAT[l][beta ^ base]; inverse: hi ^= lo,
// lo ^= c*hi; forward: lo ^= c*hi, hi ^= lo.
//
// Bitslicing. 32 symbols of one shard (32 low-plane bytes and 32 high-plane bytes)
// become 16 bit planes: planes 0..7 hold the low byte's bits, 8..15 the high byte's,
// so bit p of a symbol's u16 value is plane p. Multiplying by a constant c is the
// 16x16 GF(2) matrix whose column p is c * 2^p: plane b of the product is the XOR of
// the planes p with bit b of c * 2^p set. The constants differ per butterfly block and
// are only known at run time, so the product is applied as masked XORs (one
// three-input LOP3 each) with masks in shared memory, in the tower's Karatsuba form:
// with c = (c_hi, c_lo) and x = (x_hi, x_lo), t0 = c_lo x_lo, t1 = (c_hi + c_lo)(x_lo +
// x_hi), t2 = 32 c_hi x_hi, and c x = (t0 + t1) y + (t0 + t2) — three 8x8 GF(2)
// matrices, 192 masks and ~216 LOP3 per product instead of a 16x16 matrix's 256.
// A constant's table entry (16 u16) holds the column bytes k_t * 2^p of its three
// GF(2^8) factors k0 = c_lo, k1 = c_hi + c_lo, k2 = 32 c_hi (24 bytes, 8 unused).
//
// Work split. The transform runs over a bitsliced scratch buffer: register r of R of
// stripe s is a block of G * 16 words at ((s * R + r) * G) * 16, holding plane p of
// 32-symbol group g of G at word ((p / 4) * G + g) * 4 + p % 4, so the lanes of a warp
// (consecutive groups) read and write each 16-byte quarter of their planes as one
// contiguous 512-byte span.
// A pass applies one or two levels. Its kernel runs one warp per CTA, persistent over
// (butterfly group, stripe) items with one lane per 32-symbol group, so a warp's lanes
// share the item's constants and read their masks as shared-memory broadcasts.
#pragma once

#include <cstdint>

#include "kernels_bits.cuh"
#include "kernels_fft.cuh"

namespace rsb {

constexpr int kFft16Threads = 256;

// A transform over a window of registers: it reads src registers [src_start, +R) and
// writes dst registers [dst_start, +R) of buffers holding src_regs / dst_regs registers
// per stripe (src may equal dst).
struct Fft16PassArgs {
  const uint32_t *src;
  uint32_t *dst;
  const uint16_t *cols;  // 16 u16 per constant (see above); constant (l, j) at R - (R >> l) + j
  uint32_t R;            // registers in the transform (a power of two)
  uint32_t level;        // lowest level of the pass
  uint32_t src_regs, src_start, dst_regs, dst_start;
  uint64_t G;            // 32-symbol groups per shard in the buffers
  uint32_t n_stripes;
  int inverse;
};

using Reg16 = uint32_t[16];

constexpr uint32_t kMask16 = 192;  // masks per tower constant

// Mask word t of a constant (layout [factor][output bit b][input bit p]): all-ones when
// bit b of k_factor * 2^p is set.
__device__ __forceinline__ uint32_t mask16(const uint16_t *cols, uint32_t t) {
  const uint8_t byte = reinterpret_cast<const uint8_t *>(cols)[(t >> 6) * 8 + (t & 7)];
  return ((byte >> ((t >> 3) & 7)) & 1) ? ~0u : 0u;
}

// All 192 masks of one constant, written by one warp: lane L owns the words w = L + 32 i
// (i = 0 .. 5), whose input bit w & 7 = L & 7 is the same for all six, so it loads the
// three column bytes f * 8 + (L & 7) once and takes bits (L >> 3) and (L >> 3) + 4 of each.
__device__ __forceinline__ void masks_warp(uint32_t *m, const uint16_t *cols, uint32_t lane) {
  const uint8_t *bytes = reinterpret_cast<const uint8_t *>(cols);
  const uint32_t p = lane & 7, b = lane >> 3;
  uint32_t v[3];
#pragma unroll
  for (int f = 0; f < 3; f++) v[f] = bytes[f * 8 + p];
#pragma unroll
  for (int f = 0; f < 3; f++) {
    m[64 * f + lane] = ((v[f] >> b) & 1) ? ~0u : 0u;
    m[64 * f + 32 + lane] = ((v[f] >> (b + 4)) & 1) ? ~0u : 0u;
  }
}

// Planes b of an 8x8 product of the 8 planes x, masks m[b * 8 + p], for output bit b.
__device__ __forceinline__ uint32_t mat8_row(const uint32_t *x, const uint32_t *m, int b) {
  const uint4 *m4 = reinterpret_cast<const uint4 *>(m + b * 8);
  const uint4 u = m4[0], v = m4[1];
  return (x[0] & u.x) ^ (x[1] & u.y) ^ (x[2] & u.z) ^ (x[3] & u.w) ^ (x[4] & v.x) ^ (x[5] & v.y) ^
         (x[6] & v.z) ^ (x[7] & v.w);
}

// d ^= c * s in Karatsuba form (masks m: 3 x 64 words).
__device__ __forceinline__ void mul16_acc(Reg16 &d, const Reg16 &s, const uint32_t *m) {
  uint32_t lx[8], hx[8], sx[8];
#pragma unroll
  for (int p = 0; p < 8; p++) lx[p] = s[p], hx[p] = s[8 + p], sx[p] = s[p] ^ s[8 + p];
#pragma unroll
  for (int b = 0; b < 8; b++) {
    const uint32_t t0 = mat8_row(lx, m, b), t1 = mat8_row(sx, m + 64, b), t2 = mat8_row(hx, m + 128, b);
    d[b] ^= t0 ^ t2;
    d[8 + b] ^= t0 ^ t1;
  }
}

// d1 ^= c * s1 and d2 ^= c * s2 with one read of the masks.
__device__ __forceinline__ void mul16_acc2(Reg16 &d1, const Reg16 &s1, Reg16 &d2, const Reg16 &s2,
                                           const uint32_t *m) {
  uint32_t l1[8], h1[8], x1[8], l2[8], h2[8], x2[8];
#pragma unroll
  for (int p = 0; p < 8; p++) {
    l1[p] = s1[p], h1[p] = s1[8 + p], x1[p] = s1[p] ^ s1[8 + p];
    l2[p] = s2[p], h2[p] = s2[8 + p], x2[p] = s2[p] ^ s2[8 + p];
  }
#pragma unroll
  for (int b = 0; b < 8; b++) {
    const uint4 *k0 = reinterpret_cast<const uint4 *>(m + b * 8);
    const uint4 *k1 = reinterpret_cast<const uint4 *>(m + 64 + b * 8);
    const uint4 *k2 = reinterpret_cast<const uint4 *>(m + 128 + b * 8);
    const uint4 a0 = k0[0], a1 = k0[1], b0 = k1[0], b1 = k1[1], c0 = k2[0], c1 = k2[1];
    auto row = [](const uint32_t *x, uint4 u, uint4 v) {
      return (x[0] & u.x) ^ (x[1] & u.y) ^ (x[2] & u.z) ^ (x[3] & u.w) ^ (x[4] & v.x) ^ (x[5] & v.y) ^
             (x[6] & v.z) ^ (x[7] & v.w);
    };
    const uint32_t t0 = row(l1, a0, a1), t1 = row(x1, b0, b1), t2 = row(h1, c0, c1);
    d1[b] ^= t0 ^ t2;
    d1[8 + b] ^= t0 ^ t1;
    const uint32_t u0 = row(l2, a0, a1), u1 = row(x2, b0, b1), u2 = row(h2, c0, c1);
    d2[b] ^= u0 ^ u2;
    d2[8 + b] ^= u0 ^ u1;
  }
}

__device__ __forceinline__ void xor16(Reg16 &d, const Reg16 &s) {
#pragma unroll
  for (int p = 0; p < 16; p++) d[p] ^= s[p];
}

// inverse: hi ^= lo, lo ^= c*hi; forward: lo ^= c*hi, hi ^= lo.
__device__ __forceinline__ void bfly16(Reg16 &lo, Reg16 &hi, const uint32_t *m, bool inverse) {
  if (inverse) {
    xor16(hi, lo);
    mul16_acc(lo, hi, m);
  } else {
    mul16_acc(lo, hi, m);
    xor16(hi, lo);
  }
}

// Two butterflies with the same constant: (lo1, hi1) and (lo2, hi2).
__device__ __forceinline__ void bfly16x2(Reg16 &lo1, Reg16 &hi1, Reg16 &lo2, Reg16 &hi2, const uint32_t *m,
                                         bool inverse) {
  if (inverse) {
    xor16(hi1, lo1);
    xor16(hi2, lo2);
    mul16_acc2(lo1, hi1, lo2, hi2, m);
  } else {
    mul16_acc2(lo1, hi1, lo2, hi2, m);
    xor16(hi1, lo1);
    xor16(hi2, lo2);
  }
}

// Quarter c (planes 4c .. 4c+3) of group g in the register block at blk (G groups).
__device__ __forceinline__ const uint32_t *quarter16(const uint32_t *blk, uint64_t G, uint64_t g, int c) {
  return blk + ((uint64_t)c * G + g) * 4;
}
__device__ __forceinline__ uint32_t *quarter16(uint32_t *blk, uint64_t G, uint64_t g, int c) {
  return blk + ((uint64_t)c * G + g) * 4;
}

__device__ __forceinline__ void load_reg16(const uint32_t *blk, uint64_t G, uint64_t g, Reg16 &r) {
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const uint4 v = *reinterpret_cast<const uint4 *>(quarter16(blk, G, g, i));
    r[4 * i] = v.x, r[4 * i + 1] = v.y, r[4 * i + 2] = v.z, r[4 * i + 3] = v.w;
  }
}

__device__ __forceinline__ void store_reg16(uint32_t *blk, uint64_t G, uint64_t g, const Reg16 &r) {
#pragma unroll
  for (int i = 0; i < 4; i++)
    *reinterpret_cast<uint4 *>(quarter16(blk, G, g, i)) = make_uint4(r[4 * i], r[4 * i + 1], r[4 * i + 2], r[4 * i + 3]);
}

// LV = 1: registers {i0, i0+h} at level L (h = 2^L). LV = 2: {i0, i0+h, i0+2h, i0+3h},
// levels L and L+1 (inverse: L then L+1; forward: L+1 then L).
//
// One warp per CTA, persistent over items (butterfly group, task): item = group * tasks
// + task, a task being one stripe's 32 symbol groups (one per lane). While an item is
// computed, the next item's registers are already being copied into shared memory with
// cp.async, so scratch loads overlap the multiplies; the item's three constants are
// expanded into masks in shared memory (broadcast reads).
template <int LV>
__global__ void __launch_bounds__(32, 16) fft16_pass_kernel(const Fft16PassArgs a) {
  constexpr int NC = LV == 2 ? 3 : 1, NR = 1 << LV;
  __shared__ __align__(16) uint32_t mk[NC][kMask16];
  __shared__ __align__(16) uint4 stage[NR][4][32];  // [register][16-byte quarter][lane]
  const uint32_t R = a.R, L = a.level, h = 1u << L, lane = threadIdx.x;
  const uint32_t chunks = (uint32_t)((a.G + 31) / 32), tasks = a.n_stripes * chunks;
  const uint32_t items = (R >> LV) * tasks;
  struct Item {
    uint32_t grp, s;
    uint64_t g;
  };
  auto locate = [&](uint32_t item) {
    Item it;
    it.grp = item / tasks;
    const uint32_t task = item - it.grp * tasks;
    it.s = task / chunks;
    it.g = (uint64_t)(task - it.s * chunks) * 32 + lane;
    return it;
  };
  auto first_reg = [&](uint32_t grp) { return (grp >> L) * (h << LV) + (grp & (h - 1)); };
  auto prefetch = [&](uint32_t item) {
    const Item it = locate(item);
    if (it.g < a.G) {
      const uint32_t i0 = first_reg(it.grp);
#pragma unroll
      for (int q = 0; q < NR; q++) {
        const uint32_t *p = a.src + ((uint64_t)it.s * a.src_regs + a.src_start + i0 + q * h) * a.G * 16;
#pragma unroll
        for (int c = 0; c < 4; c++) cp_async16(&stage[q][c][lane], quarter16(p, a.G, it.g, c));
      }
    }
    cp_async_commit();
  };
  uint32_t item = blockIdx.x;
  if (item < items) prefetch(item);
  for (; item < items; item += gridDim.x) {
    const Item it = locate(item);
    const uint32_t blk = it.grp >> L, i0 = first_reg(it.grp);
    uint32_t cidx[NC];
    if constexpr (LV == 2) {
      cidx[0] = R - (R >> L) + 2 * blk;      // level L, block of i0 / i0+h
      cidx[1] = R - (R >> L) + 2 * blk + 1;  // level L, block of i0+2h / i0+3h
      cidx[2] = R - (R >> (L + 1)) + blk;    // level L+1
    } else {
      cidx[0] = R - (R >> L) + blk;
    }
    __syncwarp();  // the previous item's masks are no longer read
#pragma unroll
    for (int c = 0; c < NC; c++) masks_warp(mk[c], a.cols + 16 * cidx[c], lane);
    cp_async_wait_all();
    __syncwarp();
    Reg16 r[NR];
#pragma unroll
    for (int q = 0; q < NR; q++)
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const uint4 v = stage[q][c][lane];
        r[q][4 * c] = v.x, r[q][4 * c + 1] = v.y, r[q][4 * c + 2] = v.z, r[q][4 * c + 3] = v.w;
      }
    __syncwarp();  // the stage is read; the next item's copies may overwrite it
    if (item + gridDim.x < items) prefetch(item + gridDim.x);
    if (it.g >= a.G) continue;
    if constexpr (LV == 2) {
      if (a.inverse) {
        bfly16(r[0], r[1], mk[0], true);
        bfly16(r[2], r[3], mk[1], true);
        bfly16x2(r[0], r[2], r[1], r[3], mk[2], true);
      } else {
        bfly16x2(r[0], r[2], r[1], r[3], mk[2], false);
        bfly16(r[0], r[1], mk[0], false);
        bfly16(r[2], r[3], mk[1], false);
      }
    } else {
      bfly16(r[0], r[1], mk[0], a.inverse != 0);
    }
    const uint64_t db = (uint64_t)it.s * a.dst_regs + a.dst_start;
#pragma unroll
    for (int q = 0; q < NR; q++) store_reg16(a.dst + (db + i0 + q * h) * a.G * 16, a.G, it.g, r[q]);
  }
}

// d ^= c * s with c's Karatsuba factors packed in kf (k0 | k1 << 8 | k2 << 16).
__device__ __forceinline__ void mul16_acc_rt(Reg16 &d, const Reg16 &s, uint32_t kf) {
  Planes8 lx, hx, sx;
#pragma unroll
  for (int p = 0; p < 8; p++) lx.v[p] = s[p], hx.v[p] = s[8 + p], sx.v[p] = s[p] ^ s[8 + p];
  const Planes8 t0 = mul8_rt(lx, kf & 0xff), t1 = mul8_rt(sx, (kf >> 8) & 0xff), t2 = mul8_rt(hx, kf >> 16);
#pragma unroll
  for (int b = 0; b < 8; b++) {
    d[b] ^= t0.v[b] ^ t2.v[b];
    d[8 + b] ^= t0.v[b] ^ t1.v[b];
  }
}

__device__ __forceinline__ void bfly16_rt(Reg16 &lo, Reg16 &hi, uint32_t kf, bool inverse) {
  if (inverse) {
    xor16(hi, lo);
    mul16_acc_rt(lo, hi, kf);
  } else {
    mul16_acc_rt(lo, hi, kf);
    xor16(hi, lo);
  }
}

// The factors of constant i of a table (bytes 24..26 of its entry).
__device__ __forceinline__ uint32_t const_factors(const uint16_t *cols, uint32_t i) {
  return *reinterpret_cast<const uint32_t *>(cols + 16 * (size_t)i + 12);
}

// fft16_pass_kernel with the constants applied through mul8_rt: no mask tables.
template <int LV>
__global__ void __launch_bounds__(32, 16) fft16_pass_rt_kernel(const Fft16PassArgs a) {
  constexpr int NR = 1 << LV;
  __shared__ __align__(16) uint4 stage[NR][4][32];  // [register][16-byte quarter][lane]
  const uint32_t R = a.R, L = a.level, h = 1u << L, lane = threadIdx.x;
  const uint32_t chunks = (uint32_t)((a.G + 31) / 32), tasks = a.n_stripes * chunks;
  const uint32_t items = (R >> LV) * tasks;
  struct Item {
    uint32_t grp, s;
    uint64_t g;
  };
  auto locate = [&](uint32_t item) {
    Item it;
    it.grp = item / tasks;
    const uint32_t task = item - it.grp * tasks;
    it.s = task / chunks;
    it.g = (uint64_t)(task - it.s * chunks) * 32 + lane;
    return it;
  };
  auto first_reg = [&](uint32_t grp) { return (grp >> L) * (h << LV) + (grp & (h - 1)); };
  constexpr int NK = LV == 2 ? 3 : 1;
  uint32_t kf_next[NK];  // the next item's constants, loaded with its registers
  auto prefetch = [&](uint32_t item) {
    const Item it = locate(item);
    const uint32_t blk = it.grp >> L;
    if constexpr (LV == 2) {
      kf_next[0] = const_factors(a.cols, R - (R >> L) + 2 * blk);      // level L, i0 / i0+h
      kf_next[1] = const_factors(a.cols, R - (R >> L) + 2 * blk + 1);  // level L, i0+2h / i0+3h
      kf_next[2] = const_factors(a.cols, R - (R >> (L + 1)) + blk);    // level L+1
    } else {
      kf_next[0] = const_factors(a.cols, R - (R >> L) + blk);
    }
    if (it.g < a.G) {
      const uint32_t i0 = first_reg(it.grp);
#pragma unroll
      for (int q = 0; q < NR; q++) {
        const uint32_t *p = a.src + ((uint64_t)it.s * a.src_regs + a.src_start + i0 + q * h) * a.G * 16;
#pragma unroll
        for (int c = 0; c < 4; c++) cp_async16(&stage[q][c][lane], quarter16(p, a.G, it.g, c));
      }
    }
    cp_async_commit();
  };
  uint32_t item = blockIdx.x;
  if (item < items) prefetch(item);
  for (; item < items; item += gridDim.x) {
    const Item it = locate(item);
    const uint32_t i0 = first_reg(it.grp);
    uint32_t kf[NK];
#pragma unroll
    for (int c = 0; c < NK; c++) kf[c] = kf_next[c];
    cp_async_wait_all();
    __syncwarp();
    Reg16 r[NR];
#pragma unroll
    for (int q = 0; q < NR; q++)
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const uint4 v = stage[q][c][lane];
        r[q][4 * c] = v.x, r[q][4 * c + 1] = v.y, r[q][4 * c + 2] = v.z, r[q][4 * c + 3] = v.w;
      }
    __syncwarp();  // the stage is read; the next item's copies may overwrite it
    if (item + gridDim.x < items) prefetch(item + gridDim.x);
    if (it.g >= a.G) continue;
    if constexpr (LV == 2) {
      if (a.inverse) {
        bfly16_rt(r[0], r[1], kf[0], true);
        bfly16_rt(r[2], r[3], kf[1], true);
        bfly16_rt(r[0], r[2], kf[2], true);
        bfly16_rt(r[1], r[3], kf[2], true);
      } else {
        bfly16_rt(r[0], r[2], kf[2], false);
        bfly16_rt(r[1], r[3], kf[2], false);
        bfly16_rt(r[0], r[1], kf[0], false);
        bfly16_rt(r[2], r[3], kf[1], false);
      }
    } else {
      bfly16_rt(r[0], r[1], kf[0], a.inverse != 0);
    }
    const uint64_t db = (uint64_t)it.s * a.dst_regs + a.dst_start;
#pragma unroll
    for (int q = 0; q < NR; q++) store_reg16(a.dst + (db + i0 + q * h) * a.G * 16, a.G, it.g, r[q]);
  }
}

// Radix-16 pass with the runtime-constant networks: levels L .. L+3 of one item's 16
// registers {i0 + q h : q = 0..15}, four warps per CTA. The item's registers are staged
// in shared memory (32 KiB); warp w runs two levels on one grouping of four registers,
// the CTA exchanges through shared memory, and warp w runs the other two levels on the
// other grouping and stores. Inverse: levels L, L+1 on registers 4w .. 4w+3, then L+2,
// L+3 on w, w+4, w+8, w+12; forward: the mirror image. The constant of level L+l for the
// block at register i0 + q h is entry R - (R >> (L+l)) + ((grp >> L) << (3-l)) + (q >> (l+1)),
// as in the radix-4 kernels. Each item reads and writes the scratch once for four levels
// instead of two.
__global__ void __launch_bounds__(128, 4) fft16_pass16_kernel(const Fft16PassArgs a) {
  __shared__ __align__(16) uint4 stage[16][4][32];  // [register][16-byte quarter][lane]
  const uint32_t R = a.R, L = a.level, h = 1u << L;
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t chunks = (uint32_t)((a.G + 31) / 32), tasks = a.n_stripes * chunks;
  const uint32_t items = (R >> 4) * tasks;
  auto cidx = [&](uint32_t l, uint32_t gb, uint32_t q) {
    return R - (R >> (L + l)) + (gb << (3 - l)) + (q >> (l + 1));
  };
  for (uint32_t item = blockIdx.x; item < items; item += gridDim.x) {
    const uint32_t grp = item / tasks, task = item - grp * tasks;
    const uint32_t s = task / chunks;
    const uint64_t gbase = (uint64_t)(task - s * chunks) * 32;
    const uint32_t gb = grp >> L, i0 = gb * (h << 4) + (grp & (h - 1));
    const uint64_t rstride = (uint64_t)h * a.G * 16;  // words between the item's registers
    const uint32_t *sbase = a.src + ((uint64_t)s * a.src_regs + a.src_start + i0) * a.G * 16;
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const uint32_t idx = threadIdx.x + 128u * i;
      const uint32_t ln = idx & 31u, c = (idx >> 5) & 3u, q = idx >> 7;
      const uint64_t g = gbase + ln;
      if (g < a.G) cp_async16(&stage[q][c][ln], quarter16(sbase + q * rstride, a.G, g, c));
    }
    cp_async_commit();
    // This warp's six constants (two levels per grouping), loaded while the copies land.
    uint32_t ka[3], kb[3];
    if (a.inverse) {
      ka[0] = const_factors(a.cols, cidx(0, gb, 4 * w));
      ka[1] = const_factors(a.cols, cidx(0, gb, 4 * w + 2));
      ka[2] = const_factors(a.cols, cidx(1, gb, 4 * w));
      kb[0] = const_factors(a.cols, cidx(2, gb, w));
      kb[1] = const_factors(a.cols, cidx(2, gb, w + 8));
      kb[2] = const_factors(a.cols, cidx(3, gb, w));
    } else {
      ka[0] = const_factors(a.cols, cidx(2, gb, w));
      ka[1] = const_factors(a.cols, cidx(2, gb, w + 8));
      ka[2] = const_factors(a.cols, cidx(3, gb, w));
      kb[0] = const_factors(a.cols, cidx(0, gb, 4 * w));
      kb[1] = const_factors(a.cols, cidx(0, gb, 4 * w + 2));
      kb[2] = const_factors(a.cols, cidx(1, gb, 4 * w));
    }
    cp_async_wait_all();
    __syncthreads();
    // First grouping: inverse 4w + j, forward w + 4j.
    const uint32_t qa = a.inverse ? 4 * w : w, sa = a.inverse ? 1 : 4;
    const uint32_t qb = a.inverse ? w : 4 * w, sb = a.inverse ? 4 : 1;
    Reg16 r[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const uint4 v = stage[qa + j * sa][c][lane];
        r[j][4 * c] = v.x, r[j][4 * c + 1] = v.y, r[j][4 * c + 2] = v.z, r[j][4 * c + 3] = v.w;
      }
    if (a.inverse) {
      bfly16_rt(r[0], r[1], ka[0], true);
      bfly16_rt(r[2], r[3], ka[1], true);
      bfly16_rt(r[0], r[2], ka[2], true);
      bfly16_rt(r[1], r[3], ka[2], true);
    } else {
      bfly16_rt(r[0], r[2], ka[2], false);
      bfly16_rt(r[1], r[3], ka[2], false);
      bfly16_rt(r[0], r[1], ka[0], false);
      bfly16_rt(r[2], r[3], ka[1], false);
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int c = 0; c < 4; c++)
        stage[qa + j * sa][c][lane] = make_uint4(r[j][4 * c], r[j][4 * c + 1], r[j][4 * c + 2], r[j][4 * c + 3]);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const uint4 v = stage[qb + j * sb][c][lane];
        r[j][4 * c] = v.x, r[j][4 * c + 1] = v.y, r[j][4 * c + 2] = v.z, r[j][4 * c + 3] = v.w;
      }
    __syncthreads();  // the stage is free for the next item's copies
    if (a.inverse) {
      bfly16_rt(r[0], r[1], kb[0], true);
      bfly16_rt(r[2], r[3], kb[1], true);
      bfly16_rt(r[0], r[2], kb[2], true);
      bfly16_rt(r[1], r[3], kb[2], true);
    } else {
      bfly16_rt(r[0], r[2], kb[2], false);
      bfly16_rt(r[1], r[3], kb[2], false);
      bfly16_rt(r[0], r[1], kb[0], false);
      bfly16_rt(r[2], r[3], kb[1], false);
    }
    const uint64_t g = gbase + lane;
    if (g < a.G) {
      const uint64_t db = (uint64_t)s * a.dst_regs + a.dst_start + i0;
#pragma unroll
      for (int j = 0; j < 4; j++) store_reg16(a.dst + (db + (uint64_t)(qb + j * sb) * h) * a.G * 16, a.G, g, r[j]);
    }
  }
}

// Radix-2^V passes (V = 5 here; fft16_pass16_kernel is the V = 4 case written out) with
// the runtime-constant networks: levels L .. L+V-1 of
// one item's 2^V registers {i0 + q h : q < 2^V}, 2^(V-2) warps per CTA. The item's
// registers are staged in shared memory (2^V x 2 KiB); the levels run in stages of two
// (and one last single level for V = 5), each warp taking four registers per stage, and
// the CTA exchanges through shared memory between stages; the last stage stores to the
// destination. A two-level stage at relative level l takes registers base + j 2^l (j <
// 4), base = warp w with two zero bits inserted at bit l; the single level 4 of V = 5
// takes the pairs (2w, 2w + 16) and (2w + 1, 2w + 17). Inverse: stages by ascending
// level; forward: the mirror image. The constant of level L+l for the block at register
// i0 + q h is entry R - (R >> (L+l)) + ((grp >> L) << (V-1-l)) + (q >> (l+1)), as in the
// radix-4 kernels. Each item reads and writes the scratch once for V levels.
template <int V>
struct Fft16Wide {
  static constexpr int kWarps = 1 << (V - 2), kThreads = 32 * kWarps, kRegs = 1 << V;
  static constexpr int kSmem = kRegs * 4 * 32 * 16;
};

template <int V>
__global__ void __launch_bounds__(Fft16Wide<V>::kThreads, 8 / (1 << (V - 3)))
    fft16_pass_wide_kernel(const Fft16PassArgs a) {
  using Sh = Fft16Wide<V>;
  extern __shared__ __align__(16) uint4 wstage[];  // [register][16-byte quarter][lane]
  const uint32_t R = a.R, L = a.level, h = 1u << L;
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t chunks = (uint32_t)((a.G + 31) / 32), tasks = a.n_stripes * chunks;
  const uint32_t items = (R >> V) * tasks;
  auto cidx = [&](uint32_t l, uint32_t gb, uint32_t q) {
    return R - (R >> (L + l)) + (gb << (V - 1 - l)) + (q >> (l + 1));
  };
  auto slot = [&](uint32_t q, uint32_t c) -> uint4 & { return wstage[(q * 4 + c) * 32 + lane]; };
  auto load4 = [&](Reg16 (&r)[4], const uint32_t (&q)[4]) {
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const uint4 v = slot(q[j], c);
        r[j][4 * c] = v.x, r[j][4 * c + 1] = v.y, r[j][4 * c + 2] = v.z, r[j][4 * c + 3] = v.w;
      }
  };
  auto save4 = [&](const Reg16 (&r)[4], const uint32_t (&q)[4]) {
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int c = 0; c < 4; c++) slot(q[j], c) = make_uint4(r[j][4 * c], r[j][4 * c + 1], r[j][4 * c + 2], r[j][4 * c + 3]);
  };
  // The registers and constants of this warp in stage t (in inverse order: t = 0 the
  // levels 0, 1; t = 1 the levels 2, 3; t = 2 the level 4 of V = 5).
  struct Stage {
    uint32_t q[4];
    uint32_t k[3];
  };
  auto stage_of = [&](int t, uint32_t gb) {
    Stage st;
    if (t < 2) {
      const uint32_t l = 2 * t, base = (w & ((1u << l) - 1)) | ((w >> l) << (l + 2));
#pragma unroll
      for (int j = 0; j < 4; j++) st.q[j] = base + ((uint32_t)j << l);
      st.k[0] = const_factors(a.cols, cidx(l, gb, base));
      st.k[1] = const_factors(a.cols, cidx(l, gb, base + (2u << l)));
      st.k[2] = const_factors(a.cols, cidx(l + 1, gb, base));
    } else {
      st.q[0] = 2 * w, st.q[1] = 2 * w + 16, st.q[2] = 2 * w + 1, st.q[3] = 2 * w + 17;
      st.k[0] = st.k[1] = st.k[2] = const_factors(a.cols, cidx(4, gb, 2 * w));
    }
    return st;
  };
  auto run = [&](int t, Reg16 (&r)[4], const Stage &st) {
    if (t == 2) {
      bfly16_rt(r[0], r[1], st.k[0], a.inverse != 0);
      bfly16_rt(r[2], r[3], st.k[0], a.inverse != 0);
    } else if (a.inverse) {
      bfly16_rt(r[0], r[1], st.k[0], true);
      bfly16_rt(r[2], r[3], st.k[1], true);
      bfly16_rt(r[0], r[2], st.k[2], true);
      bfly16_rt(r[1], r[3], st.k[2], true);
    } else {
      bfly16_rt(r[0], r[2], st.k[2], false);
      bfly16_rt(r[1], r[3], st.k[2], false);
      bfly16_rt(r[0], r[1], st.k[0], false);
      bfly16_rt(r[2], r[3], st.k[1], false);
    }
  };
  constexpr int NS = V == 5 ? 3 : 2;
  for (uint32_t item = blockIdx.x; item < items; item += gridDim.x) {
    const uint32_t grp = item / tasks, task = item - grp * tasks;
    const uint32_t s = task / chunks;
    const uint64_t gbase = (uint64_t)(task - s * chunks) * 32;
    const uint32_t gb = grp >> L, i0 = gb * (h << V) + (grp & (h - 1));
    const uint64_t rstride = (uint64_t)h * a.G * 16;  // words between the item's registers
    const uint32_t *sbase = a.src + ((uint64_t)s * a.src_regs + a.src_start + i0) * a.G * 16;
#pragma unroll
    for (int i = 0; i < Sh::kRegs * 4 * 32 / Sh::kThreads; i++) {
      const uint32_t idx = threadIdx.x + (uint32_t)Sh::kThreads * i;
      const uint32_t ln = idx & 31u, c = (idx >> 5) & 3u, q = idx >> 7;
      const uint64_t g = gbase + ln;
      if (g < a.G) cp_async16(&wstage[idx], quarter16(sbase + q * rstride, a.G, g, c));
    }
    cp_async_commit();
    Stage st = stage_of(a.inverse ? 0 : NS - 1, gb);  // constants load while the copies land
    cp_async_wait_all();
    __syncthreads();
    Reg16 r[4];
#pragma unroll
    for (int n = 0; n < NS; n++) {
      const int t = a.inverse ? n : NS - 1 - n;
      if (n > 0) st = stage_of(t, gb);
      load4(r, st.q);
      if (n + 1 < NS) {
        run(t, r, st);
        save4(r, st.q);
        __syncthreads();
      }
    }
    __syncthreads();  // every warp has read its last stage: the next item may overwrite it
    {
      const int t = a.inverse ? NS - 1 : 0;
      run(t, r, st);
      const uint64_t g = gbase + lane;
      if (g < a.G) {
        const uint64_t db = (uint64_t)s * a.dst_regs + a.dst_start + i0;
#pragma unroll
        for (int j = 0; j < 4; j++) store_reg16(a.dst + (db + (uint64_t)st.q[j] * h) * a.G * 16, a.G, g, r[j]);
      }
    }
  }
}

// Which pass kernels run (rs_set_fft16_pass): 2 (default) the runtime-constant networks
// in passes of four levels (radix 16 through shared memory), of five for one pass when
// the level count is odd, then of two; 1 radix-4 passes (and an odd top level alone)
// only; 0 the mask tables. The scaling, glue and store kernels take the runtime-constant
// networks for 1 and 2. Measured on B200 (2 KiB shards), 2 against 1: (1024,1024) x 64
// stripes 411 -> 463 GB/s, (4096,12288) x 2 240 -> 312 GB/s; the five-level pass for odd
// counts against a four-level and a one-level pass: (512,512) 476 -> 498 GB/s,
// (2048,2048) 371 -> 387 GB/s (at (1024,1024), 5 + 5 levels ran 2% slower than 4 + 4 + 2).
inline int &fft16_pass_variant() {
  static int v = 2;
  return v;
}
inline bool fft16_rt() { return fft16_pass_variant() >= 1; }

// The passes of a transform of 2^lg registers, in launch order: (lowest level, levels).
// Inverse: levels ascending; forward: the same passes in reverse order.
inline int fft16_passes(int lg, bool inverse, int (*out)[2]) {
  int n = 0, L = 0;
  if (fft16_pass_variant() == 2) {
    if (lg >= 5 && lg % 2 == 1) out[n][0] = L, out[n++][1] = 5, L = 5;
    for (; L + 3 < lg; L += 4) out[n][0] = L, out[n++][1] = 4;
  }
  for (; L + 1 < lg; L += 2) out[n][0] = L, out[n++][1] = 2;
  if (L < lg) out[n][0] = L, out[n++][1] = 1;
  if (!inverse)
    for (int i = 0; i < n / 2; i++)
      for (int j = 0; j < 2; j++) std::swap(out[i][j], out[n - 1 - i][j]);
  return n;
}

// Launch of a pass: one warp per CTA, up to 16 per SM, persistent over the items.
inline cudaError_t launch_fft16_pass(const Fft16PassArgs &a, int lv, cudaStream_t st) {
  const uint64_t tasks = (uint64_t)a.n_stripes * ((a.G + 31) / 32), items = ((uint64_t)a.R >> lv) * tasks;
  if (items >= (1ull << 32)) return cudaErrorInvalidValue;
  if (lv == 4 || lv == 5) {  // 512 threads per SM (registers): 4 CTAs of 128 or 2 of 256
    const int ctas = lv == 4 ? 4 : 2;
    const unsigned gw = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(items, (uint64_t)sm_count() * ctas));
    if (lv == 4) {
      fft16_pass16_kernel<<<gw, 128, 0, st>>>(a);
    } else {
      auto kern = fft16_pass_wide_kernel<5>;
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Fft16Wide<5>::kSmem);
      if (e != cudaSuccess) return e;
      kern<<<gw, Fft16Wide<5>::kThreads, Fft16Wide<5>::kSmem, st>>>(a);
    }
    return cudaGetLastError();
  }
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(items, (uint64_t)sm_count() * 16));
  if (fft16_rt()) {
    if (lv == 2)
      fft16_pass_rt_kernel<2><<<grid, 32, 0, st>>>(a);
    else
      fft16_pass_rt_kernel<1><<<grid, 32, 0, st>>>(a);
  } else if (lv == 2) {
    fft16_pass_kernel<2><<<grid, 32, 0, st>>>(a);
  } else {
    fft16_pass_kernel<1><<<grid, 32, 0, st>>>(a);
  }
  return cudaGetLastError();
}

// Shard bytes -> bit planes: row r of stripe s (low plane [0,N), high plane [N,2N)),
// symbol groups g0 .. g0+G-1, into scratch register r; symbols past N read as zero.
// Rows are strided, or (one stripe) taken from the device pointer table in_ptrs.
__global__ void __launch_bounds__(kFft16Threads)
    fft16_load_kernel(const uint8_t *in_base, uint64_t in_row, uint64_t in_stripe, const uint8_t *const *in_ptrs,
                      uint32_t rows, uint64_t N, uint64_t g0, uint64_t G, uint32_t n_stripes, uint32_t R,
                      uint32_t *dst) {
  const uint64_t total = (uint64_t)n_stripes * rows * G;
  for (uint64_t t = (uint64_t)blockIdx.x * kFft16Threads + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * kFft16Threads) {
    const uint64_t g = t % G, sr = t / G;
    const uint64_t r = sr % rows, s = sr / rows;
    const uint8_t *row = in_ptrs ? in_ptrs[r] : in_base + s * in_stripe + r * in_row;
    const uint64_t col = (g0 + g) * 32, remain = N - col;
    uint32_t lo[8], hi[8];
    load32(row + col, remain, lo);
    load32(row + N + col, remain, hi);
    bit_transpose(lo);
    bit_transpose(hi);
    Reg16 x;
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = lo[i], x[8 + i] = hi[i];
    store_reg16(dst + (s * R + r) * G * 16, G, g, x);
  }
}

// Bit planes -> shard bytes: scratch registers [0, rows) of each stripe (R per stripe)
// into symbol groups g0 .. g0+G-1 of output rows out_base + s * out_stripe + r * out_row,
// or (one stripe) out_ptrs[r].
__global__ void __launch_bounds__(kFft16Threads)
    fft16_store_kernel(const uint32_t *src, uint32_t R, uint32_t rows, uint64_t N, uint64_t g0, uint64_t G,
                       uint32_t n_stripes, uint8_t *out_base, uint64_t out_row, uint64_t out_stripe,
                       uint8_t *const *out_ptrs) {
  const uint64_t total = (uint64_t)n_stripes * rows * G;
  for (uint64_t t = (uint64_t)blockIdx.x * kFft16Threads + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * kFft16Threads) {
    const uint64_t g = t % G, sr = t / G;
    const uint64_t r = sr % rows, s = sr / rows;
    Reg16 x;
    load_reg16(src + (s * R + r) * G * 16, G, g, x);
    uint32_t lo[8], hi[8];
#pragma unroll
    for (int i = 0; i < 8; i++) lo[i] = x[i], hi[i] = x[8 + i];
    bit_transpose(lo);
    bit_transpose(hi);
    uint8_t *row = out_ptrs ? out_ptrs[r] : out_base + s * out_stripe + r * out_row;
    const uint64_t col = (g0 + g) * 32, remain = N - col;
    store32(row + col, remain, lo);
    store32(row + N + col, remain, hi);
  }
}

// Glue of the interpolation of k points that are not a power of two (src/fft.rs:198-239):
// dst[dst_start + i] ^= c * src[src_start + i] for i < count, per stripe; with
// cols == nullptr the constant is 1 (plain XOR).
// RT: the constant goes through the compiled nibble networks (mul16_acc_rt) instead of
// shared-memory masks; it is the same for every thread of the launch.
template <bool RT>
__global__ void __launch_bounds__(kFft16Threads)
    fft16_mulxor_kernel(const uint32_t *src, uint32_t src_regs, uint32_t src_start, uint32_t *dst, uint32_t dst_regs,
                        uint32_t dst_start, uint32_t count, uint64_t G, uint32_t n_stripes, const uint16_t *cols) {
  __shared__ __align__(16) uint32_t mk[RT ? 1 : kMask16];
  uint32_t kf = 0;
  if (cols) {
    if constexpr (RT) {
      kf = const_factors(cols, 0);
    } else {
      for (uint32_t t = threadIdx.x; t < kMask16; t += blockDim.x) mk[t] = mask16(cols, t);
      __syncthreads();
    }
  }
  const uint64_t total = (uint64_t)n_stripes * count * G;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t g = t % G, si = t / G;
    const uint64_t i = si % count, s = si / count;
    Reg16 x, y;
    load_reg16(src + (s * src_regs + src_start + i) * G * 16, G, g, x);
    uint32_t *d = dst + (s * dst_regs + dst_start + i) * G * 16;
    load_reg16(d, G, g, y);
    if (!cols)
      xor16(y, x);
    else if constexpr (RT)
      mul16_acc_rt(y, x, kf);
    else
      mul16_acc(y, x, mk);
    store_reg16(d, G, g, y);
  }
}

// ---- erasure decoding on the FFT route (one stripe, shards through a pointer table) ----
//
// Masks of one constant from its table entry into shared memory (all threads of the CTA).
__device__ __forceinline__ void masks_from_cols(uint32_t *mk, const uint16_t *cols) {
  for (uint32_t t = threadIdx.x; t < kMask16; t += blockDim.x) mk[t] = mask16(cols, t);
}

// d = M * s (product only)
__device__ __forceinline__ void mul16_set(Reg16 &d, const Reg16 &s, const uint32_t *m) {
#pragma unroll
  for (int b = 0; b < 16; b++) d[b] = 0;
  mul16_acc(d, s, m);
}

// Register r of C (one CTA per register, N of them): the shard at point r times its
// constant c_r (cols + 16 r), or zero where c_r = 0 (erased points and padding past
// the last shard, whose pointer is not read). Symbol groups g0 .. g0+G-1.
template <bool RT>
__global__ void __launch_bounds__(kFft16Threads)
    fft16_scale_load_kernel(const uint8_t *const *ptrs, const uint16_t *cols, uint32_t n, uint64_t Nsym,
                            uint64_t g0, uint64_t G, uint32_t *dst) {
  __shared__ __align__(16) uint32_t mk[RT ? 1 : kMask16];
  __shared__ int live;
  const uint32_t r = blockIdx.x;
  const uint16_t *c = cols + 16 * (uint64_t)r;
  if (threadIdx.x == 0) {
    int any = 0;
    for (int p = 0; p < 16; p++) any |= c[p];
    live = r < n && any;
  }
  uint32_t kf = 0;
  if constexpr (RT)
    kf = const_factors(c, 0);
  else
    masks_from_cols(mk, c);
  __syncthreads();
  for (uint64_t g = threadIdx.x; g < G; g += blockDim.x) {
    Reg16 y;
    if (live) {
      const uint8_t *row = ptrs[r];
      const uint64_t col = (g0 + g) * 32, remain = Nsym - col;
      uint32_t lo[8], hi[8];
      load32(row + col, remain, lo);
      load32(row + Nsym + col, remain, hi);
      bit_transpose(lo);
      bit_transpose(hi);
      Reg16 x;
#pragma unroll
      for (int i = 0; i < 8; i++) x[i] = lo[i], x[8 + i] = hi[i];
      if constexpr (RT) {
#pragma unroll
        for (int i = 0; i < 16; i++) y[i] = 0;
        mul16_acc_rt(y, x, kf);
      } else {
        mul16_set(y, x, mk);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 16; i++) y[i] = 0;
    }
    store_reg16(dst + (uint64_t)r * G * 16, G, g, y);
  }
}

// Formal derivative in the novel basis (one CTA per output register j < N):
// D_j = sum over levels t with bit t of j clear of kappa_t * C_{j + 2^t}, kappa_t the
// constant derivative of the normalised subspace polynomial of level t.
template <bool RT>
__global__ void __launch_bounds__(kFft16Threads)
    fft16_derivative_kernel(const uint32_t *src, uint32_t *dst, const uint16_t *kcols, uint32_t lg, uint64_t G) {
  __shared__ __align__(16) uint32_t mk[RT ? 1 : 16][RT ? 1 : kMask16];
  const uint32_t j = blockIdx.x;
  if constexpr (!RT) {
    for (uint32_t t = threadIdx.x; t < lg * kMask16; t += blockDim.x) {
      const uint32_t c = t / kMask16, w = t - c * kMask16;
      mk[c][w] = mask16(kcols + 16 * c, w);
    }
    __syncthreads();
  }
  for (uint64_t g = threadIdx.x; g < G; g += blockDim.x) {
    Reg16 acc;
#pragma unroll
    for (int i = 0; i < 16; i++) acc[i] = 0;
    for (uint32_t t = 0; t < lg; t++) {
      if ((j >> t) & 1) continue;
      Reg16 x;
      load_reg16(src + (uint64_t)(j + (1u << t)) * G * 16, G, g, x);
      if constexpr (RT)
        mul16_acc_rt(acc, x, const_factors(kcols, t));
      else
        mul16_acc(acc, x, mk[t]);
    }
    store_reg16(dst + (uint64_t)j * G * 16, G, g, acc);
  }
}

// Rebuilt shards (one CTA per target i): point rows[i] of W times its constant
// (tcols + 16 i), back to bytes at ptrs[rows[i]].
template <bool RT>
__global__ void __launch_bounds__(kFft16Threads)
    fft16_scale_store_kernel(const uint32_t *src, const uint32_t *rows, const uint16_t *tcols,
                             uint8_t *const *ptrs, uint64_t Nsym, uint64_t g0, uint64_t G) {
  __shared__ __align__(16) uint32_t mk[RT ? 1 : kMask16];
  const uint32_t i = blockIdx.x, r = rows[i];
  uint32_t kf = 0;
  if constexpr (RT)
    kf = const_factors(tcols, i);
  else
    masks_from_cols(mk, tcols + 16 * (uint64_t)i);
  __syncthreads();
  uint8_t *row = ptrs[r];
  for (uint64_t g = threadIdx.x; g < G; g += blockDim.x) {
    Reg16 x, y;
    load_reg16(src + (uint64_t)r * G * 16, G, g, x);
    if constexpr (RT) {
#pragma unroll
      for (int b = 0; b < 16; b++) y[b] = 0;
      mul16_acc_rt(y, x, kf);
    } else {
      mul16_set(y, x, mk);
    }
    uint32_t lo[8], hi[8];
#pragma unroll
    for (int b = 0; b < 8; b++) lo[b] = y[b], hi[b] = y[8 + b];
    bit_transpose(lo);
    bit_transpose(hi);
    const uint64_t col = (g0 + g) * 32, remain = Nsym - col;
    store32(row + col, remain, lo);
    store32(row + Nsym + col, remain, hi);
  }
}

}  // namespace rsb
