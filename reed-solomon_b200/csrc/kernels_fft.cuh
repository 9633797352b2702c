// FFT-route encode kernels: the Lin-Chung-Han additive FFT of the reference's
// generated programs (src/fft.rs, src/fft_programs.rs), bitsliced for CUDA cores.
//
// For a (K, K) shape with K a power of two the reference's encode program is an
// inverse transform of the K data rows on the coset {0..K-1} (interpolation,
// src/fft.rs:198-203) followed by a forward transform on the coset {K..2K-1}
// (src/fft.rs:330-343); its outputs are the K parity rows in order. The kernels run the
// same transform pair over a searched basis of {0..K-1} (fftc::fft_basis below), which
// yields the same parity bytes in another register order with cheaper constants.
//
// Bitslicing. A thread's 32 byte columns of one shard (8 words) are transposed into
// 8 bit planes (32 bits each); the transpose is its own inverse, so the same network
// turns parity planes back into bytes. Multiplying a register by a constant c is then
// the GF(2) matrix of c applied to the planes: plane b of c*x is the XOR of planes b'
// of x for which bit b of c*2^b' is set. With c known at compile time that is a short
// fixed XOR network (about 12 three-input LOP3 operations per multiply-accumulate on
// 32 columns, on average over the RS(32,32) transform's constants), instead of a table
// lookup per byte.
//
// Lane pairs. K registers x 8 planes do not fit one thread for K = 32, so a lane pair
// shares each 32-column group: lane h holds program registers 2j + h. At level l >= 1 a
// butterfly pairs registers i and i + 2^l (same lane) and its constant
// WHAT_l(beta ^ P(base)) depends only on register bits above l, never on bit 0, so both
// lanes run the same straight-line code with the same constants. Level 0 pairs 2j with
// 2j + 1: the lanes swap the register with one shuffle per plane and each keeps its
// own half of the butterfly.
#pragma once

#include <cstdint>
#include <type_traits>
#include <utility>

#include "kernels_matrix.cuh"
#include "tuning.hpp"

namespace rsb {

namespace fftc {

constexpr uint8_t xt(uint8_t v) { return (uint8_t)((v << 1) ^ ((v & 0x80) ? 0x1d : 0)); }

constexpr uint8_t gmul(uint8_t a, uint8_t b) {
  uint8_t r = 0;
  for (int i = 0; i < 8; i++) {
    if (b & 1) r ^= a;
    a = xt(a);
    b >>= 1;
  }
  return r;
}

template <int K>
constexpr int log2k() {
  int l = 0;
  while ((1 << l) < K) l++;
  return l;
}

// Subspace basis of the transform. The parity values do not depend on how the additive
// FFT enumerates V = {0 .. K-1}: for any ordered basis v_0 .. v_{n-1} of V, register i of
// the inverse transform holds point P(i) = XOR of v_j over the bits j of i, and for any
// beta in {K .. 2K-1} register i of the forward transform holds point beta ^ P(i). The
// reference's programs use v_j = 2^j and beta = K; the bases below, found by
// fft_basis_search.c, give butterfly constants with cheaper XOR networks (13% fewer
// LOP3s in the constant multiplies at K = 32, 20% at K = 16). With lane groups of 2^W
// lanes, v_0 .. v_{W-1} are single bits and the other vectors are clear of them, so a
// lane's shard index is a compile-time part plus a per-lane part.
struct FftBasis {
  uint8_t v[8];
  uint8_t beta;
};

constexpr FftBasis fft_basis(int K, int W) {
  switch (K) {
    case 2: return {{1}, 2};
    case 4: return {{2, 1}, 4};
    case 8: return {{4, 2, 1}, 8};
    case 16: return W == 1 ? FftBasis{{8, 3, 2, 4}, 16} : FftBasis{{4, 2, 9, 1}, 16};
    case 32: return W == 1 ? FftBasis{{8, 19, 4, 6, 1}, 32} : FftBasis{{4, 2, 1, 8, 24}, 32};
    case 64: return W == 2 ? FftBasis{{2, 4, 17, 41, 32, 16}, 68} : FftBasis{{2, 4, 1, 8, 40, 24}, 68};
    default: return W == 3 ? FftBasis{{32, 64, 16, 3, 8, 4, 10}, 128} : FftBasis{{32, 16, 8, 64, 7, 3, 6}, 128};
  }
}

// The basis spans {0 .. K-1}, its lane vectors are single bits, the rest avoid them, and
// beta lies in {K .. 2K-1}.
constexpr bool fft_basis_ok(int K, int W) {
  const FftBasis b = fft_basis(K, W);
  int n = 0, lanes = 0;
  while ((1 << n) < K) n++;
  bool seen[256] = {};
  for (int i = 0; i < K; i++) {
    int p = 0;
    for (int j = 0; j < n; j++)
      if ((i >> j) & 1) p ^= b.v[j];
    if (p >= K || seen[p]) return false;
    seen[p] = true;
  }
  for (int j = 0; j < W; j++) {
    if (b.v[j] & (b.v[j] - 1)) return false;
    lanes |= b.v[j];
  }
  for (int j = W; j < n; j++)
    if (b.v[j] & lanes) return false;
  return b.beta >= K && b.beta < 2 * K;
}

struct What {
  uint8_t v[8][256];  // v[l][x]: normalised subspace polynomial of level l at x
  uint8_t p[128];     // p[i] = P(i)
};

// W_0(x) = x, W_{j+1}(x) = W_j(x) (W_j(x) + W_j(v_j)), each level scaled so that its value
// at v_j is 1.
constexpr What make_what(FftBasis b, int n) {
  What w{};
  uint8_t raw[8][256] = {};
  for (int x = 0; x < 256; x++) raw[0][x] = (uint8_t)x;
  for (int j = 0; j + 1 < n; j++) {
    const uint8_t pivot = raw[j][b.v[j]];
    for (int x = 0; x < 256; x++) raw[j + 1][x] = gmul(raw[j][x], (uint8_t)(raw[j][x] ^ pivot));
  }
  for (int j = 0; j < n; j++) {
    uint8_t pivot = raw[j][b.v[j]], inv = 0;
    for (int c = 1; c < 256; c++)
      if (gmul(pivot, (uint8_t)c) == 1) {
        inv = (uint8_t)c;
        break;
      }
    for (int x = 0; x < 256; x++) w.v[j][x] = gmul(raw[j][x], inv);
  }
  for (int i = 0; i < (1 << n); i++) {
    uint8_t p = 0;
    for (int j = 0; j < n; j++)
      if ((i >> j) & 1) p ^= b.v[j];
    w.p[i] = p;
  }
  return w;
}

template <int K, int W>
inline constexpr What kWhat = make_what(fft_basis(K, W), log2k<K>());

// Bit b of c * 2^bp: entry (b, bp) of the GF(2) matrix of multiply-by-c.
constexpr bool mbit(uint8_t c, int b, int bp) { return (gmul(c, (uint8_t)(1u << bp)) >> b) & 1; }

template <int B, int E, class F>
__device__ __forceinline__ void static_for(F &&f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

using Reg = uint32_t[8];

// d ^= C * s
template <uint8_t C>
__device__ __forceinline__ void mul_acc(Reg &d, const Reg &s) {
  static_for<0, 8>([&](auto b) {
    uint32_t acc = d[b];
    static_for<0, 8>([&](auto bp) {
      if constexpr (mbit(C, decltype(b)::value, decltype(bp)::value)) acc ^= s[bp];
    });
    d[b] = acc;
  });
}

// d = C * s
template <uint8_t C>
__device__ __forceinline__ void mul_set(Reg &d, const Reg &s) {
  static_for<0, 8>([&](auto b) {
    uint32_t acc = 0;
    static_for<0, 8>([&](auto bp) {
      if constexpr (mbit(C, decltype(b)::value, decltype(bp)::value)) acc ^= s[bp];
    });
    d[b] = acc;
  });
}

__device__ __forceinline__ void xor_into(Reg &d, const Reg &s) {
#pragma unroll
  for (int b = 0; b < 8; b++) d[b] ^= s[b];
}

// Three-input XORs in d ^= C*s: ceil(n_b / 2) for output plane b with n_b terms.
constexpr int mul_cost(uint8_t c) {
  if (c <= 1) return c ? 8 : 0;
  int n = 0;
  for (int b = 0; b < 8; b++) {
    int nb = 0;
    for (int bp = 0; bp < 8; bp++) nb += mbit(c, b, bp);
    n += (nb + 1) / 2;
  }
  return n;
}

// lo/hi butterfly with constant C; inverse: hi ^= lo, lo ^= C*hi; forward: lo ^= C*hi,
// hi ^= lo (src/fft.rs:262-283). The forward pair is also hi' = lo ^ (C+1)*hi, lo' =
// hi' ^ hi, used when C+1 has the cheaper network (C = 1 then costs one register XOR).
template <uint8_t C, bool INV>
__device__ __forceinline__ void butterfly(Reg &lo, Reg &hi) {
  if constexpr (INV) {
    xor_into(hi, lo);
    if constexpr (C == 1)
      xor_into(lo, hi);
    else if constexpr (C != 0)
      mul_acc<C>(lo, hi);
  } else if constexpr (C != 0 && mul_cost(C ^ 1) < mul_cost(C)) {
    Reg t;
#pragma unroll
    for (int b = 0; b < 8; b++) t[b] = lo[b];
    if constexpr ((C ^ 1) == 1)
      xor_into(t, hi);
    else if constexpr ((C ^ 1) != 0)
      mul_acc<C ^ 1>(t, hi);
    xor_into(hi, t);
#pragma unroll
    for (int b = 0; b < 8; b++) {
      lo[b] = hi[b];
      hi[b] = t[b];
    }
  } else {
    if constexpr (C == 1)
      xor_into(lo, hi);
    else if constexpr (C != 0)
      mul_acc<C>(lo, hi);
    xor_into(hi, lo);
  }
}

// Lane groups. A group of G = 2^W lanes shares one 32-column group; lane q holds
// program registers i = (j << W) | q in its slots j = 0 .. K/G - 1.
//
// Level L >= W pairs slots j and j + 2^(L-W) within each lane; the butterfly's block
// base has only bits >= W, so its constant WHAT_L(beta ^ P(base)) is the same in every
// lane.
template <int K, int W, int L, int BETA, bool INV>
__device__ __forceinline__ void level_local(Reg (&r)[K >> W]) {
  constexpr int SJ = 1 << (L - W);  // slot stride
  static_for<0, (K >> W)>([&](auto jj) {
    constexpr int j = decltype(jj)::value;
    if constexpr (((j / SJ) & 1) == 0) {
      constexpr int base = (j << W) & ~((2 << L) - 1);
      constexpr uint8_t c = kWhat<K, W>.v[L][BETA ^ kWhat<K, W>.p[base]];
      butterfly<c, INV>(r[j], r[j + SJ]);
    }
  });
}

// d ^= mask & (E * s), mask all-ones or zero (a lane-bit select).
template <uint8_t E>
__device__ __forceinline__ void masked_mul_acc(Reg &d, const Reg &s, uint32_t mask) {
  if constexpr (E != 0) {
    Reg t;
    mul_set<E>(t, s);
#pragma unroll
    for (int b = 0; b < 8; b++) d[b] ^= t[b] & mask;
  }
}

// The lane-dependent part of a cross-lane constant at level L. The block base of
// register (j << W) | q is (j << W) | (q with bits <= L cleared); P and WHAT_L are
// GF(2)-linear, so the constant is WHAT_L(beta ^ P(j << W)) plus WHAT_L(v_t) for every
// lane bit t in (L, W) that is set in q. qm[t] is all-ones when bit t of q is set.
template <int K, int W, int L, int T>
__device__ __forceinline__ void lane_terms(Reg &d, const Reg &s, const uint32_t (&qm)[8]) {
  if constexpr (T < W) {
    masked_mul_acc<kWhat<K, W>.v[L][kWhat<K, W>.p[1 << T]]>(d, s, qm[T]);
    lane_terms<K, W, L, T + 1>(d, s, qm);
  }
}

// Level L < W: the butterfly pairs lanes q and q ^ 2^L. Each lane swaps its register
// with one shuffle per plane and keeps its own half; h1 = bit L of q (1 on the lane
// owning the upper register), h0 = 1 - h1. Lane selects are integer multiply-adds by
// 0/1 so they issue on the FMA pipe, which the LOP3-heavy butterflies leave idle.
template <int K, int W, int L, int BETA, bool INV>
__device__ __forceinline__ void level_cross(Reg (&r)[K >> W], uint32_t q, const uint32_t (&qm)[8]) {
  const uint32_t h1 = (q >> L) & 1, h0 = 1 - h1;
  static_for<0, (K >> W)>([&](auto jj) {
    constexpr int j = decltype(jj)::value;
    constexpr uint8_t c = kWhat<K, W>.v[L][BETA ^ kWhat<K, W>.p[j << W]];
    Reg p;
#pragma unroll
    for (int b = 0; b < 8; b++) p[b] = __shfl_xor_sync(0xffffffffu, r[j][b], 1 << L);
    if constexpr (INV) {
      // hi' = lo ^ hi; lo' = lo ^ c*hi'.
      Reg t, v;
#pragma unroll
      for (int b = 0; b < 8; b++) {
        t[b] = r[j][b] ^ p[b];
        v[b] = r[j][b];
      }
      if constexpr (c == 1)
        xor_into(v, t);
      else if constexpr (c != 0)
        mul_acc<c>(v, t);
      lane_terms<K, W, L, L + 1>(v, t, qm);
#pragma unroll
      for (int b = 0; b < 8; b++) r[j][b] = t[b] * h1 + v[b] * h0;
    } else {
      // lo' = lo ^ c*hi; hi' = hi ^ lo'. Lower lane: own ^ c*p; upper: own ^ p ^ c*own.
      Reg z, u;
#pragma unroll
      for (int b = 0; b < 8; b++) z[b] = r[j][b] * h1 + p[b] * h0;
      if constexpr (c == 1) {
#pragma unroll
        for (int b = 0; b < 8; b++) u[b] = z[b];
      } else if constexpr (c != 0) {
        mul_set<c>(u, z);
      } else {
#pragma unroll
        for (int b = 0; b < 8; b++) u[b] = 0;
      }
      lane_terms<K, W, L, L + 1>(u, z, qm);
#pragma unroll
      for (int b = 0; b < 8; b++) r[j][b] ^= u[b] ^ (p[b] * h1);
    }
  });
}

// With SYNC the CTA meets at a barrier after every level, keeping the warps that
// share a scheduler on the same stretch of straight-line code.
template <bool SYNC>
__device__ __forceinline__ void phase_sync() {
  if constexpr (SYNC) __syncthreads();
}

template <int K, int W, int L, int BETA, bool INV, bool SYNC>
__device__ __forceinline__ void level_any(Reg (&r)[K >> W], uint32_t q, const uint32_t (&qm)[8]) {
  if constexpr (L < W)
    level_cross<K, W, L, BETA, INV>(r, q, qm);
  else
    level_local<K, W, L, BETA, INV>(r);
  phase_sync<SYNC>();
}

// Inverse transform: levels L .. log2(K)-1 ascending.
template <int K, int W, int L, int BETA, bool SYNC>
__device__ __forceinline__ void levels_up(Reg (&r)[K >> W], uint32_t q, const uint32_t (&qm)[8]) {
  if constexpr ((1 << L) < K) {
    level_any<K, W, L, BETA, true, SYNC>(r, q, qm);
    levels_up<K, W, L + 1, BETA, SYNC>(r, q, qm);
  }
}

// Forward transform: levels L .. 0 descending.
template <int K, int W, int L, int BETA, bool SYNC>
__device__ __forceinline__ void levels_down(Reg (&r)[K >> W], uint32_t q, const uint32_t (&qm)[8]) {
  if constexpr (L >= 0) {
    level_any<K, W, L, BETA, false, SYNC>(r, q, qm);
    levels_down<K, W, L - 1, BETA, SYNC>(r, q, qm);
  }
}

}  // namespace fftc

// One step of the 8x8 bit transpose within each byte lane: swaps the high S-bit
// half of every 2S-bit block of a with the low half of b. Shifts are written as
// integer multiplies so they can issue on the FMA pipe beside the LOP3s.
template <int S, uint32_t MLO>
__device__ __forceinline__ void tswap(uint32_t &a, uint32_t &b) {
  uint32_t bs = b * (1u << S);
  uint32_t as = __umulhi(a, 1u << (32 - S));
  uint32_t na = (a & MLO) | (bs & ~MLO);
  uint32_t nb = (b & ~MLO) | (as & MLO);
  a = na;
  b = nb;
}

// 32 bytes (word i holds columns 4i..4i+3) <-> 8 bit planes (plane b, bit 8q+i holds
// bit b of byte q of word i). An involution.
__device__ __forceinline__ void bit_transpose(uint32_t (&w)[8]) {
  tswap<4, 0x0F0F0F0Fu>(w[0], w[4]);
  tswap<4, 0x0F0F0F0Fu>(w[1], w[5]);
  tswap<4, 0x0F0F0F0Fu>(w[2], w[6]);
  tswap<4, 0x0F0F0F0Fu>(w[3], w[7]);
  tswap<2, 0x33333333u>(w[0], w[2]);
  tswap<2, 0x33333333u>(w[1], w[3]);
  tswap<2, 0x33333333u>(w[4], w[6]);
  tswap<2, 0x33333333u>(w[5], w[7]);
  tswap<1, 0x55555555u>(w[0], w[1]);
  tswap<1, 0x55555555u>(w[2], w[3]);
  tswap<1, 0x55555555u>(w[4], w[5]);
  tswap<1, 0x55555555u>(w[6], w[7]);
}

__device__ __forceinline__ void load32(const uint8_t *p, uint64_t remain, uint32_t (&w)[8]) {
  if (remain >= 32 && (((uintptr_t)p & 15u) == 0)) {
    uint4 a = __ldg(reinterpret_cast<const uint4 *>(p));
    uint4 b = __ldg(reinterpret_cast<const uint4 *>(p + 16));
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
    return;
  }
#pragma unroll
  for (int i = 0; i < 8; i++) w[i] = 0;
  int n = remain < 32 ? (int)remain : 32;
  for (int t = 0; t < n; t++) w[t >> 2] |= (uint32_t)p[t] << (8 * (t & 3));
}

__device__ __forceinline__ void store32(uint8_t *p, uint64_t remain, const uint32_t (&w)[8]) {
  if (remain >= 32 && (((uintptr_t)p & 15u) == 0)) {
    *reinterpret_cast<uint4 *>(p) = make_uint4(w[0], w[1], w[2], w[3]);
    *reinterpret_cast<uint4 *>(p + 16) = make_uint4(w[4], w[5], w[6], w[7]);
    return;
  }
  int n = remain < 32 ? (int)remain : 32;
  for (int t = 0; t < n; t++) p[t] = (uint8_t)(w[t >> 2] >> (8 * (t & 3)));
}

// One stripe of a ragged FFT batch: k data rows at in_base, k parity rows at out_base,
// both row_stride apart; its 32-column groups start at group_begin in the flattened
// group space (items sorted by group_begin).
struct FftItem {
  const uint8_t *in_base;
  uint8_t *out_base;
  uint64_t row_stride;
  uint64_t len;
  uint64_t group_begin;
};

struct FftArgs {
  const uint8_t *in_base;
  uint64_t in_row_stride, in_stripe_stride;
  uint8_t *out_base;
  uint64_t out_row_stride, out_stripe_stride;
  uint64_t len;
  uint32_t n_stripes;
  uint32_t groups_per_stripe;  // 32-column groups per stripe
  // Ragged form (items != nullptr): per-stripe geometry, total_groups groups.
  const FftItem *items;
  uint32_t n_items;
  uint64_t total_groups;
  // Pointer-table form: every shard pointer is 16-byte aligned (set by the host).
  int ptrs_aligned;
  // Parity rows to store, 4 words (rows 0..127) per stripe, or per item in the ragged
  // form; null stores every row. Reconstruct uses it to rebuild only the missing parity.
  const uint32_t *store_mask;
  // The same for a single stripe, passed by value (use_store_bits != 0).
  uint32_t store_bits[4];
  int use_store_bits;
  // Ragged form: some item's rows are not 16-byte aligned (chooses the launch shape).
  int items_unaligned;
  // Launch configuration of this launch (the cost model's or a caller's choice), -1 for
  // the shape's current setting: lane-group width (0 narrow, 1 wide) and launch shape
  // (index into kFftVariants).
  int cfg_wide = -1, cfg_variant = -1;
};

__device__ __forceinline__ bool fft_store_row(const FftArgs &a, uint32_t unit, uint32_t row) {
  if (a.store_mask) return (a.store_mask[4 * (uint64_t)unit + (row >> 5)] >> (row & 31)) & 1u;
  if (a.use_store_bits) return (a.store_bits[row >> 5] >> (row & 31)) & 1u;
  return true;
}

// Where one lane pair's 32-column group lives.
struct FftLoc {
  const uint8_t *in0;   // data row 0 (pointer-table form: unused)
  uint8_t *out0;        // parity row 0
  uint64_t in_rs, out_rs;
  uint64_t col, remain;  // remain = 0 past the end
  uint32_t unit;         // stripe (strided form) or item (ragged form)
};

__device__ __forceinline__ FftLoc fft_locate(const FftArgs &a, uint64_t pair) {
  FftLoc l{};
  if (a.items) {
    if (pair >= a.total_groups) return l;
    uint32_t lo = 0, hi = a.n_items;
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (a.items[mid].group_begin <= pair)
        lo = mid;
      else
        hi = mid;
    }
    const FftItem &it = a.items[lo];
    l.unit = lo;
    l.in0 = it.in_base;
    l.out0 = it.out_base;
    l.in_rs = l.out_rs = it.row_stride;
    l.col = (pair - it.group_begin) * 32;
    l.remain = it.len - l.col;
    return l;
  }
  const uint64_t total = (uint64_t)a.n_stripes * a.groups_per_stripe;
  if (pair >= total) return l;
  uint32_t s, g;
  if (total <= 0xffffffffull) {  // 32-bit division: the common case, far cheaper
    s = (uint32_t)pair / a.groups_per_stripe;
    g = (uint32_t)pair - s * a.groups_per_stripe;
  } else {
    s = (uint32_t)(pair / a.groups_per_stripe);
    g = (uint32_t)(pair - (uint64_t)s * a.groups_per_stripe);
  }
  l.unit = s;
  l.in0 = a.in_base + s * a.in_stripe_stride;
  l.out0 = a.out_base + s * a.out_stripe_stride;
  l.in_rs = a.in_row_stride;
  l.out_rs = a.out_row_stride;
  l.col = (uint64_t)g * 32;
  l.remain = a.len - l.col;
  return l;
}

// Launch shapes of the FFT kernel: threads per CTA, CTAs per SM, and whether the CTA
// meets at a barrier after every transform level (see phase_sync).
struct FftVariant {
  int threads, ctas, sync;
};
constexpr FftVariant kFftVariants[] = {{128, 3, 0}, {128, 4, 0}, {128, 2, 0}, {256, 1, 0}};
constexpr int kFftVariantCount = sizeof(kFftVariants) / sizeof(kFftVariants[0]);

// Per-thread staging of one 32-column group in shared memory: shard slot j, half q
// (16 bytes each) of thread t sits at j*slot + q*half + t*16 with half = 16*THREADS,
// so a warp's 16-byte accesses to one (j, q) are contiguous and free of bank conflicts.
template <int THREADS>
struct FftStage {
  static constexpr int kHalf = THREADS * 16;
  static constexpr int kSlot = 2 * kHalf;
};

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
  uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Slow paths, for the last, partial group of a shard and for unaligned rows, are kept
// out of line: the unrolled per-shard code then holds one call instead of a byte loop,
// so these rarely taken paths do not fill the instruction cache.
// Unaligned rows (packed rows whose length is not a multiple of 16). A group that starts
// at least 32 bytes into its row and has at least 48 row bytes from its start is read
// as the three 16-byte aligned blocks around it, which then lie inside the row, and
// shifted into place: 3 vector loads instead of 32 byte loads. o = p mod 16.
static __device__ __forceinline__ void stage32_window(uint8_t *slot, int half, const uint8_t *p) {
  const uint32_t o = (uint32_t)((uintptr_t)p & 15u), q = o >> 2, r = (o & 3u) * 8u;
  const uint4 *blk = reinterpret_cast<const uint4 *>(p - o);
  const uint4 b0 = __ldg(blk), b1 = __ldg(blk + 1), b2 = __ldg(blk + 2);
  const uint32_t w[12] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w, b2.x, b2.y, b2.z, b2.w};
  uint32_t v[9];  // v[i] = w[q + i], selected without indexing registers at run time
#pragma unroll
  for (int i = 0; i < 9; i++) {
    uint32_t x = w[i];
    if (i + 1 < 12) x = q == 1 ? w[i + 1] : x;
    if (i + 2 < 12) x = q == 2 ? w[i + 2] : x;
    if (i + 3 < 12) x = q == 3 ? w[i + 3] : x;
    v[i] = x;
  }
  uint32_t out[8];  // bytes o + 4i .. o + 4i + 3 of the window
#pragma unroll
  for (int i = 0; i < 8; i++) out[i] = __funnelshift_r(v[i], v[i + 1], r);
  *reinterpret_cast<uint4 *>(slot) = make_uint4(out[0], out[1], out[2], out[3]);
  *reinterpret_cast<uint4 *>(slot + half) = make_uint4(out[4], out[5], out[6], out[7]);
}

// Store a whole group (32 bytes) at an unaligned p without touching bytes outside it:
// the group's bytes are placed at offset o of the 48-byte aligned window around p; the
// middle block is one 16-byte store, the two edge blocks go out as the naturally
// aligned words, halfwords and bytes that lie inside the group.
static __device__ __forceinline__ void store32_window(uint8_t *p, uint4 lo, uint4 hi) {
  const uint32_t o = (uint32_t)((uintptr_t)p & 15u), q = o >> 2, r = (o & 3u) * 8u;
  uint8_t *base = p - o;
  const uint32_t in[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
  uint32_t u[12];  // u[j] = in[j - q] (0 outside 0..7)
#pragma unroll
  for (int j = 0; j < 12; j++) {
    uint32_t x = j < 8 ? in[j] : 0u;
    x = q == 1 ? (j >= 1 && j - 1 < 8 ? in[j - 1] : 0u) : x;
    x = q == 2 ? (j >= 2 && j - 2 < 8 ? in[j - 2] : 0u) : x;
    x = q == 3 ? (j >= 3 && j - 3 < 8 ? in[j - 3] : 0u) : x;
    u[j] = x;
  }
  uint32_t W[12];  // window bytes 4i .. 4i + 3
#pragma unroll
  for (int i = 0; i < 12; i++) W[i] = __funnelshift_l(i ? u[i - 1] : 0u, u[i], r);
  // Window bytes [o, o + 32) belong to the group.
#pragma unroll
  for (int i = 0; i < 12; i++) {
    if (i >= 4 && i < 8) continue;  // the middle block, below
    const uint32_t b0 = 4u * i, b1 = b0 + 4u, g0 = o, g1 = o + 32u;
    if (b0 >= g0 && b1 <= g1) {
      *reinterpret_cast<uint32_t *>(base + b0) = W[i];
    } else if (b1 > g0 && b0 < g1) {  // a partial word: bytes [max(b0,g0), min(b1,g1))
      const uint32_t s0 = b0 > g0 ? b0 : g0, s1 = b1 < g1 ? b1 : g1;
      uint32_t x = s0;
      if ((x & 1u) && x < s1) {
        base[x] = (uint8_t)(W[i] >> (8u * (x - b0)));
        x++;
      }
      if (x + 2 <= s1) {
        *reinterpret_cast<uint16_t *>(base + x) = (uint16_t)(W[i] >> (8u * (x - b0)));
        x += 2;
      }
      if (x < s1) base[x] = (uint8_t)(W[i] >> (8u * (x - b0)));
    }
  }
  *reinterpret_cast<uint4 *>(base + 16) = make_uint4(W[4], W[5], W[6], W[7]);
}

// Stage the 32 bytes at p (remain of them valid, col bytes of the row before p) into
// this thread's slot: two async 16-byte copies when aligned and whole, the aligned
// window for interior groups of unaligned rows, else the zero-filled byte path.
static __device__ __noinline__ void stage32_slow(uint8_t *slot, int half, const uint8_t *p, uint64_t remain,
                                                 uint64_t col) {
  if (col >= 32 && remain >= 48) {
    stage32_window(slot, half, p);
  } else {
    uint32_t w[8];
    load32(p, remain, w);
    *reinterpret_cast<uint4 *>(slot) = make_uint4(w[0], w[1], w[2], w[3]);
    *reinterpret_cast<uint4 *>(slot + half) = make_uint4(w[4], w[5], w[6], w[7]);
  }
}

template <int HALF>
__device__ __forceinline__ void stage32(uint8_t *slot, const uint8_t *p, uint64_t remain, uint64_t col) {
  if (remain >= 32 && (((uintptr_t)p & 15u) == 0)) {
    cp_async16(slot, p);
    cp_async16(slot + HALF, p + 16);
  } else {
    stage32_slow(slot, HALF, p, remain, col);
  }
}

// Store the 32 bytes of a group at p (remain of them valid) on the slow paths: one
// out-of-line call, so the unrolled store loops carry a single call per slot.
static __device__ __noinline__ void store32_any(uint8_t *p, uint64_t remain, uint4 lo, uint4 hi) {
  if (remain >= 32) {
    store32_window(p, lo, hi);
  } else {
    const uint32_t w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
    store32(p, remain, w);
  }
}

// Persistent lane groups: round r handles 32-column group grp0 + r*stride of the
// flattened (stripe, group) space; lane q of a group of 2^W lanes holds registers
// (j << W) | q. The next round's 32 bytes per shard are copied into shared memory with
// cp.async while the current round computes. Every lane runs every round (on zeros
// past the end) so each shuffle sees the full warp and every barrier the full CTA.
// UNAL: the instantiation for launches whose rows are not 16-byte aligned (chosen on the
// host). Its lanes on slow rounds park their parity registers in the staging slots and
// store them from one rolled loop, issuing the next round's copies after it: the
// unrolled body then holds no out-of-line calls (+15% on 987-byte packed rows), which
// the aligned instantiation keeps for its rare partial groups, since the extra live
// state cost it 20% when shared.
template <int K, int W, bool PTRS, int THREADS, int CTAS, bool SYNC, bool UNAL = false>
__global__ void __launch_bounds__(THREADS, CTAS)
    fft_kk_kernel(const FftArgs a, const __grid_constant__ PtrTableT<PTRS> pt) {
  extern __shared__ __align__(16) uint8_t stage[];
  using namespace fftc;
  using St = FftStage<THREADS>;
  constexpr int S = K >> W;  // slots per lane
  constexpr int LG = log2k<K>();
  static_assert(fft_basis_ok(K, W), "FFT basis");
  constexpr FftBasis kB = fft_basis(K, W);
  const uint32_t tid = threadIdx.x;
  const uint32_t q = tid & ((1u << W) - 1);
  uint32_t qm[8];
#pragma unroll
  for (int t = 0; t < 8; t++) qm[t] = ((q >> t) & 1) ? 0xffffffffu : 0u;
  // Slot j holds register (j << W) | q: data shard P((j << W) | q) = P(j << W) + pq and
  // parity shard beta ^ P(...) - K = ((beta ^ K ^ P(j << W)) & ~lane bits) + rq.
  uint32_t pq = 0, lane_bits = 0;
#pragma unroll
  for (int t = 0; t < W; t++) {
    pq |= (uint32_t)kB.v[t] & qm[t];
    lane_bits |= kB.v[t];
  }
  const uint32_t rq = (((uint32_t)kB.beta ^ K) & lane_bits) ^ pq;
  auto p_upper = [&](int j) -> uint32_t {  // P(j << W), folded for a compile-time j
    uint32_t p = 0;
#pragma unroll
    for (int t = W; t < LG; t++)
      if ((j >> (t - W)) & 1) p ^= kB.v[t];
    return p;
  };
  auto in_index = [&](int j) -> uint32_t { return p_upper(j) + pq; };
  auto out_index = [&](int j) -> uint32_t { return ((kB.beta ^ K ^ p_upper(j)) & ~lane_bits) + rq; };
  const uint64_t total = a.items ? a.total_groups : (uint64_t)a.n_stripes * a.groups_per_stripe;
  const uint64_t stride = (uint64_t)gridDim.x * (THREADS >> W);
  const uint64_t rounds = (total + stride - 1) / stride;
  const uint64_t grp0 = ((uint64_t)blockIdx.x * THREADS + tid) >> W;
  uint8_t *mine = stage + tid * 16;

  auto in_ptr = [&](const FftLoc &l, int j) -> const uint8_t * {
    if constexpr (PTRS)
      return pt.in[in_index(j)];
    else
      return l.in0 + (uint64_t)in_index(j) * l.in_rs;
  };
  // Whole 32-byte groups on 16-byte aligned rows (every group but a shard's last, for
  // aligned stripes) take the unrolled fast paths; the decision is made once per round.
  auto whole = [&](const FftLoc &l) -> bool {
    if constexpr (PTRS)
      return l.remain >= 32 && a.ptrs_aligned;
    else
      return l.remain >= 32 &&
             ((reinterpret_cast<uintptr_t>(l.in0) | reinterpret_cast<uintptr_t>(l.out0) | l.in_rs | l.out_rs) &
              15u) == 0;
  };
  auto prefetch = [&](uint64_t grp) {
    const FftLoc l = fft_locate(a, grp);
    if (whole(l)) {
#pragma unroll
      for (int j = 0; j < S; j++) {
        const uint8_t *p = in_ptr(l, j) + l.col;
        cp_async16(mine + j * St::kSlot, p);
        cp_async16(mine + j * St::kSlot + St::kHalf, p + 16);
      }
    } else {
#pragma unroll 1
      for (int j = 0; j < S; j++) stage32<St::kHalf>(mine + j * St::kSlot, in_ptr(l, j) + l.col, l.remain, l.col);
    }
    cp_async_commit();
  };

  prefetch(grp0);
  for (uint64_t rd = 0; rd < rounds; rd++) {
    const uint64_t grp = grp0 + rd * stride;
    const FftLoc loc = fft_locate(a, grp);
    const bool live = loc.remain != 0;
    const uint64_t col = loc.col, remain = loc.remain;
    cp_async_wait_all();
    // Bytes -> bit planes in place, one rolled loop: the transpose code appears once
    // instead of once per slot, keeping the loop body small for the instruction cache.
#pragma unroll 1
    for (int j = 0; j < S; j++) {
      uint4 *p0 = reinterpret_cast<uint4 *>(mine + j * St::kSlot);
      uint4 *p1 = reinterpret_cast<uint4 *>(mine + j * St::kSlot + St::kHalf);
      uint4 lo = *p0, hi = *p1;
      uint32_t w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
      bit_transpose(w);
      *p0 = make_uint4(w[0], w[1], w[2], w[3]);
      *p1 = make_uint4(w[4], w[5], w[6], w[7]);
    }
    Reg r[S];
#pragma unroll
    for (int j = 0; j < S; j++) {
      uint4 lo = *reinterpret_cast<const uint4 *>(mine + j * St::kSlot);
      uint4 hi = *reinterpret_cast<const uint4 *>(mine + j * St::kSlot + St::kHalf);
      r[j][0] = lo.x, r[j][1] = lo.y, r[j][2] = lo.z, r[j][3] = lo.w;
      r[j][4] = hi.x, r[j][5] = hi.y, r[j][6] = hi.z, r[j][7] = hi.w;
    }
    if constexpr (UNAL) {
      const bool fast = live && whole(loc), early = fast || !live;
      if (early && rd + 1 < rounds) prefetch(grp + stride);
      phase_sync<SYNC>();
      levels_up<K, W, 0, 0, SYNC>(r, q, qm);
      levels_down<K, W, LG - 1, kB.beta, SYNC>(r, q, qm);
      auto out_row = [&](int j) -> uint8_t * {
        if constexpr (PTRS)
          return pt.out[out_index(j)];
        else
          return loc.out0 + (uint64_t)out_index(j) * loc.out_rs;
      };
      if (fast) {
#pragma unroll
        for (int j = 0; j < S; j++) {
          if (!fft_store_row(a, loc.unit, out_index(j))) continue;
          uint8_t *row = out_row(j);
          uint32_t w[8];
#pragma unroll
          for (int b = 0; b < 8; b++) w[b] = r[j][b];
          bit_transpose(w);
          *reinterpret_cast<uint4 *>(row + col) = make_uint4(w[0], w[1], w[2], w[3]);
          *reinterpret_cast<uint4 *>(row + col + 16) = make_uint4(w[4], w[5], w[6], w[7]);
        }
      } else if (live) {
#pragma unroll
        for (int j = 0; j < S; j++) {
          *reinterpret_cast<uint4 *>(mine + j * St::kSlot) = make_uint4(r[j][0], r[j][1], r[j][2], r[j][3]);
          *reinterpret_cast<uint4 *>(mine + j * St::kSlot + St::kHalf) =
              make_uint4(r[j][4], r[j][5], r[j][6], r[j][7]);
        }
#pragma unroll 1
        for (int j = 0; j < S; j++) {
          if (!fft_store_row(a, loc.unit, out_index(j))) continue;
          const uint4 lo = *reinterpret_cast<const uint4 *>(mine + j * St::kSlot);
          const uint4 hi = *reinterpret_cast<const uint4 *>(mine + j * St::kSlot + St::kHalf);
          uint32_t w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
          bit_transpose(w);
          store32_any(out_row(j) + col, remain, make_uint4(w[0], w[1], w[2], w[3]),
                      make_uint4(w[4], w[5], w[6], w[7]));
        }
      }
      if (!early && rd + 1 < rounds) prefetch(grp + stride);
      phase_sync<SYNC>();
      continue;
    }
    if (rd + 1 < rounds) prefetch(grp + stride);
    phase_sync<SYNC>();
    // Interpolate: inverse transform on V, levels 0 .. LG-1.
    levels_up<K, W, 0, 0, SYNC>(r, q, qm);
    // Evaluate on the coset beta + V = {K .. 2K-1}: forward transform, levels LG-1 .. 0.
    levels_down<K, W, LG - 1, kB.beta, SYNC>(r, q, qm);
    if (live) {
      const bool fast = whole(loc);
#pragma unroll
      for (int j = 0; j < S; j++) {
        if (!fft_store_row(a, loc.unit, out_index(j))) continue;
        uint8_t *row;
        if constexpr (PTRS)
          row = pt.out[out_index(j)];
        else
          row = loc.out0 + (uint64_t)out_index(j) * loc.out_rs;
        uint32_t w[8];
#pragma unroll
        for (int b = 0; b < 8; b++) w[b] = r[j][b];
        bit_transpose(w);
        const uint4 lo = make_uint4(w[0], w[1], w[2], w[3]), hi = make_uint4(w[4], w[5], w[6], w[7]);
        if (fast) {
          *reinterpret_cast<uint4 *>(row + col) = lo;
          *reinterpret_cast<uint4 *>(row + col + 16) = hi;
        } else {
          store32_any(row + col, remain, lo, hi);
        }
      }
    }
    phase_sync<SYNC>();
  }
}

// Per-K launch shape (index into kFftVariants), defaults from a sweep on B200 (16 GiB of
// 1 MiB shards per launch): K = 4, 8 and 16 prefer four 128-thread CTAs per SM; K = 32, 64
// and 128, whose slots need 255 registers, one 256-thread CTA per SM (10-12% above two
// 128-thread CTAs with the same registers and staging).
constexpr int kFftVariantDefault[8] = {0, 0, 1, 1, 1, 3, 3, 3};
inline int &fft_variant_for(int K) {
  static int v[8] = {0, 0, 1, 1, 1, 3, 3, 3};
  int l = 0;
  while ((1 << l) < K) l++;
  return v[l & 7];
}

// Automatic launch shape (the default; cleared by an explicit rs_set_fft_variant or
// rs_set_fft_lanes, restored by passing -1): on strided rows that are not 16-byte
// aligned, every 32-byte group takes the unaligned staging paths and more threads per
// group win. Measured on B200 (rows of 65537 bytes, 2^12..2^16 groups): wide lane
// groups with four 128-thread CTAs per SM were the best shape from 2^14 groups at
// every K >= 16 (up to 63% off the best at 2^12), where the aligned defaults lost
// 16-89%.
inline bool &fft_shape_auto(int K) {
  static bool a[8] = {true, true, true, true, true, true, true, true};
  int l = 0;
  while ((1 << l) < K) l++;
  return a[l & 7];
}
constexpr int fft_unaligned_variant(int K) { return K >= 16 ? 1 : 0; }

inline int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  }
  return n;
}

// Shapes with a compiled bitsliced encode kernel: the FFT kernel for (K, K) with K a
// power of two, the compile-time generator kernel (kernels_gen.cuh) for the reference's
// other generated shapes, (20,12) and common storage codes.
struct FftShape {
  int k, m;
  bool gen;  // generator kernel (no lane-group width or launch-shape choices)
};

inline const FftShape *find_fft_shape(size_t k, size_t m) {
  static const FftShape shapes[] = {{2, 2, false},   {4, 4, false},   {8, 8, false},  {16, 16, false},
                                    {32, 32, false}, {64, 64, false}, {128, 128, false},
                                    {7, 13, true},   {10, 10, true},  {14, 14, true}, {18, 6, true},
                                    {20, 12, true},  {4, 2, true},    {6, 3, true},   {8, 4, true},
                                    {10, 4, true},   {12, 4, true},   {16, 4, true},  {17, 3, true}};
  for (const FftShape &s : shapes)
    if ((size_t)s.k == k && (size_t)s.m == m) return &s;
  return nullptr;
}

// Lane-group widths tried per K (lanes per group = 2^W, slots per lane = K >> W).
constexpr int fft_w_lo(int K) { return K <= 8 ? 1 : K <= 32 ? 1 : K == 64 ? 2 : 3; }
constexpr int fft_w_hi(int K) { return K <= 8 ? 1 : K <= 32 ? 2 : K == 64 ? 3 : 4; }

// Selected lane-group width per K: 0 = fft_w_lo, 1 = fft_w_hi (rs_set_fft_lanes).
constexpr int kFftLanesDefault[8] = {0, 0, 0, 0, 0, 0, 0, 1};
inline int &fft_lanes_choice(int K) {
  static int c[8] = {0, 0, 0, 0, 0, 0, 0, 1};  // narrow groups measured fastest but for K = 128
  int l = 0;
  while ((1 << l) < K) l++;
  return c[l & 7];
}

// The tuner-table entry (tuning.hpp) of the library's automatic choice for a launch of
// this compiled shape: its generator kernel, or the (K,K) shape's current FFT launch
// shape, or on unaligned rows the wide-lane shape of its unaligned kernel; -1 when no
// entry matches.
inline int fft_auto_config(const FftShape &sh, bool aligned) {
  if (sh.gen) return kTuneConfigCount - 1;
  int wide = fft_lanes_choice(sh.k), variant = fft_variant_for(sh.k);
  if (!aligned && sh.k >= 16 && fft_shape_auto(sh.k)) {
    wide = 1;
    variant = fft_unaligned_variant(sh.k);
  }
  for (int c = 0; c < kTuneConfigCount; c++)
    if (kTuneConfigs[c].route == kTuneFft && kTuneConfigs[c].p0 == wide && kTuneConfigs[c].p1 == variant) return c;
  return -1;
}

template <int K, int W, bool PTRS, int V, bool UNAL = false>
inline cudaError_t launch_fft_kwv(const FftArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st) {
  constexpr FftVariant var = kFftVariants[V];
  uint64_t groups = a.items ? a.total_groups : (uint64_t)a.n_stripes * a.groups_per_stripe;
  uint64_t blocks = ((groups << W) + var.threads - 1) / var.threads;
  blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)sm_count() * var.ctas));
  const int smem = (K >> W) * FftStage<var.threads>::kSlot;
  auto kern = fft_kk_kernel<K, W, PTRS, var.threads, var.ctas, (bool)var.sync, UNAL>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<(unsigned)blocks, var.threads, smem, st>>>(a, pt);
  return cudaGetLastError();
}

template <int K, int W, bool PTRS>
inline cudaError_t launch_fft_kw(const FftArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st, int variant) {
  if constexpr (PTRS) {
    return launch_fft_kwv<K, W, PTRS, 0>(a, pt, st);  // single-stripe calls
  } else {
    if (variant == 1) return launch_fft_kwv<K, W, PTRS, 1>(a, pt, st);
    if (variant == 2) return launch_fft_kwv<K, W, PTRS, 2>(a, pt, st);
    if (variant == 3) return launch_fft_kwv<K, W, PTRS, 3>(a, pt, st);
    return launch_fft_kwv<K, W, PTRS, 0>(a, pt, st);
  }
}

template <int K, bool PTRS>
inline cudaError_t launch_fft_k(const FftArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st) {
  const bool forced = a.cfg_variant >= 0 || a.cfg_wide >= 0;
  const int wide = a.cfg_wide >= 0 ? a.cfg_wide : fft_lanes_choice(K);
  const int variant = a.cfg_variant >= 0 ? a.cfg_variant : fft_variant_for(K);
  if constexpr (!PTRS && K >= 16) {
    const bool unaligned =
        a.items ? a.items_unaligned != 0
                : ((reinterpret_cast<uintptr_t>(a.in_base) | reinterpret_cast<uintptr_t>(a.out_base) |
                    a.in_row_stride | a.in_stripe_stride | a.out_row_stride | a.out_stripe_stride) &
                   15u) != 0;
    if (unaligned && fft_shape_auto(K) && !forced)
      return launch_fft_kwv<K, fft_w_hi(K), PTRS, fft_unaligned_variant(K), true>(a, pt, st);
  }
  if constexpr (fft_w_lo(K) == fft_w_hi(K)) {
    return launch_fft_kw<K, fft_w_lo(K), PTRS>(a, pt, st, variant);
  } else {
    if (wide) return launch_fft_kw<K, fft_w_hi(K), PTRS>(a, pt, st, variant);
    return launch_fft_kw<K, fft_w_lo(K), PTRS>(a, pt, st, variant);
  }
}

// Per-K launchers, each compiled in its own translation unit (fft_k*.cu) so the large
// straight-line kernels build in parallel.
#define RSB_FFT_DECLARE(K)                                                                     \
  cudaError_t fft_launch_k##K(const FftArgs &a, const PtrTableT<false> &pt, cudaStream_t st); \
  cudaError_t fft_launch_k##K##p(const FftArgs &a, const PtrTableT<true> &pt, cudaStream_t st);
#define RSB_FFT_DEFINE(K)                                                                      \
  cudaError_t fft_launch_k##K(const FftArgs &a, const PtrTableT<false> &pt, cudaStream_t st) { \
    return launch_fft_k<K, false>(a, pt, st);                                                  \
  }                                                                                            \
  cudaError_t fft_launch_k##K##p(const FftArgs &a, const PtrTableT<true> &pt, cudaStream_t st) { \
    return launch_fft_k<K, true>(a, pt, st);                                                   \
  }
RSB_FFT_DECLARE(2)
RSB_FFT_DECLARE(4)
RSB_FFT_DECLARE(8)
RSB_FFT_DECLARE(16)
RSB_FFT_DECLARE(32)
RSB_FFT_DECLARE(64)
RSB_FFT_DECLARE(128)

template <int K, bool PTRS>
inline cudaError_t fft_launch_extern(const FftArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st) {
#define RSB_FFT_CALL(KK)                        \
  if constexpr (K == KK) {                      \
    if constexpr (PTRS)                         \
      return fft_launch_k##KK##p(a, pt, st);    \
    else                                        \
      return fft_launch_k##KK(a, pt, st);       \
  }
  RSB_FFT_CALL(2)
  RSB_FFT_CALL(4)
  RSB_FFT_CALL(8)
  RSB_FFT_CALL(16)
  RSB_FFT_CALL(32)
  RSB_FFT_CALL(64)
  RSB_FFT_CALL(128)
#undef RSB_FFT_CALL
  return cudaErrorInvalidValue;
}

// Generator-shape launchers (gen_k.cu).
template <bool PTRS>
cudaError_t gen8_launch(int k, int m, const FftArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st);

template <bool PTRS>
inline int launch_fft_any(const FftShape &sh, const FftArgs &a, const PtrTableT<PTRS> &pt,
                          cudaStream_t st) {
  if (a.items ? a.total_groups == 0 : (a.len == 0 || a.n_stripes == 0)) return RS_OK;
  cudaError_t e;
  if (sh.gen) {
    e = gen8_launch<PTRS>(sh.k, sh.m, a, pt, st);
    g_launches++;
    if (e != cudaSuccess) {
      set_cuda_error(e, "gen8_kernel launch");
      return RS_ERR_CUDA;
    }
    return RS_OK;
  }
  switch (sh.k) {
    case 2: e = fft_launch_extern<2, PTRS>(a, pt, st); break;
    case 4: e = fft_launch_extern<4, PTRS>(a, pt, st); break;
    case 8: e = fft_launch_extern<8, PTRS>(a, pt, st); break;
    case 16: e = fft_launch_extern<16, PTRS>(a, pt, st); break;
    case 32: e = fft_launch_extern<32, PTRS>(a, pt, st); break;
    case 64: e = fft_launch_extern<64, PTRS>(a, pt, st); break;
    case 128: e = fft_launch_extern<128, PTRS>(a, pt, st); break;
    default: return RS_ERR_INVALID_ARGUMENT;
  }
  g_launches++;
  if (e != cudaSuccess) {
    set_cuda_error(e, "fft_kk_kernel launch");
    return RS_ERR_CUDA;
  }
  return RS_OK;
}

inline int launch_fft8(const FftShape &sh, const uint8_t *in_base, uint64_t in_row, uint64_t in_stripe,
                       uint8_t *out_base, uint64_t out_row, uint64_t out_stripe, uint32_t n_stripes,
                       uint64_t len, cudaStream_t st) {
  FftArgs a{};
  a.in_base = in_base;
  a.in_row_stride = in_row;
  a.in_stripe_stride = in_stripe;
  a.out_base = out_base;
  a.out_row_stride = out_row;
  a.out_stripe_stride = out_stripe;
  a.len = len;
  a.n_stripes = n_stripes;
  a.groups_per_stripe = (uint32_t)((len + 31) / 32);
  PtrTableT<false> pt{};
  return launch_fft_any<false>(sh, a, pt, st);
}

// Ragged batch of (K, K) stripes described by a device item array.
inline int launch_fft8_items(const FftShape &sh, const FftItem *d_items, uint32_t n_items,
                             uint64_t total_groups, cudaStream_t st, const uint32_t *store_mask = nullptr,
                             bool items_unaligned = false, int cfg_wide = -1, int cfg_variant = -1) {
  FftArgs a{};
  a.items = d_items;
  a.n_items = n_items;
  a.total_groups = total_groups;
  a.store_mask = store_mask;
  a.items_unaligned = items_unaligned;
  a.cfg_wide = cfg_wide;
  a.cfg_variant = cfg_variant;
  PtrTableT<false> pt{};
  return launch_fft_any<false>(sh, a, pt, st);
}

// store_bits (4 words, parity rows 0..127): store only those parity rows; null: all.
inline int launch_fft8_ptrs(const FftShape &sh, uint8_t *const *shards, uint64_t len, cudaStream_t st,
                            const uint32_t *store_bits = nullptr) {
  FftArgs a{};
  if (store_bits) {
    a.use_store_bits = 1;
    for (int w = 0; w < 4; w++) a.store_bits[w] = store_bits[w];
  }
  a.len = len;
  a.n_stripes = 1;
  a.groups_per_stripe = (uint32_t)((len + 31) / 32);
  PtrTableT<true> pt;
  uintptr_t bits = 0;
  for (int i = 0; i < sh.k; i++) pt.in[i] = shards[i];
  for (int j = 0; j < sh.m; j++) pt.out[j] = shards[sh.k + j];
  for (int i = 0; i < sh.k + sh.m; i++) bits |= reinterpret_cast<uintptr_t>(shards[i]);
  a.ptrs_aligned = (bits & 15u) == 0;
  return launch_fft_any<true>(sh, a, pt, st);
}

}  // namespace rsb
