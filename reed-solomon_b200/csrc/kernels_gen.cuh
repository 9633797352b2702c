// Compile-time generator route: GF(2^8) encode for the reference's other generated
// shapes ((7,13), (10,10), (14,14), (18,6), src/fft_programs.rs:10-17), (20,12) and
// common storage codes ((4,2), (6,3), (8,4), (10,4), (12,4), (16,4), (17,3)), bitsliced
// like the FFT kernels of kernels_fft.cuh.
//
// The reference encodes these shapes with straight-line programs that its FFT builder
// generated (src/fft.rs:156-592). Their outputs are the systematic generator's parity
// rows (src/fft.rs:1010-1041), so on the device the generator itself is compiled in:
// a thread transposes its 32 byte columns of each of the k data shards into 8 bit
// planes, and plane b of parity j is then a fixed XOR network over the k x 8 data
// planes (bit b of G[j][i] * 2^p selects plane p of shard i). With the constants known
// at compile time that costs about 16 three-input XORs per coefficient on 32 columns,
// a quarter of the matrix kernel's SWAR form (8 LOP3 per coefficient per 4 columns);
// at k + m <= 32 an FFT program's butterflies would save little over that.
#pragma once

#include "kernels_fft.cuh"

namespace rsb {

namespace genc {

constexpr uint8_t ginv(uint8_t a) {  // a^254
  uint8_t r = 1, b = a;
  for (int e = 254; e; e >>= 1) {
    if (e & 1) r = fftc::gmul(r, b);
    b = fftc::gmul(b, b);
  }
  return r;
}

struct GenRows {
  uint8_t g[32][32];
};

// Parity rows of the systematic generator: row j is the Lagrange basis on the data
// points 0..k-1 evaluated at point k + j. The reference builds the same rows as
// vandermonde(n, k) * inverse(top k x k) (src/reedsolomon.rs:155-159,
// src/matrix.rs:183-196); the host's parity_rows (gf_host.hpp) uses this closed form too.
constexpr GenRows make_gen(int k, int m) {
  GenRows r{};
  uint8_t w[32] = {};  // barycentric weights 1 / prod_{v != u} (u - v)
  for (int u = 0; u < k; u++) {
    uint8_t prod = 1;
    for (int v = 0; v < k; v++)
      if (v != u) prod = fftc::gmul(prod, (uint8_t)(u ^ v));
    w[u] = ginv(prod);
  }
  for (int j = 0; j < m; j++) {
    const int x = k + j;
    uint8_t ell = 1;  // prod_v (x - v)
    for (int v = 0; v < k; v++) ell = fftc::gmul(ell, (uint8_t)(x ^ v));
    for (int u = 0; u < k; u++) r.g[j][u] = fftc::gmul(fftc::gmul(w[u], ell), ginv((uint8_t)(x ^ u)));
  }
  return r;
}

template <int K, int M>
inline constexpr GenRows kGen = make_gen(K, M);

}  // namespace genc

// One thread per 32-column group, persistent over the flattened (stripe, group) space
// like fft_kk_kernel, with the same cp.async staging of the next round's data bytes.
template <int KD, int MP, bool PTRS, int THREADS, int CTAS>
__global__ void __launch_bounds__(THREADS, CTAS)
    gen8_kernel(const FftArgs a, const __grid_constant__ PtrTableT<PTRS> pt) {
  static_assert(KD + MP <= 32, "generator shapes have at most 32 shards");
  extern __shared__ __align__(16) uint8_t stage[];
  using namespace fftc;
  using St = FftStage<THREADS>;
  const uint32_t tid = threadIdx.x;
  const uint64_t total = a.items ? a.total_groups : (uint64_t)a.n_stripes * a.groups_per_stripe;
  const uint64_t stride = (uint64_t)gridDim.x * THREADS;
  const uint64_t rounds = (total + stride - 1) / stride;
  const uint64_t grp0 = (uint64_t)blockIdx.x * THREADS + tid;
  uint8_t *mine = stage + tid * 16;

  auto in_ptr = [&](const FftLoc &l, int i) -> const uint8_t * {
    if constexpr (PTRS)
      return pt.in[i];
    else
      return l.in0 + (uint64_t)i * l.in_rs;
  };
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
      for (int i = 0; i < KD; i++) {
        const uint8_t *p = in_ptr(l, i) + l.col;
        cp_async16(mine + i * St::kSlot, p);
        cp_async16(mine + i * St::kSlot + St::kHalf, p + 16);
      }
    } else {
#pragma unroll 1
      for (int i = 0; i < KD; i++) stage32<St::kHalf>(mine + i * St::kSlot, in_ptr(l, i) + l.col, l.remain, l.col);
    }
    cp_async_commit();
  };

  prefetch(grp0);
  for (uint64_t rd = 0; rd < rounds; rd++) {
    const uint64_t grp = grp0 + rd * stride;
    const FftLoc loc = fft_locate(a, grp);
    cp_async_wait_all();
#pragma unroll 1
    for (int i = 0; i < KD; i++) {
      uint4 *p0 = reinterpret_cast<uint4 *>(mine + i * St::kSlot);
      uint4 *p1 = reinterpret_cast<uint4 *>(mine + i * St::kSlot + St::kHalf);
      uint4 lo = *p0, hi = *p1;
      uint32_t w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
      bit_transpose(w);
      *p0 = make_uint4(w[0], w[1], w[2], w[3]);
      *p1 = make_uint4(w[4], w[5], w[6], w[7]);
    }
    Reg r[KD];
#pragma unroll
    for (int i = 0; i < KD; i++) {
      uint4 lo = *reinterpret_cast<const uint4 *>(mine + i * St::kSlot);
      uint4 hi = *reinterpret_cast<const uint4 *>(mine + i * St::kSlot + St::kHalf);
      r[i][0] = lo.x, r[i][1] = lo.y, r[i][2] = lo.z, r[i][3] = lo.w;
      r[i][4] = hi.x, r[i][5] = hi.y, r[i][6] = hi.z, r[i][7] = hi.w;
    }
    if (rd + 1 < rounds) prefetch(grp + stride);
    if (loc.remain == 0) continue;
    const bool fast = whole(loc);
    static_for<0, MP>([&](auto jj) {
      constexpr int j = decltype(jj)::value;
      if (!fft_store_row(a, loc.unit, j)) return;
      Reg acc;
#pragma unroll
      for (int b = 0; b < 8; b++) acc[b] = 0;
      static_for<0, KD>([&](auto ii) {
        constexpr int i = decltype(ii)::value;
        mul_acc<genc::kGen<KD, MP>.g[j][i]>(acc, r[i]);
      });
      uint8_t *row;
      if constexpr (PTRS)
        row = pt.out[j];
      else
        row = loc.out0 + (uint64_t)j * loc.out_rs;
      uint32_t w[8];
#pragma unroll
      for (int b = 0; b < 8; b++) w[b] = acc[b];
      bit_transpose(w);
      const uint4 lo = make_uint4(w[0], w[1], w[2], w[3]), hi = make_uint4(w[4], w[5], w[6], w[7]);
      if (fast) {
        *reinterpret_cast<uint4 *>(row + loc.col) = lo;
        *reinterpret_cast<uint4 *>(row + loc.col + 16) = hi;
      } else {
        store32_any(row + loc.col, loc.remain, lo, hi);
      }
    });
  }
}

template <bool PTRS>
cudaError_t gen8_launch_more(int k, int m, const FftArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st);

template <int KD, int MP, bool PTRS, int THREADS, int CTAS>
inline cudaError_t launch_gen8_shape(const FftArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st) {
  const uint64_t groups = a.items ? a.total_groups : (uint64_t)a.n_stripes * a.groups_per_stripe;
  uint64_t blocks = (groups + THREADS - 1) / THREADS;
  blocks = std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)sm_count() * CTAS));
  const int smem = KD * FftStage<THREADS>::kSlot;
  auto kern = gen8_kernel<KD, MP, PTRS, THREADS, CTAS>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<(unsigned)blocks, THREADS, smem, st>>>(a, pt);
  return cudaGetLastError();
}

}  // namespace rsb
