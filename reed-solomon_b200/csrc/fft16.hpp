// FFT-route encode of ReedSolomon16 for any k >= 2 (src/fft16.rs): a step program built
// once per shape on the host and run by the kernels of kernels_fft16.cuh.
//
// Program. With t the power of two >= k, interpolation through the k data points
// follows the reference's recursion (src/fft.rs:198-239, the tower builder of
// src/fft16.rs:223-): an inverse transform where a whole half of the points is known;
// otherwise the known first half is interpolated, evaluated on the second half's points
// and subtracted, the rest interpolated recursively, and the halves combined with the
// constant WHAT[level][beta]. Evaluation then runs one forward transform of the t
// coefficients per coset {c*t .. c*t+t-1} holding parity points (c = 0 included when
// k < t). The registers live in three bitsliced buffers per stripe: C (t registers: the
// data, then the coefficients), S (t/2: interpolation scratch) and W (t: evaluation).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace rsb {

// Scratch budget per run: a wave of registers this size stays resident in L2 across
// the passes (the B200's L2 is 126 MB).
constexpr size_t kFft16ScratchBudget = (size_t)48 << 20;

struct Fft16Step {
  enum Kind : uint8_t { kTransform, kMulXor } kind;
  uint8_t src_buf, dst_buf;  // 0 = C, 1 = S, 2 = W
  bool inverse;              // transform direction
  uint32_t src_start, dst_start;
  uint32_t size;             // transform: registers (a power of two); mulxor: count
  uint64_t cols;             // first constant of the transform, or the mulxor constant;
                             // kNoConst: plain XOR
};

struct Fft16Eval {
  uint32_t beta;        // coset of the forward transform W = FFT(C)
  uint64_t cols;        // its first constant
  uint32_t r_lo, r_hi;  // W registers stored, as parity rows parity_row ...
  uint64_t parity_row;
};

struct Fft16Program {
  static constexpr uint64_t kNoConst = ~0ull;
  uint32_t k = 0, m = 0, t = 0;
  std::vector<Fft16Step> interp;
  std::vector<Fft16Eval> evals;
  std::vector<uint16_t> cols;  // 16 u16 per constant: its Karatsuba factors' column bytes
  uint64_t butterflies = 0;    // per 32-symbol group (route estimate)
  bool uses_s = false;         // the interpolation needs S (k not a power of two)
  bool eval_in_place = false;  // a single evaluation runs on C itself (no W)
  uint32_t regs_s() const { return uses_s ? t / 2 : 0; }
  uint32_t regs_w() const { return eval_in_place ? 0 : t; }
  uint32_t regs() const { return t + regs_s() + regs_w(); }  // per stripe and group
};

// Erasure decoding on the FFT route for one presence pattern (one stripe per run).
// With N the power of two >= n shards, the code is f (degree < k) evaluated at points
// 0..n-1. Only the k survivors are read; every other point of {0..N-1} is treated as
// erased (E). With the error locator L(x) = prod_{e in E} (x - e), g = f * L has
// degree < N and is known everywhere: f(i) L(i) at survivors, 0 on E. An inverse
// transform gives g's novel-basis coefficients, the formal derivative there is
// D(X_i) = sum_{t in bits(i)} kappa_t X_{i - 2^t} (each normalised subspace polynomial
// is linearized, so its derivative is a constant kappa_t), a forward transform gives g'
// everywhere, and at an erased point f(e) = g'(e) / L'(e). L at the survivors and L' on
// E are one XOR-convolution of E's indicator with the discrete log table.
struct Fft16Decode {
  uint32_t n = 0, N = 0, lg = 0;
  std::vector<uint32_t> targets;  // points to rebuild, in output order
  std::vector<uint16_t> cols;     // transform (N-1) | row scale (N) | kappa (lg) | targets
  uint64_t row_off = 0, kappa_off = 0, target_off = 0;
  uint64_t butterflies = 0;       // per 32-symbol group (route estimate)
  uint32_t regs() const { return 2 * N; }  // C + W per group
};

// survivors: the k points read; targets: the points to rebuild (k + m <= 65536).
bool fft16_decode_build(size_t k, size_t m, const std::vector<uint32_t> &survivors,
                        const std::vector<uint32_t> &targets, Fft16Decode &d);
// Whether the decode's estimated work is below the matrix route's (rows x k
// coefficients plus building those rows).
bool fft16_decode_preferred(const Fft16Decode &d, size_t k);
size_t fft16_decode_scratch_bytes(const Fft16Decode &d, size_t len, size_t budget);
// d_ptrs: device table of the n shard pointers (survivors read, targets written);
// d_targets: the target points on the device, of which the first n_targets are stored.
int fft16_decode_run(const Fft16Decode &d, const uint16_t *d_cols, uint8_t *scratch, size_t scratch_bytes,
                     uint8_t *const *d_ptrs, const uint32_t *d_targets, size_t n_targets, size_t len,
                     cudaStream_t st);

// False (no FFT route) for k < 2.
bool fft16_build(size_t k, size_t m, Fft16Program &p);
// Whether the FFT route's estimated work is below the tower matrix kernel's.
bool fft16_preferred(const Fft16Program &p);
// Whether the FFT route is expected to finish first for n_stripes stripes of len-byte
// shards: about 5.2 us per launch plus 0.065 ns per butterfly and 32-symbol group,
// against the matrix kernel's max(1.07 us per data shard, 0.46 ns per coefficient and
// shard byte). Small calls are latency-bound (the FFT's chain of pass launches; the
// matrix kernel's walk over the k data rows), large ones throughput-bound. Constants
// fitted to B200 timings of both routes on 23 calls from (16,16) x 16 stripes of 2 KiB
// to (4096,12288) and (2000,50) x 64 KiB; the fitted choice is within 3% of the faster
// route on each of them.
bool fft16_faster(const Fft16Program &p, size_t len, size_t n_stripes);
// The same against the GF(2^8) matrix kernel, which a shape with k + m <= 256 can use
// instead (every coefficient in the subfield): about 0.2 ns per coefficient and shard
// byte on B200 (RS(32,32) at 343 GB/s, (100,156) x 64 x 16 KiB at 81 GB/s), the
// per-shard latency term scaled by the same 0.57 as the (100,156) throughput against
// the tower kernel. Measured there: tower FFT 123 GB/s, the GF(2^8) matrix kernel 81.
bool fft16_faster_than_gf8_matrix(const Fft16Program &p, size_t len, size_t n_stripes);
// Scratch for one run: all stripes at once when that fits `budget`, else the largest
// slice of one stripe's 32-symbol groups that does (at least one group).
size_t fft16_scratch_bytes(const Fft16Program &p, size_t n_stripes, size_t len, size_t budget);
// Encodes n_stripes stripes: data row r of stripe s at in_base + s*in_stripe + r*in_row,
// parity row j at out_base + s*out_stripe + j*out_row; with d_ptrs (one stripe) the rows
// are its k + m device pointers. All work is enqueued on `st`, using `scratch`.
int fft16_run(const Fft16Program &p, const uint16_t *d_cols, uint8_t *scratch, size_t scratch_bytes,
              const uint8_t *in_base, uint64_t in_row, uint64_t in_stripe, uint8_t *out_base, uint64_t out_row,
              uint64_t out_stripe, uint8_t *const *d_ptrs, size_t n_stripes, size_t len, cudaStream_t st);

}  // namespace rsb
