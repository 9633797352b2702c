// C ABI of the rs_b200 library (include/rs_b200.h): codec and decoder handles,
// reference-order argument checks, plan caches, host- and device-pointer calls.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "runtime.hpp"
#include "gf_host.hpp"
#include "kernels_matrix.cuh"
#include "kernels_fft.cuh"
#include "kernels_bits.cuh"
#include "kernels_plan.cuh"
#include "codec8.hpp"

namespace rsb {

std::atomic<uint64_t> g_launches{0};
static thread_local char g_last_error[256];

void set_cuda_error(cudaError_t e, const char *what) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what, cudaGetErrorString(e));
  cudaGetLastError();
}

int ensure_device(int *device_out) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return RS_ERR_NO_DEVICE;
  }
  int dev = 0;
  RSB_CU(cudaGetDevice(&dev));
  if (device_out) *device_out = dev;
  return RS_OK;
}

cudaError_t scratch_alloc(void **p, size_t bytes, cudaStream_t st) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, st);
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev]) {
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      e = cudaMemPoolCreate(&pools[dev], &props);
      if (e != cudaSuccess) {
        pools[dev] = nullptr;
        return e;
      }
      uint64_t keep = 1ull << 30;
      cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  return cudaMallocFromPoolAsync(p, bytes, pools[dev], st);
}

Gf16Tables::Gf16Tables() : log(65536, 0), exp(2 * 65535, 0) {
  // Smallest element of full order 65535 = 3 * 5 * 17 * 257.
  auto power = [](uint16_t b, uint32_t e) {
    uint16_t r = 1;
    while (e) {
      if (e & 1) r = gf16_mul(r, b);
      b = gf16_mul(b, b);
      e >>= 1;
    }
    return r;
  };
  uint16_t g = 2;
  for (;; g++) {
    if (power(g, 65535 / 3) != 1 && power(g, 65535 / 5) != 1 && power(g, 65535 / 17) != 1 &&
        power(g, 65535 / 257) != 1)
      break;
  }
  uint16_t x = 1;
  for (uint32_t i = 0; i < 65535; i++) {
    exp[i] = x;
    exp[i + 65535] = x;
    log[x] = (uint16_t)i;
    x = gf16_mul(x, g);
  }
}

const Gf16Tables &gf16() {
  static const Gf16Tables t;
  return t;
}

// ------------------------------------------------------------------------------
// Kernel launch helpers
// ------------------------------------------------------------------------------

static size_t g8_smem(uint32_t rows, uint32_t k) { return 8192 + (size_t)rows * k; }

template <int V, bool PTRS, bool VERIFY>
static int launch_gf8_t(const ApplyArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st) {
  constexpr MatrixVariant mv = kMatrixVariants[V];
  auto kern = gf8_matrix_kernel<mv.out_tile, mv.row_chunk, PTRS, VERIFY>;
  size_t smem = g8_smem(a.rows, a.k);
  if (smem > 48 * 1024) RSB_CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  uint64_t tiles = (a.len + kTileBytes - 1) / kTileBytes;
  dim3 grid((unsigned)tiles, std::min<uint32_t>(a.n_stripes, 65535), (a.rows + mv.row_chunk - 1) / mv.row_chunk);
  kern<<<grid, kThreads, smem, st>>>(a, pt);
  g_launches++;
  RSB_CU(cudaGetLastError());
  return RS_OK;
}

int launch_gf8(const ApplyArgs &a, const PtrTable *pt, bool verify, cudaStream_t st) {
  if (a.len == 0 || a.rows == 0 || a.n_stripes == 0) return RS_OK;
  if (pt) {
    PtrTableT<true> t;
    memcpy(t.in, pt->in, sizeof(t.in));
    memcpy(t.out, pt->out, sizeof(t.out));
    return verify ? launch_gf8_t<0, true, true>(a, t, st) : launch_gf8_t<0, true, false>(a, t, st);
  }
  PtrTableT<false> t{};
  if (verify) return launch_gf8_t<0, false, true>(a, t, st);
  if (matrix_bits()) {
    g_launches++;
    cudaError_t e = launch_gf8_bits(a, st);
    if (e != cudaSuccess) {
      set_cuda_error(e, "gf8_bits_kernel launch");
      return RS_ERR_CUDA;
    }
    return RS_OK;
  }
  switch (matrix_variant()) {
    case 1: return launch_gf8_t<1, false, false>(a, t, st);
    case 2: return launch_gf8_t<2, false, false>(a, t, st);
    case 3: return launch_gf8_t<3, false, false>(a, t, st);
    default: return launch_gf8_t<0, false, false>(a, t, st);
  }
}

// ------------------------------------------------------------------------------
// GF(2^8) codec
// ------------------------------------------------------------------------------

// Row pitch of device staging for host-pointer calls: whole 16-byte units, so every
// staged shard starts aligned and the kernels' vector paths apply whatever the shard
// length (a packed odd length would put most rows on the byte paths).
static size_t pitch16(size_t len) { return (len + 15) & ~size_t(15); }


// Encode route for a shape and length: the compiled kernel where the shape has one and
// the shard holds at least two 32-column groups, else the matrix kernel. Row alignment
// does not change the route: with the aligned-window staging of unaligned rows the
// generator kernels measured 1.1-2.5x the matrix kernel there too ((10,10), (20,12) at
// 1..256 stripes; (10,4) at 4 KiB 0.73-1.4x), and the FFT kernels stay further ahead.
bool use_fft8(const rs8_codec *c, size_t len) {
  int r = c->route.load();
  if (r == 1 || !c->gen->fft) return false;
  if (r == 2) return true;
  return len >= 64;
}

// The compiled kernel rereads all k data rows and does an encode's work, about (k+m)
// bytes per column at its rate (~3.5 TB/s; ~2.1 at K = 64, ~1.4 at K = 128), to save
// missing_parity * k matrix coefficients per column (2 LOP3 per byte each, ~11 Tops/s):
// it pays from missing_parity * k ~ 1.6 (k+m) at 3.5 TB/s. Measured on B200: RS(32,32)
// with 8 missing parity rows +17% at 1 MiB shards, (64,64) with 16 +51%, (10,4) with 1
// -15%. With the subset-table matrix kernel (twice the coefficient rate of the kernels
// these figures came from) the bar rose; the factors below come from a sweep of 0.5-3x
// the earlier ones on batches of 1..m erasures at 4 KiB, 64 KiB and 1 MiB (B200):
// (128,128) best at 3x (up to 11% at 1 MiB), (64,64) at 2x, (32,32) at 1.5x, (16,16)
// at 1x, the generator shapes from 1.5x of a factor of 4 ((20,12) at 4 KiB 22%); all
// within a few percent of the best of the sweep, and regeneration still beats none
// (up to 25%).
bool regen_parity_pays(const Gen8 &g, size_t missing_parity, int route) {
  if (!g.fft || missing_parity == 0 || route == 1) return false;
  if (route == 2) return true;
  const size_t factor = g.fft->gen ? 6 : g.k >= 128 ? 12 : g.k >= 64 ? 6 : g.k >= 32 ? 3 : 2;
  return missing_parity * g.k >= factor * (g.k + g.m);
}

int encode8_strided(rs8_codec *c, const uint8_t *in_base, uint64_t in_row, uint64_t in_stripe,
                           uint8_t *out_base, uint64_t out_row, uint64_t out_stripe, size_t n_stripes,
                           size_t len, cudaStream_t st) {
  const Gen8 &g = *c->gen;
  if (use_fft8(c, len))
    return launch_fft8(*g.fft, in_base, in_row, in_stripe, out_base, out_row, out_stripe,
                       (uint32_t)n_stripes, len, st);
  ApplyArgs a{};
  a.in_base = in_base;
  a.in_row_stride = in_row;
  a.in_stripe_stride = in_stripe;
  a.out_base = out_base;
  a.out_row_stride = out_row;
  a.out_stripe_stride = out_stripe;
  a.coeffs = g.d_rows;
  a.k = (uint32_t)g.k;
  a.rows = (uint32_t)g.m;
  a.len = len;
  a.n_stripes = (uint32_t)n_stripes;
  return launch_gf8(a, nullptr, false, st);
}

// Builds (or fetches) the plan of one presence pattern with the device Gauss-Jordan.
static int plan8_for(const Gen8 &g, PlanCache &cache, Exec &ex, const Presence &pres,
                     std::shared_ptr<const Plan> &out) {
  out = cache.find(pres);
  if (out) return RS_OK;
  auto plan = std::make_shared<Plan>();
  plan->presence = pres;
  plan->device = g.device;
  split_pattern(pres, g.k, g.k + g.m, plan->survivors, plan->missing_data, plan->missing_parity);
  if (plan->survivors.size() < g.k) return RS_TOO_FEW_SHARDS_PRESENT;
  size_t rows = plan->missing_data.size() + plan->missing_parity.size();
  std::vector<uint16_t> host(g.k + std::max<size_t>(rows, 1) + 1);
  for (size_t t = 0; t < g.k; t++) host[t] = (uint16_t)plan->survivors[t];
  size_t off = g.k;
  for (uint32_t x : plan->missing_data) host[off++] = (uint16_t)x;
  for (uint32_t x : plan->missing_parity) host[off++] = (uint16_t)x;
  host[g.k + std::max<size_t>(rows, 1)] = (uint16_t)rows;
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  size_t idx_bytes = host.size() * 2;
  size_t out_bytes = std::max<size_t>(rows, 1) * g.k;
  RSB_TRY(ex.aux.ensure(idx_bytes + 16 + sizeof(int)));
  void *d_rows = nullptr;
  RSB_CU(cudaMalloc(&d_rows, out_bytes));
  plan->d_rows = d_rows;
  uint16_t *d_idx = reinterpret_cast<uint16_t *>(ex.aux.ptr);
  int *d_status = reinterpret_cast<int *>(ex.aux.ptr + ((idx_bytes + 15) & ~size_t(15)));
  RSB_CU(cudaMemcpyAsync(d_idx, host.data(), idx_bytes, cudaMemcpyHostToDevice, ex.stream));
  PlanArgs pa{};
  pa.gen = g.d_rows;
  pa.k = (uint32_t)g.k;
  pa.m = (uint32_t)g.m;
  pa.survivors = d_idx;
  pa.targets = d_idx + g.k;
  pa.n_targets = d_idx + g.k + std::max<size_t>(rows, 1);
  pa.max_rows = (uint32_t)std::max<size_t>(rows, 1);
  pa.out = reinterpret_cast<uint8_t *>(d_rows);
  pa.status = d_status;
  size_t smem = plan_smem((uint32_t)g.k).total;
  if (smem > 48 * 1024)
    RSB_CU(cudaFuncSetAttribute(gf8_plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gf8_plan_kernel<<<1, 256, smem, ex.stream>>>(pa);
  g_launches++;
  RSB_CU(cudaGetLastError());
  int status = 0;
  RSB_CU(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, ex.stream));
  RSB_CU(cudaStreamSynchronize(ex.stream));
  if (status) return RS_SINGULAR_MATRIX;
  out = cache.insert(pres, plan);
  return RS_OK;
}

// Shared body of every GF(2^8) reconstruct (src/reedsolomon.rs:615-641, :829-891).
// With `dev` the shard pointers are device pointers and work is enqueued on `st`;
// `route` is the codec's (0 automatic, 1 matrix, 2 compiled kernel).
static int reconstruct8(const Gen8 &g, PlanCache *cache, const Plan *fixed, Exec &ex,
                        uint8_t *const *shards, const size_t *lens, const uint8_t *present,
                        size_t n_shards, bool data_only, bool dev, cudaStream_t st, int route = 0) {
  size_t n = g.k + g.m;
  if (!shards || !lens || !present) return RS_ERR_INVALID_ARGUMENT;
  if (n_shards != n) return n_shards < n ? RS_TOO_FEW_SHARDS : RS_TOO_MANY_SHARDS;
  Presence pres;
  size_t n_present = 0, len = 0;
  RSB_TRY(scan_shards(lens, present, n, false, pres, n_present, len));
  if (fixed && pres != fixed->presence) return RS_INVALID_SHARD_FLAGS;
  if (n_present == n) return RS_OK;
  if (!fixed && n_present < g.k) return RS_TOO_FEW_SHARDS_PRESENT;
  if (len == 0) return RS_TOO_FEW_SHARDS_PRESENT;
  std::shared_ptr<const Plan> hold;
  const Plan *plan = fixed;
  if (!plan) {
    RSB_TRY(plan8_for(g, *cache, ex, pres, hold));
    plan = hold.get();
  }
  RSB_TRY(check_absent_buffers(lens, present, n, g.k, len, data_only));
  size_t rows = plan->missing_data.size() + (data_only ? 0 : plan->missing_parity.size());
  if (rows == 0) return RS_OK;
  PtrTable pt;
  std::vector<uint32_t> outs(plan->missing_data);
  if (!data_only) outs.insert(outs.end(), plan->missing_parity.begin(), plan->missing_parity.end());
  ApplyArgs a{};
  a.coeffs = reinterpret_cast<const uint8_t *>(plan->d_rows);
  a.k = (uint32_t)g.k;
  a.rows = (uint32_t)rows;
  a.len = len;
  a.n_stripes = 1;
  if (dev) {
    RSB_CU(cudaSetDevice(g.device));
    // Shards of at least 64 KiB on a shape with a compiled kernel: the matrix route
    // rebuilds the missing data rows (its plan's leading rows), then the compiled
    // kernel regenerates the missing parity from the whole data rows, storing only
    // those rows. Smaller calls are latency-bound and keep the single launch.
    const bool split = !data_only && len >= 64 && (route == 2 || len >= ((size_t)64 << 10)) &&
                       regen_parity_pays(g, plan->missing_parity.size(), route);
    const size_t mrows = split ? plan->missing_data.size() : rows;
    if (mrows) {
      a.rows = (uint32_t)mrows;
      for (size_t t = 0; t < g.k; t++) pt.in[t] = shards[plan->survivors[t]];
      for (size_t j = 0; j < mrows; j++) pt.out[j] = shards[outs[j]];
      RSB_TRY(launch_gf8(a, &pt, false, st));
    }
    if (!split) return RS_OK;
    uint32_t bits[4] = {0, 0, 0, 0};
    for (uint32_t x : plan->missing_parity) bits[(x - g.k) / 32] |= 1u << ((x - g.k) % 32);
    return launch_fft8_ptrs(*g.fft, shards, len, st, bits);
  }
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  const size_t pitch = pitch16(len);
  RSB_TRY(ex.buf.ensure((g.k + rows) * pitch));
  a.in_base = ex.buf.ptr;
  a.in_row_stride = pitch;
  a.out_base = ex.buf.ptr + g.k * pitch;
  a.out_row_stride = pitch;
  if (host_staged((g.k + rows) * pitch)) {
    // As rs8_encode: survivors gathered into pinned memory by host threads, one copy each
    // way, the rebuilt rows scattered back.
    RSB_TRY(ex.io.ensure((g.k + rows) * pitch));
    uint8_t *h = ex.io.ptr;
    gather_rows(h, pitch, g.k, len, [&](size_t t) { return shards[plan->survivors[t]]; });
    RSB_CU(cudaMemcpyAsync(ex.buf.ptr, h, g.k * pitch, cudaMemcpyHostToDevice, ex.stream));
    RSB_TRY(launch_gf8(a, nullptr, false, ex.stream));
    RSB_CU(cudaMemcpyAsync(h + g.k * pitch, ex.buf.ptr + g.k * pitch, rows * pitch, cudaMemcpyDeviceToHost,
                           ex.stream));
    RSB_CU(cudaStreamSynchronize(ex.stream));
    scatter_rows(h + g.k * pitch, pitch, rows, len, [&](size_t j) { return shards[outs[j]]; });
    return RS_OK;
  }
  for (size_t t = 0; t < g.k; t++)
    RSB_CU(cudaMemcpyAsync(ex.buf.ptr + t * pitch, shards[plan->survivors[t]], len,
                           cudaMemcpyHostToDevice, ex.stream));
  RSB_TRY(launch_gf8(a, nullptr, false, ex.stream));
  for (size_t j = 0; j < rows; j++)
    RSB_CU(cudaMemcpyAsync(shards[outs[j]], ex.buf.ptr + (g.k + j) * pitch, len,
                           cudaMemcpyDeviceToHost, ex.stream));
  RSB_CU(cudaStreamSynchronize(ex.stream));
  return RS_OK;
}

static int check_equal_lengths(const size_t n, size_t len) {
  (void)n;
  if (len == 0) return RS_EMPTY_SHARD;
  return RS_OK;
}

}  // namespace rsb

// ==============================================================================
// Exported entry points
// ==============================================================================

using namespace rsb;

extern "C" {

const char *rs_strerror(int status) {
  switch (status) {
    case RS_OK: return "Ok";
    case RS_TOO_FEW_SHARDS: return "The number of provided shards is smaller than the one in codec";
    case RS_TOO_MANY_SHARDS: return "The number of provided shards is greater than the one in codec";
    case RS_TOO_FEW_DATA_SHARDS: return "The number of provided data shards is smaller than the one in codec";
    case RS_TOO_MANY_DATA_SHARDS: return "The number of provided data shards is greater than the one in codec";
    case RS_TOO_FEW_PARITY_SHARDS: return "The number of provided parity shards is smaller than the one in codec";
    case RS_TOO_MANY_PARITY_SHARDS: return "The number of provided parity shards is greater than the one in codec";
    case RS_TOO_FEW_BUFFER_SHARDS: return "The number of provided buffer shards is smaller than the number of parity shards in codec";
    case RS_TOO_MANY_BUFFER_SHARDS: return "The number of provided buffer shards is greater than the number of parity shards in codec";
    case RS_INCORRECT_SHARD_SIZE: return "At least one of the provided shards is not of the correct size";
    case RS_TOO_FEW_SHARDS_PRESENT: return "The number of shards present is smaller than number of parity shards, cannot reconstruct missing shards";
    case RS_EMPTY_SHARD: return "The first shard provided is of zero length";
    case RS_INVALID_SHARD_FLAGS: return "The number of flags does not match the total number of shards";
    case RS_INVALID_INDEX: return "The data shard index provided is greater or equal to the number of data shards in codec";
    case RS_SINGULAR_MATRIX: return "The decode matrix for this shard pattern is singular and cannot be inverted";
    case RS_ERR_CUDA: return g_last_error[0] ? g_last_error : "CUDA runtime error";
    case RS_ERR_ALLOC: return "Device or host allocation failed";
    case RS_ERR_INVALID_ARGUMENT: return "Invalid argument";
    case RS_ERR_NO_DEVICE: return "No usable CUDA device";
    case RS_ERR_TIMEOUT: return "A bounded device wait timed out";
    case RS_ERR_LENGTH_MISMATCH: return "Input and output lengths differ";
    case RS_ERR_TOO_LARGE: return "The request needs more than the fixed working area holds";
    default: return "Unknown status";
  }
}

uint32_t rs_abi_version(void) { return (1u << 16) | 0u; }

int rs_device_check(void) { return ensure_device(nullptr); }

uint64_t rs_kernel_launch_count(void) { return g_launches.load(); }

static int log2_index(size_t k) {
  int l = 0;
  while (((size_t)1 << l) < k) l++;
  return l & 7;
}

int rs_set_fft_variant(size_t k, int variant) {
  const FftShape *sh = find_fft_shape(k, k);
  if (!sh || sh->gen || variant < -1 || variant >= kFftVariantCount) return -1;
  int &v = fft_variant_for((int)k);
  int old = v;
  v = variant < 0 ? kFftVariantDefault[log2_index(k)] : variant;
  fft_shape_auto((int)k) = variant < 0;
  return old;
}

int rs_fft_variant_count(void) { return kFftVariantCount; }

int rs_set_matrix_variant(int variant) {
  if (variant < 0 || variant >= kMatrixVariantCount) return -1;
  int old = matrix_variant();
  matrix_variant() = variant;
  return old;
}

int rs_matrix_variant_count(void) { return kMatrixVariantCount; }

int rs_set_matrix_bits(int on) {
  if (on < 0 || on > 4) return -1;
  const int old = matrix_bits();
  matrix_bits() = on;
  return old;
}

int rs_set_fft_lanes(size_t k, int wide) {
  const FftShape *sh = find_fft_shape(k, k);
  if (!sh || sh->gen || wide < -1 || wide > 1) return -1;
  int &c = fft_lanes_choice((int)k);
  int old = c;
  c = wide < 0 ? kFftLanesDefault[log2_index(k)] : wide;
  fft_shape_auto((int)k) = wide < 0;
  return old;
}

int rs_set_host_staging(int on) {
  return host_staging_on().exchange(on ? 1 : 0);
}

int rs_set_host_copy_threads(int n) {
  const int old = host_copy_threads().load();
  if (n >= 1 && n <= 64) host_copy_threads().store(n);
  return old;
}

int rs_generator_rows(int field, size_t k, size_t m, uint16_t *out, size_t out_len) {
  if (!out || (field != 8 && field != 16)) return RS_ERR_INVALID_ARGUMENT;
  if (k == 0) return RS_TOO_FEW_DATA_SHARDS;
  if (m == 0) return RS_TOO_FEW_PARITY_SHARDS;
  if (k + m > (field == 8 ? 256u : 65536u)) return RS_TOO_MANY_SHARDS;
  if (out_len != k * m) return RS_INCORRECT_SHARD_SIZE;
  if (field == 8) {
    std::vector<uint8_t> rows;
    parity_rows<F8>(k, m, rows);
    for (size_t t = 0; t < rows.size(); t++) out[t] = rows[t];
  } else {
    std::vector<uint16_t> rows;
    parity_rows<F16>(k, m, rows);
    memcpy(out, rows.data(), rows.size() * 2);
  }
  return RS_OK;
}

int rs_decode_rows(int field, size_t k, size_t m, const uint8_t *present, uint16_t *out, size_t out_len,
                   size_t *n_rows) {
  if (!present || !out || !n_rows || (field != 8 && field != 16)) return RS_ERR_INVALID_ARGUMENT;
  size_t n = k + m;
  Presence pres(n);
  for (size_t i = 0; i < n; i++)
    if (present[i]) pres.set(i);
  std::vector<uint32_t> surv, md, mp;
  split_pattern(pres, k, n, surv, md, mp);
  if (surv.size() < k) return RS_TOO_FEW_SHARDS_PRESENT;
  std::vector<size_t> nodes(surv.begin(), surv.end()), targets(md.begin(), md.end());
  targets.insert(targets.end(), mp.begin(), mp.end());
  *n_rows = targets.size();
  if (out_len < targets.size() * k) return RS_INCORRECT_SHARD_SIZE;
  if (field == 8) {
    std::vector<uint8_t> rows;
    lagrange_rows<F8>(nodes, targets, rows);
    for (size_t t = 0; t < rows.size(); t++) out[t] = rows[t];
  } else {
    std::vector<uint16_t> rows;
    lagrange_rows<F16>(nodes, targets, rows);
    memcpy(out, rows.data(), rows.size() * 2);
  }
  return RS_OK;
}

// ---------------------------------- rs8 --------------------------------------

int rs8_new(size_t k, size_t m, rs8_t **out) {
  if (!out) return RS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (k == 0) return RS_TOO_FEW_DATA_SHARDS;
  if (m == 0) return RS_TOO_FEW_PARITY_SHARDS;
  if (k + m > 256) return RS_TOO_MANY_SHARDS;
  int dev = 0;
  RSB_TRY(ensure_device(&dev));
  auto gen = std::make_shared<Gen8>();
  gen->device = dev;
  gen->k = k;
  gen->m = m;
  parity_rows<F8>(k, m, gen->rows);
  RSB_CU(cudaMalloc(&gen->d_rows, k * m));
  RSB_CU(cudaMemcpy(gen->d_rows, gen->rows.data(), k * m, cudaMemcpyHostToDevice));
  gen->fft = find_fft_shape(k, m);
  auto c = new (std::nothrow) rs8_codec();
  if (!c) return RS_ERR_ALLOC;
  c->gen = gen;
  c->plans = std::make_shared<PlanCache>();
  int st = make_exec(dev, c->exec);
  if (st) {
    delete c;
    return st;
  }
  *out = c;
  return RS_OK;
}

int rs8_clone(const rs8_t *codec, rs8_t **out) {
  if (!codec || !out) return RS_ERR_INVALID_ARGUMENT;
  auto c = new (std::nothrow) rs8_codec();
  if (!c) return RS_ERR_ALLOC;
  c->gen = codec->gen;
  c->plans = std::make_shared<PlanCache>();
  c->plans->copy_from(*codec->plans);
  c->route.store(codec->route.load());
  int st = make_exec(codec->gen->device, c->exec);
  if (st) {
    delete c;
    return st;
  }
  *out = c;
  return RS_OK;
}

void rs8_free(rs8_t *codec) { delete codec; }

size_t rs8_data_shard_count(const rs8_t *c) { return c ? c->gen->k : 0; }
size_t rs8_parity_shard_count(const rs8_t *c) { return c ? c->gen->m : 0; }
size_t rs8_total_shard_count(const rs8_t *c) { return c ? c->gen->k + c->gen->m : 0; }

int rs8_equal(const rs8_t *a, const rs8_t *b) {
  if (!a || !b) return 0;
  return a->gen->k == b->gen->k && a->gen->m == b->gen->m;
}

int rs8_parity_matrix(const rs8_t *c, uint8_t *out, size_t out_len) {
  if (!c || !out) return RS_ERR_INVALID_ARGUMENT;
  if (out_len != c->gen->rows.size()) return RS_INCORRECT_SHARD_SIZE;
  memcpy(out, c->gen->rows.data(), out_len);
  return RS_OK;
}

const char *rs8_encode_route(const rs8_t *c, size_t len) {
  if (!c) return "matrix";
  if (!use_fft8(c, len)) return "matrix";
  return c->gen->fft->gen ? "generator-bitsliced" : "fft-bitsliced";
}

int rs8_set_route(rs8_t *c, int route) {
  if (!c || route < 0 || route > 2) return RS_ERR_INVALID_ARGUMENT;
  c->route.store(route);
  return RS_OK;
}

// Host shards of a stripe too large for one round trip to pay: the columns are cut into
// chunks (encoding is column-wise, so each chunk is an independent stripe of shorter
// shards) that rotate over the pipeline streams. Each chunk's shards are copied in, the
// chunk is encoded, and its parity copied out on its stream; the copy-out of chunk c is
// issued after chunk c + 1 is queued, because a copy into pageable host memory returns
// only when it has finished: the next chunk's copy-in (another copy engine) and kernel
// then run while it waits. Pinned shards make every copy asynchronous.
static constexpr size_t kChunkStripeBytes = 8u << 20;  // data bytes per chunk (all shards)

static int encode8_host_chunked(rs8_t *c, uint8_t *const *shards, size_t len) {
  const Gen8 &g = *c->gen;
  Exec &ex = *c->exec;
  const size_t n = g.k + g.m;
  const size_t cols = std::max<size_t>(4096, (kChunkStripeBytes / g.k) & ~size_t(4095));
  const size_t n_chunks = (len + cols - 1) / cols;
  RSB_TRY(ex.pipe_streams());
  RSB_TRY(ex.pipe_buf.ensure(Exec::kPipe * n * cols));
  auto copy_out = [&](size_t ch) -> int {
    const size_t c0 = ch * cols, w = std::min(cols, len - c0);
    const int slot = (int)(ch % Exec::kPipe);
    uint8_t *base = ex.pipe_buf.ptr + slot * n * cols;
    for (size_t j = 0; j < g.m; j++)
      RSB_CU(cudaMemcpyAsync(shards[g.k + j] + c0, base + (g.k + j) * cols, w, cudaMemcpyDeviceToHost,
                             ex.pipe[slot]));
    return RS_OK;
  };
  for (size_t ch = 0; ch < n_chunks; ch++) {
    const size_t c0 = ch * cols, w = std::min(cols, len - c0);
    const int slot = (int)(ch % Exec::kPipe);
    cudaStream_t st = ex.pipe[slot];
    uint8_t *base = ex.pipe_buf.ptr + slot * n * cols;
    for (size_t i = 0; i < g.k; i++)
      RSB_CU(cudaMemcpyAsync(base + i * cols, shards[i] + c0, w, cudaMemcpyHostToDevice, st));
    RSB_TRY(encode8_strided(c, base, cols, 0, base + g.k * cols, cols, 0, 1, w, st));
    if (ch > 0) RSB_TRY(copy_out(ch - 1));
  }
  RSB_TRY(copy_out(n_chunks - 1));
  for (auto st : ex.pipe) RSB_CU(cudaStreamSynchronize(st));
  return RS_OK;
}

// src/reedsolomon.rs:271-278 then :701-722
int rs8_encode(rs8_t *c, uint8_t *const *shards, size_t n_shards, size_t len) {
  if (!c || !shards) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  size_t n = g.k + g.m;
  if (n_shards != n) return n_shards < n ? RS_TOO_FEW_SHARDS : RS_TOO_MANY_SHARDS;
  RSB_TRY(check_equal_lengths(n, len));
  Exec &ex = *c->exec;
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  for (size_t i = 0; i < n; i++)
    if (!shards[i]) return RS_ERR_INVALID_ARGUMENT;
  const size_t pitch = pitch16(len);
  if (!host_staged(n * pitch)) return encode8_host_chunked(c, shards, len);
  // The shards are gathered into pinned memory by host threads and cross the link as one
  // copy each way: pageable copies of separate shards ran at 8-23 GB/s host to device and
  // 3-13 GB/s back on B200 hosts, against ~55 GB/s pinned.
  RSB_TRY(ex.buf.ensure(n * pitch));
  RSB_TRY(ex.io.ensure(n * pitch));
  uint8_t *h = ex.io.ptr;
  gather_rows(h, pitch, g.k, len, [&](size_t i) { return shards[i]; });
  RSB_CU(cudaMemcpyAsync(ex.buf.ptr, h, g.k * pitch, cudaMemcpyHostToDevice, ex.stream));
  RSB_TRY(encode8_strided(c, ex.buf.ptr, pitch, 0, ex.buf.ptr + g.k * pitch, pitch, 0, 1, len, ex.stream));
  RSB_CU(cudaMemcpyAsync(h + g.k * pitch, ex.buf.ptr + g.k * pitch, g.m * pitch, cudaMemcpyDeviceToHost,
                         ex.stream));
  RSB_CU(cudaStreamSynchronize(ex.stream));
  scatter_rows(h + g.k * pitch, pitch, g.m, len, [&](size_t j) { return shards[g.k + j]; });
  return RS_OK;
}

// src/reedsolomon.rs:284-309
int rs8_encode_sep(rs8_t *c, const uint8_t *const *data, size_t n_data, uint8_t *const *parity,
                   size_t n_parity, size_t len) {
  if (!c || !data || !parity) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  if (n_data != g.k) return n_data < g.k ? RS_TOO_FEW_DATA_SHARDS : RS_TOO_MANY_DATA_SHARDS;
  if (n_parity != g.m) return n_parity < g.m ? RS_TOO_FEW_PARITY_SHARDS : RS_TOO_MANY_PARITY_SHARDS;
  if (len == 0) return RS_OK;
  std::vector<uint8_t *> all(g.k + g.m);
  for (size_t i = 0; i < g.k; i++) all[i] = const_cast<uint8_t *>(data[i]);
  for (size_t j = 0; j < g.m; j++) all[g.k + j] = parity[j];
  return rs8_encode(c, all.data(), all.size(), len);
}

// src/reedsolomon.rs:667-697
int rs8_encode_rows(rs8_t *c, const uint8_t *data, size_t data_len, size_t row_len,
                    uint8_t *parity, size_t parity_len) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  if (data_len != g.k * row_len) return RS_INCORRECT_SHARD_SIZE;
  if (parity_len != g.m * row_len) return RS_INCORRECT_SHARD_SIZE;
  if (row_len == 0) return RS_OK;
  if (!data || !parity) return RS_ERR_INVALID_ARGUMENT;
  Exec &ex = *c->exec;
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  size_t n = g.k + g.m;
  const size_t pitch = pitch16(row_len);
  RSB_TRY(ex.buf.ensure(n * pitch));
  uint8_t *d_par = ex.buf.ptr + g.k * pitch;
  if (host_staged(n * pitch)) {  // as rs8_encode
    RSB_TRY(ex.io.ensure(n * pitch));
    uint8_t *h = ex.io.ptr;
    gather_rows(h, pitch, g.k, row_len, [&](size_t i) { return data + i * row_len; });
    RSB_CU(cudaMemcpyAsync(ex.buf.ptr, h, g.k * pitch, cudaMemcpyHostToDevice, ex.stream));
    RSB_TRY(encode8_strided(c, ex.buf.ptr, pitch, 0, d_par, pitch, 0, 1, row_len, ex.stream));
    RSB_CU(cudaMemcpyAsync(h + g.k * pitch, d_par, g.m * pitch, cudaMemcpyDeviceToHost, ex.stream));
    RSB_CU(cudaStreamSynchronize(ex.stream));
    scatter_rows(h + g.k * pitch, pitch, g.m, row_len, [&](size_t j) { return parity + j * row_len; });
    return RS_OK;
  }
  RSB_CU(cudaMemcpy2DAsync(ex.buf.ptr, pitch, data, row_len, row_len, g.k, cudaMemcpyHostToDevice, ex.stream));
  RSB_TRY(encode8_strided(c, ex.buf.ptr, pitch, 0, d_par, pitch, 0, 1, row_len, ex.stream));
  RSB_CU(cudaMemcpy2DAsync(parity, row_len, d_par, pitch, row_len, g.m, cudaMemcpyDeviceToHost, ex.stream));
  RSB_CU(cudaStreamSynchronize(ex.stream));
  return RS_OK;
}

int rs8_encode_batch(rs8_t *c, const uint8_t *data, size_t data_stride, uint8_t *parity, size_t parity_stride,
                     size_t n_stripes, size_t row_len) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  if (n_stripes == 0 || row_len == 0) return RS_OK;
  if (!data || !parity) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  const size_t din = g.k * row_len, dout = g.m * row_len;
  if (data_stride < din || parity_stride < dout) return RS_INCORRECT_SHARD_SIZE;
  Exec &ex = *c->exec;
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  RSB_TRY(ex.pipe_streams());
  // Device rows at a 16-byte pitch (pitched copies when row_len is not a multiple).
  const size_t pitch = pitch16(row_len), ddin = g.k * pitch, ddout = g.m * pitch;
  // Chunks of about 64 MiB per slot, one slot per stream.
  const size_t per = ddin + ddout;
  size_t chunk = std::max<size_t>(1, ((size_t)64 << 20) / per);
  chunk = std::min(chunk, n_stripes);
  RSB_TRY(ex.pipe_buf.ensure(Exec::kPipe * chunk * per));
  for (size_t s0 = 0, it = 0; s0 < n_stripes; s0 += chunk, it++) {
    const size_t cnt = std::min(chunk, n_stripes - s0);
    const int slot = (int)(it % Exec::kPipe);
    cudaStream_t st = ex.pipe[slot];
    uint8_t *d_in = ex.pipe_buf.ptr + slot * chunk * per;
    uint8_t *d_out = d_in + chunk * ddin;
    if (pitch == row_len && data_stride == din) {
      RSB_CU(cudaMemcpyAsync(d_in, data + s0 * din, cnt * din, cudaMemcpyHostToDevice, st));
    } else if (data_stride == din) {  // stripes back to back: one pitched copy of all rows
      RSB_CU(cudaMemcpy2DAsync(d_in, pitch, data + s0 * din, row_len, row_len, cnt * g.k, cudaMemcpyHostToDevice,
                               st));
    } else {
      for (size_t s = 0; s < cnt; s++)
        RSB_CU(cudaMemcpy2DAsync(d_in + s * ddin, pitch, data + (s0 + s) * data_stride, row_len, row_len, g.k,
                                 cudaMemcpyHostToDevice, st));
    }
    RSB_TRY(encode8_strided(c, d_in, pitch, ddin, d_out, pitch, ddout, cnt, row_len, st));
    if (pitch == row_len && parity_stride == dout) {
      RSB_CU(cudaMemcpyAsync(parity + s0 * dout, d_out, cnt * dout, cudaMemcpyDeviceToHost, st));
    } else if (parity_stride == dout) {
      RSB_CU(cudaMemcpy2DAsync(parity + s0 * dout, row_len, d_out, pitch, row_len, cnt * g.m, cudaMemcpyDeviceToHost,
                               st));
    } else {
      for (size_t s = 0; s < cnt; s++)
        RSB_CU(cudaMemcpy2DAsync(parity + (s0 + s) * parity_stride, row_len, d_out + s * ddout, pitch, row_len, g.m,
                                 cudaMemcpyDeviceToHost, st));
    }
  }
  for (auto st : ex.pipe) RSB_CU(cudaStreamSynchronize(st));
  return RS_OK;
}

// src/reedsolomon.rs:430-463
int rs8_verify(rs8_t *c, const uint8_t *const *shards, size_t n_shards, size_t len, int *ok) {
  if (!c || !shards || !ok) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  size_t n = g.k + g.m;
  if (n_shards != n) return n_shards < n ? RS_TOO_FEW_SHARDS : RS_TOO_MANY_SHARDS;
  RSB_TRY(check_equal_lengths(n, len));
  Exec &ex = *c->exec;
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  const size_t pitch = pitch16(len);
  RSB_TRY(ex.buf.ensure(n * pitch));
  RSB_TRY(ex.aux.ensure(64));
  for (size_t i = 0; i < n; i++)
    if (!shards[i]) return RS_ERR_INVALID_ARGUMENT;
  if (host_staged(n * pitch)) {  // as rs8_encode: one copy of the gathered stripe
    RSB_TRY(ex.io.ensure(n * pitch));
    gather_rows(ex.io.ptr, pitch, n, len, [&](size_t i) { return shards[i]; });
    RSB_CU(cudaMemcpyAsync(ex.buf.ptr, ex.io.ptr, n * pitch, cudaMemcpyHostToDevice, ex.stream));
  } else {
    for (size_t i = 0; i < n; i++)
      RSB_CU(cudaMemcpyAsync(ex.buf.ptr + i * pitch, shards[i], len, cudaMemcpyHostToDevice, ex.stream));
  }
  uint32_t *flag = reinterpret_cast<uint32_t *>(ex.aux.ptr);
  RSB_CU(cudaMemsetAsync(flag, 0, 4, ex.stream));
  ApplyArgs a{};
  a.in_base = ex.buf.ptr;
  a.in_row_stride = pitch;
  a.out_base = ex.buf.ptr + g.k * pitch;
  a.out_row_stride = pitch;
  a.coeffs = g.d_rows;
  a.k = (uint32_t)g.k;
  a.rows = (uint32_t)g.m;
  a.len = len;
  a.n_stripes = 1;
  a.mismatch = flag;
  RSB_TRY(launch_gf8(a, nullptr, true, ex.stream));
  uint32_t h = 0;
  RSB_CU(cudaMemcpyAsync(&h, flag, 4, cudaMemcpyDeviceToHost, ex.stream));
  RSB_CU(cudaStreamSynchronize(ex.stream));
  *ok = h ? 0 : 1;
  return RS_OK;
}

int rs8_reconstruct(rs8_t *c, uint8_t *const *shards, const size_t *lens, const uint8_t *present,
                    size_t n_shards, int data_only) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  return reconstruct8(*c->gen, c->plans.get(), nullptr, *c->exec, shards, lens, present, n_shards,
                      data_only != 0, false, nullptr);
}

// src/reedsolomon.rs:514-535
int rs8_reconstruct_rows(rs8_t *c, uint8_t *rows, size_t rows_len, size_t row_len,
                         const uint8_t *present, size_t n_present) {
  if (!c || !present) return RS_ERR_INVALID_ARGUMENT;
  size_t n = c->gen->k + c->gen->m;
  if (n_present != n) return RS_INVALID_SHARD_FLAGS;
  if (row_len == 0) return RS_EMPTY_SHARD;
  if (rows_len != n * row_len) return RS_INCORRECT_SHARD_SIZE;
  if (!rows) return RS_ERR_INVALID_ARGUMENT;
  std::vector<uint8_t *> shards(n);
  std::vector<size_t> lens(n, row_len);
  for (size_t i = 0; i < n; i++) shards[i] = rows + i * row_len;
  return rs8_reconstruct(c, shards.data(), lens.data(), present, n, 0);
}

// src/reedsolomon.rs:484-505
int rs8_prepare_decode(rs8_t *c, const uint8_t *present, size_t n_present, rs8_dec_t **out) {
  if (!c || !out) return RS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const Gen8 &g = *c->gen;
  size_t n = g.k + g.m;
  if (n_present != n) return RS_INVALID_SHARD_FLAGS;
  if (!present) return RS_ERR_INVALID_ARGUMENT;
  Presence pres(n);
  size_t count = 0;
  for (size_t i = 0; i < n; i++)
    if (present[i]) {
      pres.set(i);
      count++;
    }
  if (count < g.k) return RS_TOO_FEW_SHARDS_PRESENT;
  std::shared_ptr<const Plan> plan;
  RSB_TRY(plan8_for(g, *c->plans, *c->exec, pres, plan));
  auto d = new (std::nothrow) rs8_decoder();
  if (!d) return RS_ERR_ALLOC;
  d->gen = c->gen;
  d->plan = plan;
  d->exec = c->exec;
  *out = d;
  return RS_OK;
}

int rs8_dec_reconstruct(rs8_dec_t *d, uint8_t *const *shards, const size_t *lens,
                        const uint8_t *present, size_t n_shards, int data_only) {
  if (!d) return RS_ERR_INVALID_ARGUMENT;
  return reconstruct8(*d->gen, nullptr, d->plan.get(), *d->exec, shards, lens, present, n_shards,
                      data_only != 0, false, nullptr);
}

int rs8_dec_clone(const rs8_dec_t *d, rs8_dec_t **out) {
  if (!d || !out) return RS_ERR_INVALID_ARGUMENT;
  auto c = new (std::nothrow) rs8_decoder(*d);
  if (!c) return RS_ERR_ALLOC;
  *out = c;
  return RS_OK;
}

void rs8_dec_free(rs8_dec_t *d) { delete d; }

// ---------------------------- rs8 device variants ----------------------------

int rs8_encode_dev(rs8_t *c, uint8_t *const *d_shards, size_t n_shards, size_t len, void *stream) {
  if (!c || !d_shards) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  size_t n = g.k + g.m;
  if (n_shards != n) return n_shards < n ? RS_TOO_FEW_SHARDS : RS_TOO_MANY_SHARDS;
  RSB_TRY(check_equal_lengths(n, len));
  RSB_CU(cudaSetDevice(g.device));
  cudaStream_t st = (cudaStream_t)stream;
  if (use_fft8(c, len)) return launch_fft8_ptrs(*g.fft, d_shards, len, st);
  PtrTable pt;
  for (size_t i = 0; i < g.k; i++) pt.in[i] = d_shards[i];
  for (size_t j = 0; j < g.m; j++) pt.out[j] = d_shards[g.k + j];
  ApplyArgs a{};
  a.coeffs = g.d_rows;
  a.k = (uint32_t)g.k;
  a.rows = (uint32_t)g.m;
  a.len = len;
  a.n_stripes = 1;
  return launch_gf8(a, &pt, false, st);
}

int rs8_encode_sep_dev(rs8_t *c, const uint8_t *const *d_data, size_t n_data, uint8_t *const *d_parity,
                       size_t n_parity, size_t len, void *stream) {
  if (!c || !d_data || !d_parity) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  if (n_data != g.k) return n_data < g.k ? RS_TOO_FEW_DATA_SHARDS : RS_TOO_MANY_DATA_SHARDS;
  if (n_parity != g.m) return n_parity < g.m ? RS_TOO_FEW_PARITY_SHARDS : RS_TOO_MANY_PARITY_SHARDS;
  if (len == 0) return RS_OK;
  std::vector<uint8_t *> all(g.k + g.m);
  for (size_t i = 0; i < g.k; i++) all[i] = const_cast<uint8_t *>(d_data[i]);
  for (size_t j = 0; j < g.m; j++) all[g.k + j] = d_parity[j];
  return rs8_encode_dev(c, all.data(), all.size(), len, stream);
}

int rs8_encode_rows_dev(rs8_t *c, const uint8_t *d_data, size_t row_len, uint8_t *d_parity,
                        void *stream) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  if (row_len == 0) return RS_OK;
  if (!d_data || !d_parity) return RS_ERR_INVALID_ARGUMENT;
  RSB_CU(cudaSetDevice(c->gen->device));
  return encode8_strided(c, d_data, row_len, 0, d_parity, row_len, 0, 1, row_len, (cudaStream_t)stream);
}

int rs8_encode_batch_dev(rs8_t *c, const uint8_t *d_data, size_t data_stride, uint8_t *d_parity,
                         size_t parity_stride, size_t n_stripes, size_t row_len, void *stream) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  if (row_len == 0 || n_stripes == 0) return RS_OK;
  if (!d_data || !d_parity) return RS_ERR_INVALID_ARGUMENT;
  RSB_CU(cudaSetDevice(c->gen->device));
  return encode8_strided(c, d_data, row_len, data_stride, d_parity, row_len, parity_stride, n_stripes,
                         row_len, (cudaStream_t)stream);
}

int rs8_verify_dev(rs8_t *c, const uint8_t *const *d_shards, size_t n_shards, size_t len, int *ok,
                   void *stream) {
  if (!c || !d_shards || !ok) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  size_t n = g.k + g.m;
  if (n_shards != n) return n_shards < n ? RS_TOO_FEW_SHARDS : RS_TOO_MANY_SHARDS;
  RSB_TRY(check_equal_lengths(n, len));
  Exec &ex = *c->exec;
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  cudaStream_t st = (cudaStream_t)stream;
  RSB_TRY(ex.aux.ensure(64));
  uint32_t *flag = reinterpret_cast<uint32_t *>(ex.aux.ptr);
  RSB_CU(cudaMemsetAsync(flag, 0, 4, st));
  PtrTable pt;
  for (size_t i = 0; i < g.k; i++) pt.in[i] = d_shards[i];
  for (size_t j = 0; j < g.m; j++) pt.out[j] = const_cast<uint8_t *>(d_shards[g.k + j]);
  ApplyArgs a{};
  a.coeffs = g.d_rows;
  a.k = (uint32_t)g.k;
  a.rows = (uint32_t)g.m;
  a.len = len;
  a.n_stripes = 1;
  a.mismatch = flag;
  RSB_TRY(launch_gf8(a, &pt, true, st));
  uint32_t h = 0;
  RSB_CU(cudaMemcpyAsync(&h, flag, 4, cudaMemcpyDeviceToHost, st));
  RSB_CU(cudaStreamSynchronize(st));
  *ok = h ? 0 : 1;
  return RS_OK;
}

int rs8_reconstruct_dev(rs8_t *c, uint8_t *const *d_shards, const size_t *lens, const uint8_t *present,
                        size_t n_shards, int data_only, void *stream) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  return reconstruct8(*c->gen, c->plans.get(), nullptr, *c->exec, d_shards, lens, present, n_shards,
                      data_only != 0, true, (cudaStream_t)stream, c->route.load());
}

int rs8_reconstruct_batch_dev(rs8_t *c, uint8_t *d_rows, size_t stripe_stride, size_t n_stripes,
                              size_t row_len, const uint8_t *present, int data_only, int *statuses,
                              void *stream) {
  if (!c || !present) return RS_ERR_INVALID_ARGUMENT;
  if (n_stripes == 0) return RS_OK;
  if (row_len == 0) return RS_EMPTY_SHARD;
  if (!d_rows) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  const size_t k = g.k, n = g.k + g.m;
  cudaStream_t st = (cudaStream_t)stream;
  // Where the shape has a compiled encode kernel, missing parity is regenerated by it
  // from the data rows once they are whole, storing only the missing rows: the matrix
  // route then applies (missing data) x k decode coefficients per column instead of
  // (missing data + missing parity) x k, where that pays (regen_parity_pays). Measured
  // on B200 (RS(32,32), 1..m erasures per stripe, both forms timed in one process):
  // +10% at 4 KiB shards, +21% at 16 KiB, +28% at 64 KiB.
  const bool split = !data_only && use_fft8(c, row_len);
  const int route = c->route.load();
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  // Device layout: one uploaded header (survivors | targets, m per stripe | target
  // counts | parity items | parity masks), then the decode rows and plan statuses the
  // plan kernel writes. The header is filled in pinned host memory as the stripes are
  // scanned and goes up in one copy.
  const size_t b_surv = n_stripes * k * 2, b_targ = n_stripes * g.m * 2, b_nt = n_stripes * 2;
  const size_t o_targ = al(b_surv), o_nt = o_targ + al(b_targ), o_items = o_nt + al(b_nt);
  const size_t max_header = o_items + al(n_stripes * sizeof(FftItem)) + al(n_stripes * 4 * sizeof(uint32_t));
  Exec &ex = *c->exec;
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  HostStage::Buf *hb = nullptr;
  RSB_TRY(ex.stage.acquire(max_header, hb));
  uint8_t *h = hb->ptr;
  uint16_t *surv = reinterpret_cast<uint16_t *>(h), *targ = reinterpret_cast<uint16_t *>(h + o_targ),
           *ntarg = reinterpret_cast<uint16_t *>(h + o_nt);
  FftItem *items = reinterpret_cast<FftItem *>(h + o_items);  // split: stripes with missing parity
  std::vector<uint32_t> masks;                                 // split: 4 words of missing parity rows per item
  size_t n_items = 0;
  uint32_t max_rows = 0;
  size_t live = 0;
  // Per stripe, one branch-free pass sorts the shard indexes into present, missing data
  // and missing parity (random flags made the branchy scan mispredict: 2.7x slower).
  uint16_t ls[257], md[257], mp[257];
  for (size_t s = 0; s < n_stripes; s++) {
    const uint8_t *pf = present + s * n;
    uint16_t *sv = surv + s * k, *tg = targ + s * g.m;
    size_t ns = 0, r = 0, n_mp = 0;
    for (size_t i = 0; i < n; i++) {
      const size_t pr = pf[i] != 0, dat = i < k;
      ls[ns] = md[r] = mp[n_mp] = (uint16_t)i;
      ns += pr;
      r += (pr ^ 1) & dat;
      n_mp += (pr ^ 1) & (dat ^ 1);
    }
    memcpy(sv, ls, 2 * std::min(ns, k));
    ntarg[s] = 0;
    if (statuses) statuses[s] = RS_OK;
    if (ns == n) continue;
    if (ns < k) {
      if (statuses) statuses[s] = RS_TOO_FEW_SHARDS_PRESENT;
      for (size_t t = 0; t < k; t++) sv[t] = (uint16_t)t;
      continue;
    }
    memcpy(tg, md, 2 * r);  // r <= n - ns <= m once k shards are present
    if (split && n_mp && regen_parity_pays(g, n_mp, route)) {
      FftItem f{};
      f.in_base = d_rows + s * stripe_stride;
      f.out_base = d_rows + s * stripe_stride + k * row_len;
      f.row_stride = row_len;
      f.len = row_len;
      f.group_begin = n_items ? items[n_items - 1].group_begin + (row_len + 31) / 32 : 0;
      items[n_items++] = f;
      masks.resize(masks.size() + 4, 0u);
      for (size_t j = 0; j < n_mp; j++) masks[masks.size() - 4 + (mp[j] - k) / 32] |= 1u << ((mp[j] - k) % 32);
    } else if (!data_only) {
      for (size_t j = 0; j < n_mp; j++) tg[r++] = mp[j];
    }
    ntarg[s] = (uint16_t)r;
    max_rows = std::max<uint32_t>(max_rows, (uint32_t)r);
    live++;
  }
  if (live == 0) return RS_OK;
  const size_t o_masks = o_items + al(n_items * sizeof(FftItem));
  const size_t header = o_masks + masks.size() * sizeof(uint32_t);
  if (!masks.empty()) memcpy(h + o_masks, masks.data(), masks.size() * sizeof(uint32_t));
  const size_t o_rows = al(header), b_rows = n_stripes * (size_t)g.m * k;
  const size_t o_stat = o_rows + al(b_rows);
  RSB_TRY(ex.aux.ensure(o_stat + al(n_stripes * sizeof(int))));
  uint8_t *base = ex.aux.ptr;
  RSB_CU(cudaMemcpyAsync(base, h, header, cudaMemcpyHostToDevice, st));
  RSB_TRY(ex.stage.release(*hb, st));
  if (max_rows > 0) {
    PlanArgs pa{};
    pa.gen = g.d_rows;
    pa.k = (uint32_t)k;
    pa.m = (uint32_t)g.m;
    pa.survivors = reinterpret_cast<uint16_t *>(base);
    pa.targets = reinterpret_cast<uint16_t *>(base + o_targ);
    pa.n_targets = reinterpret_cast<uint16_t *>(base + o_nt);
    pa.max_rows = (uint32_t)g.m;
    pa.out = base + o_rows;
    pa.status = reinterpret_cast<int *>(base + o_stat);
    size_t smem = plan_smem((uint32_t)k).total;
    if (smem > 48 * 1024)
      RSB_CU(cudaFuncSetAttribute(gf8_plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    gf8_plan_kernel<<<(unsigned)n_stripes, 256, smem, st>>>(pa);
    g_launches++;
    RSB_CU(cudaGetLastError());
    ApplyArgs a{};
    a.in_base = d_rows;
    a.in_row_stride = row_len;
    a.in_stripe_stride = stripe_stride;
    a.out_base = d_rows;
    a.out_row_stride = row_len;
    a.out_stripe_stride = stripe_stride;
    a.coeffs = base + o_rows;
    a.coeff_stripe_stride = (uint64_t)g.m * k;
    a.rows_per_stripe = pa.n_targets;
    a.in_map = pa.survivors;
    a.out_map = pa.targets;
    a.k = (uint32_t)k;
    a.rows = (uint32_t)g.m;
    a.len = row_len;
    a.n_stripes = (uint32_t)n_stripes;
    RSB_TRY(launch_gf8(a, nullptr, false, st));
  }
  if (n_items == 0) return RS_OK;
  const uint64_t groups = items[n_items - 1].group_begin + (row_len + 31) / 32;
  return launch_fft8_items(*g.fft, reinterpret_cast<const FftItem *>(base + o_items), (uint32_t)n_items, groups,
                           st, reinterpret_cast<const uint32_t *>(base + o_masks),
                           ((reinterpret_cast<uintptr_t>(d_rows) | stripe_stride | row_len) & 15) != 0);
}

// ------------------------------- gf slices -----------------------------------

int gf8_mul_slice_dev(uint8_t *d_out, const uint8_t *d_in, size_t n, uint8_t c, int xor_into,
                      void *stream) {
  if (n == 0) return RS_OK;
  if (!d_out || !d_in) return RS_ERR_INVALID_ARGUMENT;
  uint64_t tiles = (n + kTileBytes - 1) / kTileBytes;
  unsigned grid = (unsigned)std::min<uint64_t>(tiles, 148 * 16);
  gf8_mul_slice_kernel<<<grid, kThreads, 0, (cudaStream_t)stream>>>(d_out, d_in, n, c, xor_into);
  g_launches++;
  RSB_CU(cudaGetLastError());
  return RS_OK;
}

int gf8_mul_slice(uint8_t *out, size_t out_len, const uint8_t *in, size_t in_len, uint8_t c,
                  int xor_into) {
  if (out_len != in_len) return RS_ERR_LENGTH_MISMATCH;
  if (out_len == 0) return RS_OK;
  if (!out || !in) return RS_ERR_INVALID_ARGUMENT;
  RSB_TRY(ensure_device(nullptr));
  uint8_t *d = nullptr;
  RSB_CU(cudaMalloc(&d, 2 * out_len));
  int st = RS_OK;
  do {
    if (cudaMemcpy(d, in, in_len, cudaMemcpyHostToDevice) != cudaSuccess) { st = RS_ERR_CUDA; break; }
    if (xor_into && cudaMemcpy(d + out_len, out, out_len, cudaMemcpyHostToDevice) != cudaSuccess) { st = RS_ERR_CUDA; break; }
    st = gf8_mul_slice_dev(d + out_len, d, out_len, c, xor_into, nullptr);
    if (st) break;
    if (cudaMemcpy(out, d + out_len, out_len, cudaMemcpyDeviceToHost) != cudaSuccess) st = RS_ERR_CUDA;
  } while (0);
  if (st == RS_ERR_CUDA) set_cuda_error(cudaGetLastError(), "gf8_mul_slice copy");
  cudaFree(d);
  return st;
}

}  // extern "C"
