// C ABI of the ReedSolomon16 (GF((2^8)^2) tower) coder: include/rs_b200.h.
// Split-plane wire: a shard of 2N bytes is N low bytes then N high bytes
// (src/reedsolomon16.rs:4-7).
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "runtime.hpp"
#include "codec8.hpp"
#include "gf_host.hpp"
#include "fft16.hpp"
#include "kernels_fft.cuh"
#include "kernels_lagrange.cuh"
#include "kernels_matrix.cuh"

namespace rsb {

// Karatsuba constants of a tower coefficient c = (c_hi, c_lo):
// k0 = c_lo, k1 = c_hi ^ c_lo, k2 = c_hi * 32 (src/reedsolomon16.rs:61-94).
static inline uint32_t split16(uint16_t c) {
  uint8_t hi = c >> 8, lo = c & 0xff;
  return (uint32_t)lo | ((uint32_t)(uint8_t)(hi ^ lo) << 8) | ((uint32_t)gf8_mul(hi, 32) << 16);
}

struct Gen16 {
  int device = 0;
  size_t k = 0, m = 0;
  uint32_t *d_split = nullptr;
  // FFT route (any k >= 2): the step program and its constants on the device.
  std::unique_ptr<Fft16Program> fft;
  uint16_t *d_fft_cols = nullptr;
  ~Gen16() {
    cudaSetDevice(device);
    if (d_split) cudaFree(d_split);
    if (d_fft_cols) cudaFree(d_fft_cols);
  }
};

static int build_fft16(Gen16 &g) {
  auto p = std::make_unique<Fft16Program>();
  if (!fft16_build(g.k, g.m, *p)) return RS_OK;
  RSB_CU(cudaMalloc(&g.d_fft_cols, p->cols.size() * 2));
  RSB_CU(cudaMemcpy(g.d_fft_cols, p->cols.data(), p->cols.size() * 2, cudaMemcpyHostToDevice));
  g.fft = std::move(p);
  return RS_OK;
}

// FFT-route encode with stream-ordered scratch. 48 MiB keeps a wave's registers
// resident in L2 (126 MB) across the passes; larger scratch measured slower.
static int fft16_encode(const Gen16 &g, const uint8_t *in_base, uint64_t in_row, uint64_t in_stripe,
                        uint8_t *out_base, uint64_t out_row, uint64_t out_stripe, size_t n_stripes, size_t len,
                        uint8_t *const *d_ptrs, cudaStream_t st) {
  const size_t bytes = fft16_scratch_bytes(*g.fft, n_stripes, len, kFft16ScratchBudget);
  uint8_t *scratch = nullptr;
  RSB_CU(scratch_alloc(reinterpret_cast<void **>(&scratch), bytes, st));
  int rc = fft16_run(*g.fft, g.d_fft_cols, scratch, bytes, in_base, in_row, in_stripe, out_base, out_row, out_stripe,
                     d_ptrs, n_stripes, len, st);
  scratch_free(scratch, st);
  return rc;
}

// Lagrange rows from `nodes` to `targets`, built on the device as split constants
// (kernels_lagrange.cuh). *out is a fresh device allocation of targets x nodes u32.
static int lagrange16_device(const std::vector<uint16_t> &nodes, const std::vector<uint16_t> &targets,
                             uint32_t **out) {
  const uint32_t k = (uint32_t)nodes.size(), nt = (uint32_t)targets.size();
  const size_t entries = std::max<size_t>((size_t)k * nt, 1);
  RSB_CU(cudaMalloc(out, entries * 4));
  if (!k || !nt) return RS_OK;
  // scratch: nodes | targets | w | ell | hit
  size_t off_t = (k * 2 + 15) & ~size_t(15), off_w = off_t + ((nt * 2 + 15) & ~size_t(15));
  size_t off_e = off_w + ((k * 2 + 15) & ~size_t(15)), off_h = off_e + ((nt * 2 + 15) & ~size_t(15));
  size_t bytes = off_h + nt * 4;
  uint8_t *s = nullptr;
  RSB_CU(cudaMalloc(&s, bytes));
  int st = RS_OK;
  do {
    uint16_t *d_nodes = reinterpret_cast<uint16_t *>(s), *d_t = reinterpret_cast<uint16_t *>(s + off_t);
    uint16_t *d_w = reinterpret_cast<uint16_t *>(s + off_w), *d_ell = reinterpret_cast<uint16_t *>(s + off_e);
    uint32_t *d_hit = reinterpret_cast<uint32_t *>(s + off_h);
    if (cudaMemcpy(d_nodes, nodes.data(), k * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_t, targets.data(), nt * 2, cudaMemcpyHostToDevice) != cudaSuccess) {
      st = RS_ERR_CUDA;
      break;
    }
    lagrange16_weights<<<(k + 255) / 256, 256>>>(d_nodes, k, d_w);
    lagrange16_ell<<<(nt + 255) / 256, 256>>>(d_nodes, k, d_t, nt, d_ell, d_hit);
    uint64_t n = (uint64_t)k * nt;
    lagrange16_rows<<<(unsigned)((n + 255) / 256), 256>>>(d_nodes, k, d_t, nt, d_w, d_ell, d_hit, *out, nullptr);
    g_launches += 3;
    if (cudaDeviceSynchronize() != cudaSuccess) st = RS_ERR_CUDA;
  } while (0);
  if (st) set_cuda_error(cudaGetLastError(), "lagrange16_device");
  cudaFree(s);
  return st;
}

static int launch_gf16(const Apply16Args &a, bool verify, cudaStream_t st) {
  if (a.n_sym == 0 || a.rows == 0 || a.n_stripes == 0) return RS_OK;
  Apply16Args b = a;
  dim3 grid;
  unsigned threads;
  gf16_launch_shape(b, sm_count(), grid, threads);
  if (verify)
    gf16_matrix_kernel<4, true><<<grid, threads, 0, st>>>(b);
  else
    gf16_matrix_kernel<4, false><<<grid, threads, 0, st>>>(b);
  g_launches++;
  RSB_CU(cudaGetLastError());
  return RS_OK;
}

// Shard-length rule of the tower coder, src/reedsolomon16.rs:758-772.
static int check_len16(size_t len) {
  if (len == 0) return RS_EMPTY_SHARD;
  if (len % 2) return RS_INCORRECT_SHARD_SIZE;
  return RS_OK;
}

}  // namespace rsb

using namespace rsb;

struct rs16_codec {
  std::shared_ptr<const Gen16> gen;
  std::shared_ptr<PlanCache> plans;
  std::shared_ptr<Exec> exec;
  std::atomic<int> route{0};  // 0 automatic, 1 matrix, 2 FFT where available
  // k + m <= 256: every evaluation point 0..k+m-1 lies in the GF(2^8) subfield
  // (high byte 0), so every generator and decode coefficient does too, and a subfield
  // constant c multiplies a tower symbol plane by plane: c(hi*y + lo) = (c*hi)y + c*lo.
  // The tower code is then ReedSolomon(k, m) applied to every byte of the split-plane
  // shards, and the automatic route runs it on the GF(2^8) codec's kernels.
  rs8_t *sub = nullptr;
  ~rs16_codec() { rs8_free(sub); }
};

namespace rsb {
// The GF(2^8) codec that runs this shape on the automatic route, or null.
static rs8_t *subfield(const rs16_codec *c) { return c->route.load() == 0 ? c->sub : nullptr; }

// Whether an encode of n_stripes stripes of len-byte shards runs on the subfield codec:
// always where that codec has a compiled kernel for the call (FFT or generator shapes);
// on its matrix kernel only when the tower FFT is not estimated to finish first.
static bool subfield_encode(const rs16_codec *c, size_t len, size_t n_stripes) {
  rs8_t *sub = subfield(c);
  if (!sub) return false;
  if (use_fft8(sub, len) || !c->gen->fft) return true;
  return !fft16_faster_than_gf8_matrix(*c->gen->fft, len, std::max<size_t>(n_stripes, 1));
}

// len / n_stripes: the call's shard length and stripe count; len 0: the shape alone
// (its throughput estimate, as rs16_encode_route reports it).
static bool use_fft16(const rs16_codec *c, size_t len = 0, size_t n_stripes = 1) {
  int r = c->route.load();
  if (r == 1 || !c->gen->fft) return false;
  if (r == 2) return true;
  return len == 0 ? fft16_preferred(*c->gen->fft) : fft16_faster(*c->gen->fft, len, n_stripes);
}
}  // namespace rsb

struct rs16_decoder {
  std::shared_ptr<const Gen16> gen;
  std::shared_ptr<const Plan> plan;
  std::shared_ptr<Exec> exec;
  // k + m <= 256 on the automatic route: the GF(2^8) codec's prepared decoder of the same
  // pattern, which rebuilds the shards once the tower's checks have passed.
  std::shared_ptr<rs8_dec_t> sub;
};

namespace rsb {

// Plan of one presence pattern: closed-form Lagrange rows from the survivors to each
// missing shard (data ascending, then parity ascending), built on the device.
// route: 0 by estimated cost, 1 matrix (Lagrange rows), 2 FFT decode.
static int plan16_for(const Gen16 &g, PlanCache &cache, const Presence &pres,
                      std::shared_ptr<const Plan> &out, int route = 0) {
  out = cache.find(pres);
  if (out) return RS_OK;
  auto plan = std::make_shared<Plan>();
  plan->presence = pres;
  plan->device = g.device;
  split_pattern(pres, g.k, g.k + g.m, plan->survivors, plan->missing_data, plan->missing_parity);
  if (plan->survivors.size() < g.k) return RS_TOO_FEW_SHARDS_PRESENT;
  std::vector<uint16_t> nodes(plan->survivors.begin(), plan->survivors.end());
  std::vector<uint16_t> targets(plan->missing_data.begin(), plan->missing_data.end());
  targets.insert(targets.end(), plan->missing_parity.begin(), plan->missing_parity.end());
  RSB_CU(cudaSetDevice(g.device));
  // FFT-route decode where its estimated work is lower than the matrix route's.
  if (!targets.empty()) {
    auto dec = std::make_shared<Fft16Decode>();
    std::vector<uint32_t> t32(targets.begin(), targets.end());
    if (route != 1 && fft16_decode_build(g.k, g.m, plan->survivors, t32, *dec) &&
        (route == 2 || fft16_decode_preferred(*dec, g.k))) {
      const size_t cbytes = dec->cols.size() * 2, toff = (cbytes + 15) & ~size_t(15);
      void *d = nullptr;
      RSB_CU(cudaMalloc(&d, toff + t32.size() * 4));
      plan->d_rows = d;
      RSB_CU(cudaMemcpy(d, dec->cols.data(), cbytes, cudaMemcpyHostToDevice));
      RSB_CU(cudaMemcpy(static_cast<uint8_t *>(d) + toff, t32.data(), t32.size() * 4, cudaMemcpyHostToDevice));
      plan->fft16 = dec;
      plan->fft16_targets_off = toff;
      out = cache.insert(pres, plan);
      return RS_OK;
    }
  }
  uint32_t *d = nullptr;
  int st = lagrange16_device(nodes, targets, &d);
  plan->d_rows = d;
  if (st) return st;
  out = cache.insert(pres, plan);
  return RS_OK;
}

// Runs out = rows x in over device rows; `in_ptrs`/`out_ptrs` are host arrays of
// device pointers, copied into a stream-ordered device table.
static int apply16_ptrs(const uint32_t *coeffs, uint32_t k, uint32_t rows, const uint8_t *const *in_ptrs,
                        uint8_t *const *out_ptrs, size_t len, bool verify, uint32_t *mismatch,
                        cudaStream_t st) {
  std::vector<const uint8_t *> table(k + rows);
  for (uint32_t i = 0; i < k; i++) table[i] = in_ptrs[i];
  for (uint32_t j = 0; j < rows; j++) table[k + j] = out_ptrs[j];
  void *d_table = nullptr;
  RSB_CU(scratch_alloc(&d_table, table.size() * sizeof(void *), st));
  RSB_CU(cudaMemcpyAsync(d_table, table.data(), table.size() * sizeof(void *), cudaMemcpyHostToDevice, st));
  Apply16Args a{};
  a.in_ptrs = reinterpret_cast<const uint8_t *const *>(d_table);
  a.out_ptrs = reinterpret_cast<uint8_t *const *>(static_cast<char *>(d_table) + k * sizeof(void *));
  a.coeffs = coeffs;
  a.k = k;
  a.rows = rows;
  a.n_sym = len / 2;
  a.n_stripes = 1;
  a.mismatch = mismatch;
  int st_ = launch_gf16(a, verify, st);
  scratch_free(d_table, st);
  return st_;
}

// Rebuilds the first `rows` targets of an FFT-route plan (missing data first, then
// missing parity). Device shards go through a stream-ordered pointer table; host shards
// are staged: survivors copied in, rebuilt rows copied back.
static int fft16_reconstruct(const Gen16 &g, const Plan &plan, Exec &ex, uint8_t *const *shards, size_t len,
                             size_t rows, bool dev, cudaStream_t st) {
  const Fft16Decode &d = *plan.fft16;
  const size_t n = g.k + g.m;
  const uint16_t *d_cols = static_cast<const uint16_t *>(plan.d_rows);
  const uint32_t *d_targets =
      reinterpret_cast<const uint32_t *>(static_cast<const uint8_t *>(plan.d_rows) + plan.fft16_targets_off);
  const size_t sbytes = fft16_decode_scratch_bytes(d, len, kFft16ScratchBudget);
  RSB_CU(cudaSetDevice(g.device));
  if (dev) {
    uint8_t *mem = nullptr;
    const size_t tbytes = (n * sizeof(void *) + 255) & ~size_t(255);
    RSB_CU(scratch_alloc(reinterpret_cast<void **>(&mem), tbytes + sbytes, st));
    int rc = RS_OK;
    if (cudaMemcpyAsync(mem, shards, n * sizeof(void *), cudaMemcpyHostToDevice, st) != cudaSuccess) rc = RS_ERR_CUDA;
    if (rc == RS_OK)
      rc = fft16_decode_run(d, d_cols, mem + tbytes, sbytes, reinterpret_cast<uint8_t *const *>(mem), d_targets,
                            rows, len, st);
    scratch_free(mem, st);
    return rc;
  }
  std::lock_guard<std::mutex> lock(ex.mu);
  const size_t tbytes = (n * sizeof(void *) + 255) & ~size_t(255);
  RSB_TRY(ex.buf.ensure(n * len));
  RSB_TRY(ex.aux.ensure(tbytes + sbytes));
  std::vector<uint8_t *> ptrs(n);
  for (size_t i = 0; i < n; i++) ptrs[i] = ex.buf.ptr + i * len;
  // Staged (as rs16_encode): the present rows gathered into pinned memory in their slots
  // of the n-row layout, which crosses the link in one copy each way.
  const bool staged = host_staged(n * len);
  if (staged) {
    RSB_TRY(ex.io.ensure(n * len));
    uint8_t *h = ex.io.ptr;
    const std::vector<uint32_t> &sv = plan.survivors;
    gather_rows(h, len, sv.size(), len, [&](size_t i) { return shards[sv[i]]; });
    // gather_rows packed them; move each to its slot, last first (a slot index is at
    // least its survivor position, so no row is overwritten before it moves).
    for (size_t i = sv.size(); i-- > 0;)
      if (sv[i] != i) memmove(h + (size_t)sv[i] * len, h + i * len, len);
    RSB_CU(cudaMemcpyAsync(ex.buf.ptr, h, n * len, cudaMemcpyHostToDevice, ex.stream));
  } else {
    for (uint32_t s : plan.survivors)
      RSB_CU(cudaMemcpyAsync(ptrs[s], shards[s], len, cudaMemcpyHostToDevice, ex.stream));
  }
  RSB_CU(cudaMemcpyAsync(ex.aux.ptr, ptrs.data(), n * sizeof(void *), cudaMemcpyHostToDevice, ex.stream));
  RSB_TRY(fft16_decode_run(d, d_cols, ex.aux.ptr + tbytes, sbytes, reinterpret_cast<uint8_t *const *>(ex.aux.ptr),
                           d_targets, rows, len, ex.stream));
  if (staged) {
    RSB_CU(cudaMemcpyAsync(ex.io.ptr, ex.buf.ptr, n * len, cudaMemcpyDeviceToHost, ex.stream));
    RSB_CU(cudaStreamSynchronize(ex.stream));
    const uint8_t *h = ex.io.ptr;
    for (size_t j = 0; j < rows; j++) memcpy(shards[d.targets[j]], h + (size_t)d.targets[j] * len, len);
    return RS_OK;
  }
  for (size_t j = 0; j < rows; j++)
    RSB_CU(cudaMemcpyAsync(shards[d.targets[j]], ptrs[d.targets[j]], len, cudaMemcpyDeviceToHost, ex.stream));
  RSB_CU(cudaStreamSynchronize(ex.stream));
  return RS_OK;
}

static int reconstruct16(const Gen16 &g, PlanCache *cache, const Plan *fixed, Exec &ex, int route,
                         uint8_t *const *shards, const size_t *lens, const uint8_t *present,
                         size_t n_shards, bool data_only, bool dev, cudaStream_t st, rs8_t *sub = nullptr,
                         rs8_dec_t *sub_dec = nullptr) {
  size_t n = g.k + g.m;
  if (!shards || !lens || !present) return RS_ERR_INVALID_ARGUMENT;
  if (n_shards != n) return n_shards < n ? RS_TOO_FEW_SHARDS : RS_TOO_MANY_SHARDS;
  Presence pres;
  size_t n_present = 0, len = 0;
  RSB_TRY(scan_shards(lens, present, n, true, pres, n_present, len));
  if (fixed && pres != fixed->presence) return RS_INVALID_SHARD_FLAGS;
  if (n_present == n) return RS_OK;
  if (!fixed && n_present < g.k) return RS_TOO_FEW_SHARDS_PRESENT;
  if (len == 0) return RS_TOO_FEW_SHARDS_PRESENT;
  if (sub && !fixed) {  // the tower's checks passed; the subfield codec rebuilds
    RSB_TRY(check_absent_buffers(lens, present, n, g.k, len, data_only));
    return dev ? rs8_reconstruct_dev(sub, shards, lens, present, n, data_only ? 1 : 0, st)
               : rs8_reconstruct(sub, shards, lens, present, n, data_only ? 1 : 0);
  }
  if (sub_dec && fixed && !dev) {  // a prepared decoder on the subfield codec
    RSB_TRY(check_absent_buffers(lens, present, n, g.k, len, data_only));
    return rs8_dec_reconstruct(sub_dec, shards, lens, present, n, data_only ? 1 : 0);
  }
  std::shared_ptr<const Plan> hold;
  const Plan *plan = fixed;
  if (!plan) {
    RSB_TRY(plan16_for(g, *cache, pres, hold, route));
    plan = hold.get();
  }
  RSB_TRY(check_absent_buffers(lens, present, n, g.k, len, data_only));
  size_t rows = plan->missing_data.size() + (data_only ? 0 : plan->missing_parity.size());
  if (rows == 0) return RS_OK;
  std::vector<uint32_t> outs(plan->missing_data);
  if (!data_only) outs.insert(outs.end(), plan->missing_parity.begin(), plan->missing_parity.end());
  if (plan->fft16) return fft16_reconstruct(g, *plan, ex, shards, len, rows, dev, st);
  const uint32_t *coeffs = reinterpret_cast<const uint32_t *>(plan->d_rows);
  if (dev) {
    RSB_CU(cudaSetDevice(g.device));
    std::vector<const uint8_t *> ins(g.k);
    std::vector<uint8_t *> os(rows);
    for (size_t t = 0; t < g.k; t++) ins[t] = shards[plan->survivors[t]];
    for (size_t j = 0; j < rows; j++) os[j] = shards[outs[j]];
    return apply16_ptrs(coeffs, (uint32_t)g.k, (uint32_t)rows, ins.data(), os.data(), len, false, nullptr, st);
  }
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  RSB_TRY(ex.buf.ensure((g.k + rows) * len));
  const bool staged = host_staged((g.k + rows) * len);  // as rs16_encode
  if (staged) {
    RSB_TRY(ex.io.ensure((g.k + rows) * len));
    gather_rows(ex.io.ptr, len, g.k, len, [&](size_t t) { return shards[plan->survivors[t]]; });
    RSB_CU(cudaMemcpyAsync(ex.buf.ptr, ex.io.ptr, g.k * len, cudaMemcpyHostToDevice, ex.stream));
  } else {
    for (size_t t = 0; t < g.k; t++)
      RSB_CU(cudaMemcpyAsync(ex.buf.ptr + t * len, shards[plan->survivors[t]], len, cudaMemcpyHostToDevice,
                             ex.stream));
  }
  Apply16Args a{};
  a.in_base = ex.buf.ptr;
  a.in_row_stride = len;
  a.out_base = ex.buf.ptr + g.k * len;
  a.out_row_stride = len;
  a.coeffs = coeffs;
  a.k = (uint32_t)g.k;
  a.rows = (uint32_t)rows;
  a.n_sym = len / 2;
  a.n_stripes = 1;
  RSB_TRY(launch_gf16(a, false, ex.stream));
  if (staged) {
    RSB_CU(cudaMemcpyAsync(ex.io.ptr + g.k * len, ex.buf.ptr + g.k * len, rows * len, cudaMemcpyDeviceToHost,
                           ex.stream));
    RSB_CU(cudaStreamSynchronize(ex.stream));
    scatter_rows(ex.io.ptr + g.k * len, len, rows, len, [&](size_t j) { return shards[outs[j]]; });
    return RS_OK;
  }
  for (size_t j = 0; j < rows; j++)
    RSB_CU(cudaMemcpyAsync(shards[outs[j]], ex.buf.ptr + (g.k + j) * len, len, cudaMemcpyDeviceToHost,
                           ex.stream));
  RSB_CU(cudaStreamSynchronize(ex.stream));
  return RS_OK;
}

}  // namespace rsb

extern "C" {

int rs16_new(size_t k, size_t m, rs16_t **out) {
  if (!out) return RS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (k == 0) return RS_TOO_FEW_DATA_SHARDS;
  if (m == 0) return RS_TOO_FEW_PARITY_SHARDS;
  if (k + m > 65536) return RS_TOO_MANY_SHARDS;
  int dev = 0;
  RSB_TRY(ensure_device(&dev));
  auto gen = std::make_shared<Gen16>();
  gen->device = dev;
  gen->k = k;
  gen->m = m;
  std::vector<uint16_t> nodes(k), targets(m);
  for (size_t i = 0; i < k; i++) nodes[i] = (uint16_t)i;
  for (size_t j = 0; j < m; j++) targets[j] = (uint16_t)(k + j);
  uint32_t *d = nullptr;
  int st0 = lagrange16_device(nodes, targets, &d);
  gen->d_split = d;
  if (st0) return st0;
  RSB_TRY(build_fft16(*gen));
  auto c = new (std::nothrow) rs16_codec();
  if (!c) return RS_ERR_ALLOC;
  c->gen = gen;
  c->plans = std::make_shared<PlanCache>();
  int st = make_exec(dev, c->exec);
  if (st == RS_OK && k + m <= 256) st = rs8_new(k, m, &c->sub);
  if (st) {
    delete c;
    return st;
  }
  *out = c;
  return RS_OK;
}

int rs16_clone(const rs16_t *codec, rs16_t **out) {
  if (!codec || !out) return RS_ERR_INVALID_ARGUMENT;
  auto c = new (std::nothrow) rs16_codec();
  if (!c) return RS_ERR_ALLOC;
  c->gen = codec->gen;
  c->plans = std::make_shared<PlanCache>();
  c->plans->copy_from(*codec->plans);
  c->route.store(codec->route.load());
  int st = make_exec(codec->gen->device, c->exec);
  if (st == RS_OK && codec->sub) st = rs8_clone(codec->sub, &c->sub);
  if (st) {
    delete c;
    return st;
  }
  *out = c;
  return RS_OK;
}

void rs16_free(rs16_t *codec) { delete codec; }
size_t rs16_data_shard_count(const rs16_t *c) { return c ? c->gen->k : 0; }
size_t rs16_parity_shard_count(const rs16_t *c) { return c ? c->gen->m : 0; }
size_t rs16_total_shard_count(const rs16_t *c) { return c ? c->gen->k + c->gen->m : 0; }
int rs16_equal(const rs16_t *a, const rs16_t *b) {
  if (!a || !b) return 0;
  return a->gen->k == b->gen->k && a->gen->m == b->gen->m;
}

// The generator rows as the device kernels apply them: read back the split constants
// and join them (c_lo = k0, c_hi = k1 ^ k0).
int rs16_parity_matrix(const rs16_t *c, uint16_t *out, size_t out_len) {
  if (!c || !out) return RS_ERR_INVALID_ARGUMENT;
  if (out_len != c->gen->k * c->gen->m) return RS_INCORRECT_SHARD_SIZE;
  std::vector<uint32_t> split(out_len);
  RSB_CU(cudaSetDevice(c->gen->device));
  RSB_CU(cudaMemcpy(split.data(), c->gen->d_split, out_len * 4, cudaMemcpyDeviceToHost));
  for (size_t t = 0; t < out_len; t++) {
    uint8_t lo = split[t] & 0xff, hi = (uint8_t)((split[t] >> 8) ^ lo);
    out[t] = (uint16_t)((hi << 8) | lo);
  }
  return RS_OK;
}

const char *rs16_encode_route(const rs16_t *c) {
  if (!c) return "invalid";
  if (subfield(c)) return "subfield";
  return use_fft16(c) ? "fft" : "matrix";
}

const char *rs16_encode_route_for(const rs16_t *c, size_t len, size_t n_stripes) {
  if (!c) return "invalid";
  if (subfield_encode(c, len, n_stripes)) return "subfield";
  return use_fft16(c, len, std::max<size_t>(n_stripes, 1)) ? "fft" : "matrix";
}

int rs16_set_route(rs16_t *c, int route) {
  if (!c || route < 0 || route > 2) return RS_ERR_INVALID_ARGUMENT;
  c->route.store(route);
  return RS_OK;
}

// src/reedsolomon16.rs:412-419
int rs16_encode(rs16_t *c, uint8_t *const *shards, size_t n_shards, size_t len) {
  if (!c || !shards) return RS_ERR_INVALID_ARGUMENT;
  const Gen16 &g = *c->gen;
  size_t n = g.k + g.m;
  if (n_shards != n) return n_shards < n ? RS_TOO_FEW_SHARDS : RS_TOO_MANY_SHARDS;
  RSB_TRY(check_len16(len));
  if (subfield_encode(c, len, 1)) return rs8_encode(c->sub, shards, n_shards, len);
  for (size_t i = 0; i < n; i++)
    if (!shards[i]) return RS_ERR_INVALID_ARGUMENT;
  Exec &ex = *c->exec;
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  RSB_TRY(ex.buf.ensure(n * len));
  // Up to kStagedCallBytes (host_staged) the data rows are gathered into pinned memory
  // and cross the link in one copy (a tower stripe can hold thousands of shards: one
  // pageable copy each costs microseconds apiece); the parity comes back the same way.
  const bool staged = host_staged(n * len);
  if (staged) {
    RSB_TRY(ex.io.ensure(n * len));
    gather_rows(ex.io.ptr, len, g.k, len, [&](size_t i) { return shards[i]; });
    RSB_CU(cudaMemcpyAsync(ex.buf.ptr, ex.io.ptr, g.k * len, cudaMemcpyHostToDevice, ex.stream));
  } else {
    for (size_t i = 0; i < g.k; i++)
      RSB_CU(cudaMemcpyAsync(ex.buf.ptr + i * len, shards[i], len, cudaMemcpyHostToDevice, ex.stream));
  }
  if (use_fft16(c, len)) {
    RSB_TRY(fft16_encode(g, ex.buf.ptr, len, 0, ex.buf.ptr + g.k * len, len, 0, 1, len, nullptr, ex.stream));
  } else {
    Apply16Args a{};
    a.in_base = ex.buf.ptr;
    a.in_row_stride = len;
    a.out_base = ex.buf.ptr + g.k * len;
    a.out_row_stride = len;
    a.coeffs = g.d_split;
    a.k = (uint32_t)g.k;
    a.rows = (uint32_t)g.m;
    a.n_sym = len / 2;
    a.n_stripes = 1;
    RSB_TRY(launch_gf16(a, false, ex.stream));
  }
  if (staged) {
    RSB_CU(cudaMemcpyAsync(ex.io.ptr + g.k * len, ex.buf.ptr + g.k * len, g.m * len, cudaMemcpyDeviceToHost,
                           ex.stream));
    RSB_CU(cudaStreamSynchronize(ex.stream));
    scatter_rows(ex.io.ptr + g.k * len, len, g.m, len, [&](size_t j) { return shards[g.k + j]; });
    return RS_OK;
  }
  for (size_t j = 0; j < g.m; j++)
    RSB_CU(cudaMemcpyAsync(shards[g.k + j], ex.buf.ptr + (g.k + j) * len, len, cudaMemcpyDeviceToHost,
                           ex.stream));
  RSB_CU(cudaStreamSynchronize(ex.stream));
  return RS_OK;
}

// src/reedsolomon16.rs:422-446
int rs16_encode_sep(rs16_t *c, const uint8_t *const *data, size_t n_data, uint8_t *const *parity,
                    size_t n_parity, size_t len) {
  if (!c || !data || !parity) return RS_ERR_INVALID_ARGUMENT;
  const Gen16 &g = *c->gen;
  if (n_data != g.k) return n_data < g.k ? RS_TOO_FEW_DATA_SHARDS : RS_TOO_MANY_DATA_SHARDS;
  if (n_parity != g.m) return n_parity < g.m ? RS_TOO_FEW_PARITY_SHARDS : RS_TOO_MANY_PARITY_SHARDS;
  RSB_TRY(check_len16(len));
  std::vector<uint8_t *> all(g.k + g.m);
  for (size_t i = 0; i < g.k; i++) all[i] = const_cast<uint8_t *>(data[i]);
  for (size_t j = 0; j < g.m; j++) all[g.k + j] = parity[j];
  return rs16_encode(c, all.data(), all.size(), len);
}

// src/reedsolomon16.rs:450-505
int rs16_verify(rs16_t *c, const uint8_t *const *shards, size_t n_shards, size_t len, int *ok) {
  if (!c || !shards || !ok) return RS_ERR_INVALID_ARGUMENT;
  const Gen16 &g = *c->gen;
  size_t n = g.k + g.m;
  if (n_shards != n) return n_shards < n ? RS_TOO_FEW_SHARDS : RS_TOO_MANY_SHARDS;
  RSB_TRY(check_len16(len));
  if (rs8_t *sub = subfield(c)) return rs8_verify(sub, shards, n_shards, len, ok);
  Exec &ex = *c->exec;
  std::lock_guard<std::mutex> lock(ex.mu);
  RSB_CU(cudaSetDevice(g.device));
  RSB_TRY(ex.buf.ensure(n * len));
  RSB_TRY(ex.aux.ensure(64));
  for (size_t i = 0; i < n; i++)
    if (!shards[i]) return RS_ERR_INVALID_ARGUMENT;
  if (host_staged(n * len)) {  // as rs16_encode: one copy of the gathered stripe
    RSB_TRY(ex.io.ensure(n * len));
    gather_rows(ex.io.ptr, len, n, len, [&](size_t i) { return shards[i]; });
    RSB_CU(cudaMemcpyAsync(ex.buf.ptr, ex.io.ptr, n * len, cudaMemcpyHostToDevice, ex.stream));
  } else {
    for (size_t i = 0; i < n; i++)
      RSB_CU(cudaMemcpyAsync(ex.buf.ptr + i * len, shards[i], len, cudaMemcpyHostToDevice, ex.stream));
  }
  uint32_t *flag = reinterpret_cast<uint32_t *>(ex.aux.ptr);
  RSB_CU(cudaMemsetAsync(flag, 0, 4, ex.stream));
  Apply16Args a{};
  a.in_base = ex.buf.ptr;
  a.in_row_stride = len;
  a.out_base = ex.buf.ptr + g.k * len;
  a.out_row_stride = len;
  a.coeffs = g.d_split;
  a.k = (uint32_t)g.k;
  a.rows = (uint32_t)g.m;
  a.n_sym = len / 2;
  a.n_stripes = 1;
  a.mismatch = flag;
  RSB_TRY(launch_gf16(a, true, ex.stream));
  uint32_t h = 0;
  RSB_CU(cudaMemcpyAsync(&h, flag, 4, cudaMemcpyDeviceToHost, ex.stream));
  RSB_CU(cudaStreamSynchronize(ex.stream));
  *ok = h ? 0 : 1;
  return RS_OK;
}

int rs16_reconstruct(rs16_t *c, uint8_t *const *shards, const size_t *lens, const uint8_t *present,
                     size_t n_shards, int data_only) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  return reconstruct16(*c->gen, c->plans.get(), nullptr, *c->exec, c->route.load(), shards, lens, present, n_shards,
                       data_only != 0, false, nullptr, subfield(c));
}

// src/reedsolomon16.rs:544-565
int rs16_reconstruct_rows(rs16_t *c, uint8_t *rows, size_t rows_len, size_t row_len,
                          const uint8_t *present, size_t n_present) {
  if (!c || !present) return RS_ERR_INVALID_ARGUMENT;
  size_t n = c->gen->k + c->gen->m;
  if (n_present != n) return RS_INVALID_SHARD_FLAGS;
  if (row_len == 0 || row_len % 2) return RS_INCORRECT_SHARD_SIZE;
  if (rows_len != n * row_len) return RS_INCORRECT_SHARD_SIZE;
  if (!rows) return RS_ERR_INVALID_ARGUMENT;
  std::vector<uint8_t *> shards(n);
  std::vector<size_t> lens(n, row_len);
  for (size_t i = 0; i < n; i++) shards[i] = rows + i * row_len;
  return rs16_reconstruct(c, shards.data(), lens.data(), present, n, 0);
}

// src/reedsolomon16.rs:518-541
int rs16_prepare_decode(rs16_t *c, const uint8_t *present, size_t n_present, rs16_dec_t **out) {
  if (!c || !out) return RS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const Gen16 &g = *c->gen;
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
  RSB_TRY(plan16_for(g, *c->plans, pres, plan, c->route.load()));
  std::shared_ptr<rs8_dec_t> sub_dec;
  if (rs8_t *sub = subfield(c)) {
    rs8_dec_t *d8 = nullptr;
    RSB_TRY(rs8_prepare_decode(sub, present, n, &d8));
    sub_dec.reset(d8, rs8_dec_free);
  }
  auto d = new (std::nothrow) rs16_decoder();
  if (!d) return RS_ERR_ALLOC;
  d->gen = c->gen;
  d->plan = plan;
  d->exec = c->exec;
  d->sub = sub_dec;
  *out = d;
  return RS_OK;
}

int rs16_dec_reconstruct(rs16_dec_t *d, uint8_t *const *shards, const size_t *lens, const uint8_t *present,
                         size_t n_shards, int data_only) {
  if (!d) return RS_ERR_INVALID_ARGUMENT;
  return reconstruct16(*d->gen, nullptr, d->plan.get(), *d->exec, 0, shards, lens, present, n_shards,
                       data_only != 0, false, nullptr, nullptr, d->sub.get());
}

int rs16_dec_clone(const rs16_dec_t *d, rs16_dec_t **out) {
  if (!d || !out) return RS_ERR_INVALID_ARGUMENT;
  auto c = new (std::nothrow) rs16_decoder(*d);
  if (!c) return RS_ERR_ALLOC;
  *out = c;
  return RS_OK;
}

void rs16_dec_free(rs16_dec_t *d) { delete d; }

int rs16_encode_dev(rs16_t *c, uint8_t *const *d_shards, size_t n_shards, size_t len, void *stream) {
  if (!c || !d_shards) return RS_ERR_INVALID_ARGUMENT;
  const Gen16 &g = *c->gen;
  size_t n = g.k + g.m;
  if (n_shards != n) return n_shards < n ? RS_TOO_FEW_SHARDS : RS_TOO_MANY_SHARDS;
  RSB_TRY(check_len16(len));
  if (subfield_encode(c, len, 1)) return rs8_encode_dev(c->sub, d_shards, n_shards, len, stream);
  RSB_CU(cudaSetDevice(g.device));
  cudaStream_t st = (cudaStream_t)stream;
  if (use_fft16(c, len)) {
    void *d_table = nullptr;
    RSB_CU(scratch_alloc(&d_table, n * sizeof(void *), st));
    RSB_CU(cudaMemcpyAsync(d_table, d_shards, n * sizeof(void *), cudaMemcpyHostToDevice, st));
    int rc = fft16_encode(g, nullptr, 0, 0, nullptr, 0, 0, 1, len, reinterpret_cast<uint8_t *const *>(d_table), st);
    scratch_free(d_table, st);
    return rc;
  }
  return apply16_ptrs(g.d_split, (uint32_t)g.k, (uint32_t)g.m, d_shards, d_shards + g.k, len, false, nullptr, st);
}

int rs16_encode_batch_dev(rs16_t *c, const uint8_t *d_data, size_t data_stride, uint8_t *d_parity,
                          size_t parity_stride, size_t n_stripes, size_t row_len, void *stream) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  if (n_stripes == 0) return RS_OK;
  RSB_TRY(check_len16(row_len));
  if (!d_data || !d_parity) return RS_ERR_INVALID_ARGUMENT;
  if (subfield_encode(c, row_len, n_stripes))
    return rs8_encode_batch_dev(c->sub, d_data, data_stride, d_parity, parity_stride, n_stripes, row_len, stream);
  const Gen16 &g = *c->gen;
  RSB_CU(cudaSetDevice(g.device));
  if (use_fft16(c, row_len, n_stripes))
    return fft16_encode(g, d_data, row_len, data_stride, d_parity, row_len, parity_stride, n_stripes, row_len,
                        nullptr, (cudaStream_t)stream);
  Apply16Args a{};
  a.in_base = d_data;
  a.in_row_stride = row_len;
  a.in_stripe_stride = data_stride;
  a.out_base = d_parity;
  a.out_row_stride = row_len;
  a.out_stripe_stride = parity_stride;
  a.coeffs = g.d_split;
  a.k = (uint32_t)g.k;
  a.rows = (uint32_t)g.m;
  a.n_sym = row_len / 2;
  a.n_stripes = (uint32_t)n_stripes;
  return launch_gf16(a, false, (cudaStream_t)stream);
}

int rs16_reconstruct_dev(rs16_t *c, uint8_t *const *d_shards, const size_t *lens, const uint8_t *present,
                         size_t n_shards, int data_only, void *stream) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  return reconstruct16(*c->gen, c->plans.get(), nullptr, *c->exec, c->route.load(), d_shards, lens, present, n_shards,
                       data_only != 0, true, (cudaStream_t)stream, subfield(c));
}

}  // extern "C"
