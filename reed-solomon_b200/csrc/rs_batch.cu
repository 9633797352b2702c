// Mixed batches of GF(2^8) stripes (include/rs_b200.h, rs_batch_*).
//
// One batch holds stripes of any shapes, lengths and erasure patterns. Creation
// validates each stripe the way its single-stripe call would, builds the decode rows
// of every reconstruct stripe on the device (one Gauss-Jordan launch per shape), and
// groups the work: (K,K) encodes with a bitsliced FFT kernel go to one ragged FFT
// launch per K; every other encode and every reconstruct goes to one ragged matrix
// launch. The launches are captured into a CUDA graph that rs_batch_launch replays.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <vector>

#include "codec8.hpp"
#include "kernels_batch.cuh"
#include "kernels_bits.cuh"
#include "kernels_fft.cuh"
#include "kernels_plan.cuh"
#include "runtime.hpp"
#include "tuning.hpp"

using namespace rsb;

struct rs_batch {
  int device = 0;
  int flags = 0;
  std::vector<std::shared_ptr<const Gen8>> gens;  // keeps generator tables alive
  DeviceBuf mem;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  struct FftLaunch {
    const FftShape *shape;
    const FftItem *items;
    uint32_t n;
    uint64_t groups;
    const uint32_t *masks;  // parity rows to store per item; null: every row
    bool unaligned;         // some item's rows are not 16-byte aligned
    int cfg_wide = -1, cfg_variant = -1;  // FFT launch configuration (-1: the shape's)
  };
  std::vector<FftLaunch> ffts;    // encodes
  std::vector<FftLaunch> regens;  // missing parity of reconstructs, after the data rows
  const RaggedItem *ragged = nullptr;
  uint32_t n_ragged = 0;
  uint64_t ragged_blocks[2] = {0, 0};
  uint32_t n_ragged0 = 0;  // items in the first launch (ragged_split)
  size_t ragged_smem = 0;
  size_t launches = 0, fft_items = 0, matrix_items = 0;
  uint64_t bytes = 0;
  ~rs_batch() {
    cudaSetDevice(device);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace rsb {

static int batch_enqueue(rs_batch *b, cudaStream_t st) {
  for (const auto &f : b->ffts)
    RSB_TRY(launch_fft8_items(*f.shape, f.items, f.n, f.groups, st, nullptr, f.unaligned, f.cfg_wide, f.cfg_variant));
  if (b->n_ragged) {
    RSB_CU(launch_ragged(b->ragged, b->n_ragged0, b->n_ragged, b->ragged_blocks, b->ragged_smem, st));
    g_launches += ragged_launches(b->ragged_blocks);
  }
  for (const auto &f : b->regens)
    RSB_TRY(launch_fft8_items(*f.shape, f.items, f.n, f.groups, st, f.masks, f.unaligned));
  return RS_OK;
}

// Host image of the device arrays, laid out in one allocation.
struct Arena {
  std::vector<uint8_t> host;
  size_t put(const void *p, size_t n) {
    size_t off = (host.size() + 255) & ~size_t(255);
    host.resize(off + n);
    if (n) memcpy(host.data() + off, p, n);
    return off;
  }
  size_t reserve(size_t n) {
    size_t off = (host.size() + 255) & ~size_t(255);
    host.resize(off + n);
    return off;
  }
};

// A compiled-kernel launch group: the shape and, for FFT shapes, a launch configuration.
struct FftKey {
  const FftShape *shape;
  int wide, variant;
  bool operator<(const FftKey &o) const {
    if (shape != o.shape) return shape < o.shape;
    if (wide != o.wide) return wide < o.wide;
    return variant < o.variant;
  }
};

static bool rows_aligned(const rs_batch_item &it) {
  return ((reinterpret_cast<uintptr_t>(it.d_rows) | it.row_stride) & 15u) == 0;
}

static int batch_create(const rs_batch_item *items, size_t n_items, int flags, const int *configs, int *statuses,
                        rs_batch_t **out);

}  // namespace rsb

extern "C" {

int rs_batch_create(const rs_batch_item *items, size_t n_items, int flags, int *statuses, rs_batch_t **out) {
  return batch_create(items, n_items, flags, nullptr, statuses, out);
}

int rs_batch_create_configured(const rs_batch_item *items, size_t n_items, int flags, const int *configs,
                               int *statuses, rs_batch_t **out) {
  return batch_create(items, n_items, flags, configs, statuses, out);
}

int rs_tuning_config_count(void) { return kTuneConfigCount; }

int rs_tuning_features(void) { return kTuneFeatures; }

int rs_tuning_config(int index, int *route, int *p0, int *p1) {
  if (index < 0 || index >= kTuneConfigCount) return RS_ERR_INVALID_ARGUMENT;
  if (route) *route = kTuneConfigs[index].route;
  if (p0) *p0 = kTuneConfigs[index].p0;
  if (p1) *p1 = kTuneConfigs[index].p1;
  return RS_OK;
}

int rs_batch_choose(const rs_batch_item *items, size_t n_items, rs_mlp_t *model, int *configs) {
  if (!model || !configs || (!items && n_items)) return RS_ERR_INVALID_ARGUMENT;
  int n_in = 0, n_out = 0;
  RSB_TRY(rs_mlp_dims(model, &n_in, nullptr, &n_out));
  if (n_in != kTuneFeatures || n_out != kTuneConfigCount) return RS_ERR_INVALID_ARGUMENT;
  // Encode items with a compiled kernel, grouped by shape and row alignment: each group
  // is one launch of the batch, so it takes one configuration.
  std::map<std::pair<const Gen8 *, bool>, std::vector<size_t>> groups;
  for (size_t i = 0; i < n_items; i++) {
    configs[i] = -1;
    const rs_batch_item &it = items[i];
    if (!it.codec || !it.d_rows || it.op != RS_BATCH_ENCODE || it.row_len == 0 || it.row_stride < it.row_len)
      continue;
    if (!it.codec->gen->fft || it.codec->route.load() != 0) continue;
    groups[{it.codec->gen.get(), rows_aligned(it)}].push_back(i);
  }
  std::vector<float> x;
  for (auto &kv : groups) {
    const Gen8 &g = *kv.first.first;
    for (size_t i : kv.second) {
      float f[kTuneFeatures];
      tune_features(g.k, g.m, items[i].row_len, 0, tune_batch(g.k, g.m, items[i].row_len, kv.second.size()),
                    kv.first.second, f);
      x.insert(x.end(), f, f + kTuneFeatures);
    }
  }
  const size_t rows = x.size() / kTuneFeatures;
  if (!rows) return RS_OK;
  std::vector<float> pred(rows * kTuneConfigCount);
  float *d = nullptr;
  RSB_CU(cudaMalloc(&d, (x.size() + pred.size()) * sizeof(float)));
  int st = RS_OK;
  if (cudaMemcpy(d, x.data(), x.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
    st = RS_ERR_CUDA;
  if (!st) st = rs_mlp_predict(model, d, (int)rows, d + x.size());
  if (!st && cudaMemcpy(pred.data(), d + x.size(), pred.size() * sizeof(float), cudaMemcpyDeviceToHost) !=
                 cudaSuccess)
    st = RS_ERR_CUDA;
  cudaFree(d);
  if (st) return st;
  // Per group: the applicable configuration with the least predicted total time (the
  // model predicts log time per stripe's launch). The batch's matrix launch has one tile
  // shape, so the matrix route is represented by configuration 0. The group keeps the
  // library's automatic choice unless the model predicts a clear gain over it
  // (kTrustGain): the model was fitted on uniform launches and a batch's launch groups
  // are ragged, where a small predicted gain is within its error (measured on the
  // 10,000-stripe mixed batch: unguarded choices lost 6-7% against the automatic ones,
  // which were within 0.3% of the exhaustive best there).
  constexpr double kTrustGain = 0.10;
  size_t row = 0;
  for (auto &kv : groups) {
    const FftShape &sh = *kv.first.first->fft;
    const int auto_cfg = fft_auto_config(sh, kv.first.second);
    double best = 0, at_auto = 0;
    int pick = -1;
    for (int c = 0; c < kTuneConfigCount; c++) {
      const TuneConfig &tc = kTuneConfigs[c];
      const bool ok = tc.route == kTuneMatrix ? tc.p0 == 0 : tc.route == kTuneFft ? !sh.gen : sh.gen;
      if (!ok) continue;
      double total = 0;
      for (size_t r = 0; r < kv.second.size(); r++) total += std::exp((double)pred[(row + r) * kTuneConfigCount + c]);
      if (c == auto_cfg) at_auto = total;
      if (pick < 0 || total < best) {
        best = total;
        pick = c;
      }
    }
    if (auto_cfg >= 0 && best > (1.0 - kTrustGain) * at_auto) pick = -1;
    for (size_t i : kv.second) configs[i] = pick;
    row += kv.second.size();
  }
  return RS_OK;
}

}  // extern "C"

namespace rsb {

static int batch_create(const rs_batch_item *items, size_t n_items, int flags, const int *configs, int *statuses,
                        rs_batch_t **out) {
  if (!out || (!items && n_items)) return RS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::unique_ptr<rs_batch> b(new (std::nothrow) rs_batch());
  if (!b) return RS_ERR_ALLOC;
  b->flags = flags;
  std::vector<int> status(n_items, RS_OK);
  int device = -1;

  struct Recon {
    size_t item;
    std::vector<uint32_t> surv, targets;
  };
  std::map<const Gen8 *, std::vector<Recon>> recon;  // per shape
  std::map<FftKey, std::vector<size_t>> fft_groups;  // compiled shape and configuration -> items
  struct Regen {
    size_t item;
    std::vector<uint32_t> parity;  // missing parity shard indexes
    bool only;                     // no data rows to rebuild first
  };
  std::map<const FftShape *, std::vector<Regen>> regen_groups;
  std::vector<size_t> matrix_encodes;

  for (size_t i = 0; i < n_items; i++) {
    const rs_batch_item &it = items[i];
    if (!it.codec || !it.d_rows || it.op < 0 || it.op > 2) {
      status[i] = RS_ERR_INVALID_ARGUMENT;
      continue;
    }
    const Gen8 &g = *it.codec->gen;
    if (device < 0) device = g.device;
    if (g.device != device) {
      status[i] = RS_ERR_INVALID_ARGUMENT;
      continue;
    }
    if (it.row_len == 0) {
      status[i] = RS_EMPTY_SHARD;
      continue;
    }
    if (it.row_stride < it.row_len) {
      status[i] = RS_INCORRECT_SHARD_SIZE;
      continue;
    }
    const size_t n = g.k + g.m;
    if (it.op == RS_BATCH_ENCODE) {
      const int cfg = configs ? configs[i] : -1;
      if (cfg < -1 || cfg >= kTuneConfigCount) {
        status[i] = RS_ERR_INVALID_ARGUMENT;
        continue;
      }
      if (cfg >= 0 && !(flags & RS_BATCH_MATRIX_ONLY)) {
        // An explicit configuration: the matrix route, or the shape's compiled kernel
        // with this launch configuration (an error where the shape has no such kernel).
        const TuneConfig &tc = kTuneConfigs[cfg];
        if (tc.route == kTuneMatrix) {
          matrix_encodes.push_back(i);
        } else if (g.fft && (tc.route == kTuneGen) == g.fft->gen) {
          fft_groups[{g.fft, tc.route == kTuneFft ? tc.p0 : -1, tc.route == kTuneFft ? tc.p1 : -1}].push_back(i);
        } else {
          status[i] = RS_ERR_INVALID_ARGUMENT;
          continue;
        }
        b->bytes += n * it.row_len;
        continue;
      }
      b->bytes += n * it.row_len;
      if (!(flags & RS_BATCH_MATRIX_ONLY) && use_fft8(it.codec, it.row_len))
        fft_groups[{g.fft, -1, -1}].push_back(i);
      else
        matrix_encodes.push_back(i);
      continue;
    }
    if (!it.present) {
      status[i] = RS_ERR_INVALID_ARGUMENT;
      continue;
    }
    Presence pres(n);
    size_t cnt = 0;
    for (size_t r = 0; r < n; r++)
      if (it.present[r]) {
        pres.set(r);
        cnt++;
      }
    if (cnt == n) continue;  // nothing to rebuild
    if (cnt < g.k) {
      status[i] = RS_TOO_FEW_SHARDS_PRESENT;
      continue;
    }
    Recon rc;
    rc.item = i;
    std::vector<uint32_t> md, mp;
    split_pattern(pres, g.k, n, rc.surv, md, mp);
    const size_t rebuilt = md.size() + (it.op == RS_BATCH_RECONSTRUCT ? mp.size() : 0);
    if (rebuilt == 0) continue;
    b->bytes += (g.k + rebuilt) * it.row_len;
    // Missing parity of a shape with a compiled encode kernel is regenerated by that
    // kernel after the data rows are whole, storing only the missing rows, where that
    // beats the matrix route (regen_parity_pays).
    const bool regen = it.op == RS_BATCH_RECONSTRUCT && !(flags & RS_BATCH_MATRIX_ONLY) &&
                       use_fft8(it.codec, it.row_len) && regen_parity_pays(g, mp.size(), it.codec->route.load());
    rc.targets = md;
    if (it.op == RS_BATCH_RECONSTRUCT && !regen) rc.targets.insert(rc.targets.end(), mp.begin(), mp.end());
    if (regen) regen_groups[g.fft].push_back({i, mp, md.empty()});
    if (rc.targets.empty()) continue;
    recon[&g].push_back(std::move(rc));
  }
  if (statuses)
    for (size_t i = 0; i < n_items; i++) statuses[i] = status[i];
  if (device < 0) {
    *out = b.release();
    return RS_OK;
  }
  b->device = device;
  RSB_CU(cudaSetDevice(device));
  RSB_CU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  for (size_t i = 0; i < n_items; i++)
    if (status[i] == RS_OK && items[i].codec) b->gens.push_back(items[i].codec->gen);

  // ---- plan inputs, in one arena ----
  Arena ar;
  struct PlanGroup {
    const Gen8 *g;
    size_t surv_off, targ_off, nt_off, rows_off, stat_off, count;
  };
  std::vector<PlanGroup> pgs;
  for (auto &kv : recon) {
    const Gen8 &g = *kv.first;
    auto &list = kv.second;
    std::vector<uint16_t> surv(list.size() * g.k), targ(list.size() * g.m, 0), nt(list.size());
    for (size_t p = 0; p < list.size(); p++) {
      for (size_t t = 0; t < g.k; t++) surv[p * g.k + t] = (uint16_t)list[p].surv[t];
      for (size_t t = 0; t < list[p].targets.size(); t++) targ[p * g.m + t] = (uint16_t)list[p].targets[t];
      nt[p] = (uint16_t)list[p].targets.size();
    }
    PlanGroup pg;
    pg.g = &g;
    pg.count = list.size();
    pg.surv_off = ar.put(surv.data(), surv.size() * 2);
    pg.targ_off = ar.put(targ.data(), targ.size() * 2);
    pg.nt_off = ar.put(nt.data(), nt.size() * 2);
    pg.rows_off = ar.reserve(list.size() * g.m * g.k);
    pg.stat_off = ar.reserve(list.size() * sizeof(int));
    pgs.push_back(pg);
  }
  // ---- ragged matrix items (device pointers patched in after allocation) ----
  std::vector<RaggedItem> ragged;
  uint32_t max_k = 1;
  for (size_t i : matrix_encodes) {
    const Gen8 &g = *items[i].codec->gen;
    RaggedItem r{};
    r.base = items[i].d_rows;
    r.row_stride = items[i].row_stride;
    r.len = items[i].row_len;
    r.coeffs = g.d_rows;
    r.k = (uint32_t)g.k;
    r.rows = (uint32_t)g.m;
    ragged.push_back(r);
    max_k = std::max<uint32_t>(max_k, (uint32_t)g.k);
  }
  struct Patch {
    size_t ragged_index, rows_off, surv_off, targ_off;
  };
  std::vector<Patch> patches;
  for (auto &pg : pgs) {
    const Gen8 &g = *pg.g;
    auto &list = recon[pg.g];
    for (size_t p = 0; p < list.size(); p++) {
      const rs_batch_item &it = items[list[p].item];
      RaggedItem r{};
      r.base = it.d_rows;
      r.row_stride = it.row_stride;
      r.len = it.row_len;
      r.k = (uint32_t)g.k;
      r.rows = (uint32_t)list[p].targets.size();
      patches.push_back({ragged.size(), pg.rows_off + p * g.m * g.k, pg.surv_off + p * g.k * 2,
                         pg.targ_off + p * g.m * 2});
      ragged.push_back(r);
      max_k = std::max<uint32_t>(max_k, (uint32_t)g.k);
    }
  }
  uint64_t blocks = 0;
  for (auto &r : ragged) {
    r.col_tiles = (uint32_t)((r.len + kTileBytes - 1) / kTileBytes);
    uint32_t chunks = (r.rows + kRowChunk - 1) / kRowChunk;
    r.block_begin = (uint32_t)blocks;
    blocks += (uint64_t)r.col_tiles * chunks;
  }
  if (blocks >= (1ull << 31)) return RS_ERR_INVALID_ARGUMENT;
  b->matrix_items = ragged.size();
  size_t ragged_off = ar.reserve(std::max<size_t>(ragged.size(), 1) * sizeof(RaggedItem));
  // ---- FFT items ----
  struct FftGroupOff {
    const FftShape *shape;
    size_t off, n;
    uint64_t groups;
    bool unaligned;
    int wide, variant;
  };
  std::vector<FftGroupOff> fgo;
  std::vector<std::vector<FftItem>> fft_host;
  for (auto &kv : fft_groups) {
    std::vector<FftItem> v;
    uint64_t g0 = 0;
    uintptr_t align = 0;
    for (size_t i : kv.second) {
      const rs_batch_item &it = items[i];
      align |= reinterpret_cast<uintptr_t>(it.d_rows) | it.row_stride;
      FftItem f{};
      f.in_base = it.d_rows;
      f.out_base = it.d_rows + (size_t)kv.first.shape->k * it.row_stride;
      f.row_stride = it.row_stride;
      f.len = it.row_len;
      f.group_begin = g0;
      g0 += (it.row_len + 31) / 32;
      v.push_back(f);
    }
    fgo.push_back({kv.first.shape, ar.put(v.data(), v.size() * sizeof(FftItem)), v.size(), g0, (align & 15) != 0,
                   kv.first.wide, kv.first.variant});
    b->fft_items += v.size();
    fft_host.push_back(std::move(v));
  }
  struct RegenOff {
    const FftShape *shape;
    size_t off, mask_off, n;
    uint64_t groups;
    bool unaligned;
  };
  std::vector<RegenOff> rgo;
  for (auto &kv : regen_groups) {
    std::vector<FftItem> v;
    std::vector<uint32_t> masks(4 * kv.second.size(), 0u);
    uint64_t g0 = 0;
    uintptr_t align = 0;
    for (size_t p = 0; p < kv.second.size(); p++) {
      const Regen &rg = kv.second[p];
      const rs_batch_item &it = items[rg.item];
      align |= reinterpret_cast<uintptr_t>(it.d_rows) | it.row_stride;
      FftItem f{};
      f.in_base = it.d_rows;
      f.out_base = it.d_rows + (size_t)kv.first->k * it.row_stride;
      f.row_stride = it.row_stride;
      f.len = it.row_len;
      f.group_begin = g0;
      g0 += (it.row_len + 31) / 32;
      v.push_back(f);
      for (uint32_t x : rg.parity) masks[4 * p + (x - kv.first->k) / 32] |= 1u << ((x - kv.first->k) % 32);
      if (rg.only) b->fft_items++;
    }
    size_t off = ar.put(v.data(), v.size() * sizeof(FftItem));
    rgo.push_back({kv.first, off, ar.put(masks.data(), masks.size() * sizeof(uint32_t)), v.size(), g0,
                   (align & 15) != 0});
  }

  // ---- allocate, patch device pointers, upload ----
  RSB_TRY(b->mem.ensure(std::max<size_t>(ar.host.size(), 256)));
  uint8_t *base = b->mem.ptr;
  for (const Patch &pt : patches) {
    RaggedItem &r = ragged[pt.ragged_index];
    r.coeffs = base + pt.rows_off;
    r.in_rows = reinterpret_cast<const uint16_t *>(base + pt.surv_off);
    r.out_rows = reinterpret_cast<const uint16_t *>(base + pt.targ_off);
  }
  uint64_t ragged_blocks[2];
  const uint32_t n_ragged0 = ragged_split(ragged, ragged_blocks);
  if (!ragged.empty()) memcpy(ar.host.data() + ragged_off, ragged.data(), ragged.size() * sizeof(RaggedItem));
  RSB_CU(cudaMemcpyAsync(base, ar.host.data(), ar.host.size(), cudaMemcpyHostToDevice, b->stream));

  // ---- decode rows for every reconstruct stripe: one Gauss-Jordan launch per shape ----
  for (auto &pg : pgs) {
    const Gen8 &g = *pg.g;
    PlanArgs pa{};
    pa.gen = g.d_rows;
    pa.k = (uint32_t)g.k;
    pa.m = (uint32_t)g.m;
    pa.survivors = reinterpret_cast<const uint16_t *>(base + pg.surv_off);
    pa.targets = reinterpret_cast<const uint16_t *>(base + pg.targ_off);
    pa.n_targets = reinterpret_cast<const uint16_t *>(base + pg.nt_off);
    pa.max_rows = (uint32_t)g.m;
    pa.out = base + pg.rows_off;
    pa.status = reinterpret_cast<int *>(base + pg.stat_off);
    size_t smem = plan_smem((uint32_t)g.k).total;
    if (smem > 48 * 1024)
      RSB_CU(cudaFuncSetAttribute(gf8_plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    gf8_plan_kernel<<<(unsigned)pg.count, 256, smem, b->stream>>>(pa);
    g_launches++;
    RSB_CU(cudaGetLastError());
  }
  for (auto &pg : pgs) {
    std::vector<int> st(pg.count);
    RSB_CU(cudaMemcpyAsync(st.data(), base + pg.stat_off, pg.count * sizeof(int), cudaMemcpyDeviceToHost,
                           b->stream));
    RSB_CU(cudaStreamSynchronize(b->stream));
    auto &list = recon[pg.g];
    for (size_t p = 0; p < pg.count; p++)
      if (st[p] && statuses) statuses[list[p].item] = RS_SINGULAR_MATRIX;
  }
  RSB_CU(cudaStreamSynchronize(b->stream));

  for (auto &f : fgo)
    b->ffts.push_back({f.shape, reinterpret_cast<const FftItem *>(base + f.off), (uint32_t)f.n, f.groups, nullptr,
                       f.unaligned, f.wide, f.variant});
  for (auto &f : rgo)
    b->regens.push_back({f.shape, reinterpret_cast<const FftItem *>(base + f.off), (uint32_t)f.n, f.groups,
                         reinterpret_cast<const uint32_t *>(base + f.mask_off), f.unaligned});
  b->ragged = reinterpret_cast<const RaggedItem *>(base + ragged_off);
  b->n_ragged = (uint32_t)ragged.size();
  b->ragged_blocks[0] = ragged_blocks[0];
  b->ragged_blocks[1] = ragged_blocks[1];
  b->n_ragged0 = n_ragged0;
  b->ragged_smem = 8192 + (size_t)kRowChunk * max_k;
  if (b->ragged_smem > 48 * 1024)
    RSB_CU(cudaFuncSetAttribute(gf8_ragged_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)b->ragged_smem));
  b->launches = b->ffts.size() + b->regens.size() + (b->n_ragged ? ragged_launches(b->ragged_blocks) : 0);

  if (!(flags & RS_BATCH_NO_GRAPH) && b->launches) {
    uint64_t before = g_launches.load();
    // Kernel attributes are set by a first, uncaptured enqueue; the graph then holds
    // only the launches.
    RSB_TRY(batch_enqueue(b.get(), b->stream));
    RSB_CU(cudaStreamSynchronize(b->stream));
    RSB_CU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int st = batch_enqueue(b.get(), b->stream);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    g_launches.store(before);
    if (st) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (e != cudaSuccess) {
      set_cuda_error(e, "cudaStreamEndCapture");
      return RS_ERR_CUDA;
    }
    b->graph = graph;
    RSB_CU(cudaGraphInstantiate(&b->exec, graph, 0));
  }
  *out = b.release();
  return RS_OK;
}

}  // namespace rsb

extern "C" {

int rs_batch_launch(rs_batch_t *b, void *stream) {
  if (!b) return RS_ERR_INVALID_ARGUMENT;
  if (!b->launches) return RS_OK;
  RSB_CU(cudaSetDevice(b->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (b->exec) {
    RSB_CU(cudaGraphLaunch(b->exec, st));
    g_launches += b->launches;
    return RS_OK;
  }
  return batch_enqueue(b, st);
}

int rs_batch_stats(const rs_batch_t *b, size_t *launches, size_t *fft_items, size_t *matrix_items, uint64_t *bytes) {
  if (!b) return RS_ERR_INVALID_ARGUMENT;
  if (launches) *launches = b->launches;
  if (fft_items) *fft_items = b->fft_items;
  if (matrix_items) *matrix_items = b->matrix_items;
  if (bytes) *bytes = b->bytes;
  return RS_OK;
}

void rs_batch_free(rs_batch_t *b) { delete b; }

}  // extern "C"
