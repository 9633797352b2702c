// Request server: continuous batching of encode and reconstruct requests on one GPU
// (include/rs_b200.h, rs_server_*).
//
// A scheduler thread owns the device. Requests wait in a FIFO queue and are admitted
// while a slot is free and their working set fits in the server's device arena:
// staged payload (host-memory requests), descriptors and decode plans, and the
// generator table of their shape unless it is already resident. Resident tables stay
// in the arena across requests and are evicted, least recently used first, only when
// idle and the space is needed. Admission happens continuously: every completion
// frees memory and a slot, and the scheduler admits more work at once while earlier
// work is still running on the device.
//
// Every GF(2^8) request admitted in one scheduling round forms one launch group: (K,K)
// encodes that take the bitsliced FFT go to one ragged FFT launch per K, every other
// encode and every reconstruct to one ragged matrix launch (decode rows from one
// Gauss-Jordan launch per request). A GF(2^16) request is its own group. Groups are
// spread over several streams so their work overlaps on the device; each group ends
// with a host callback that stamps its completion time.
//
// The arithmetic is the same kernels as the single-stripe entry points, so a request
// gives the same bytes alone or in a mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "codec8.hpp"
#include "fft16.hpp"
#include "gf_host.hpp"
#include "kernels_batch.cuh"
#include "kernels_bits.cuh"
#include "kernels_fft.cuh"
#include "kernels_lagrange.cuh"
#include "kernels_matrix.cuh"
#include "kernels_plan.cuh"
#include "runtime.hpp"
#include "tuning.hpp"

namespace rsb {

static uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

static size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// First-fit allocator over [0, cap) in 256-byte granules; host-side bookkeeping only.
struct SpanAllocator {
  size_t cap = 0, used = 0, peak = 0;
  std::map<size_t, size_t> free_;  // offset -> bytes
  void reset(size_t c) {
    cap = c;
    used = peak = 0;
    free_.clear();
    if (c) free_[0] = c;
  }
  bool alloc(size_t bytes, size_t &off) {
    bytes = up256(std::max<size_t>(bytes, 1));
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      off = it->first;
      size_t rest = it->second - bytes;
      free_.erase(it);
      if (rest) free_[off + bytes] = rest;
      used += bytes;
      peak = std::max(peak, used);
      return true;
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = up256(std::max<size_t>(bytes, 1));
    used -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct Span {
  size_t off = 0, bytes = 0;
  bool live = false;
};

// A resident generator table: m x k u8 (GF(2^8)) or m x k split u32 (tower).
struct Table {
  uint64_t key = 0;
  int field = 8;
  size_t k = 0, m = 0;
  Span span;
  int refs = 0;
  uint64_t last_use = 0;
  cudaEvent_t ready = nullptr;
  bool stale = false;  // its build failed: never reused, dropped once idle
  // GF(2^16) encode on the FFT route: the program; the span then holds its constants.
  std::shared_ptr<const Fft16Program> fft16;
};

static uint64_t table_key(int field, size_t k, size_t m) {
  return ((uint64_t)field << 40) | ((uint64_t)k << 20) | (uint64_t)m;
}

static size_t table_bytes(int field, size_t k, size_t m) { return field == 8 ? k * m : k * m * 4; }

static size_t fft16_table_bytes(const Fft16Program &p) { return p.cols.size() * 2; }

struct Req {
  rs_request r{};
  std::vector<uint8_t> present;
  std::vector<uint32_t> surv, targets;  // reconstruct: first k present; rebuilt rows
  uint64_t submit_ns = 0, admit_ns = 0, bytes = 0;
  int status = RS_OK;
  bool fft = false;  // GF(2^8) encode on a compiled kernel (FFT or generator shape)
  // Working set, fixed when admitted.
  Span payload, up, dev, host;  // staged rows; uploaded descriptors; device-only; pinned image
  size_t up_bytes = 0, dev_bytes = 0;
  Table *table = nullptr;
  bool builds_table = false;
  size_t table_host_off = 0;  // GF(2^8) rows to upload, inside the pinned image
  std::shared_ptr<const Fft16Program> fft16;      // GF(2^16) encode on the FFT route
  std::shared_ptr<const Fft16Program> candidate;  // its program, built at submit
  std::shared_ptr<const Fft16Decode> dec;         // GF(2^16) reconstruct on the FFT route
  std::shared_ptr<const Fft16Decode> dec_candidate;
  size_t scratch_budget = 0;                       // FFT scratch limit
};

struct Group;

}  // namespace rsb

using namespace rsb;

struct rs_server {
  rs_server_config cfg{};
  int device = 0;
  uint8_t *arena = nullptr;
  uint8_t *pinned = nullptr;
  SpanAllocator dev_alloc, host_alloc;
  std::vector<cudaStream_t> streams;
  size_t next_stream = 0;
  // Per-slot group descriptor areas (ragged and FFT item arrays).
  uint8_t *group_dev = nullptr, *group_host = nullptr;
  size_t group_area = 0;
  std::vector<int> free_group_areas;
  std::vector<cudaEvent_t> dead_events;  // of evicted tables; destroyed outside the lock

  std::unordered_map<uint64_t, std::unique_ptr<Table>> tables;
  uint8_t fft_route[8][32] = {};  // [log2 K - 1][log2 bytes]: 0 auto, 1 matrix, 2 FFT
  // The cost model's FFT launch configuration per (shape, alignment, row-bytes and
  // group-size buckets), filled on first use (scheduler thread only).
  std::map<uint64_t, std::pair<int, int>> fft_cfg;

  std::mutex mu;  // queue, completions, counters
  std::condition_variable cv_work, cv_done;
  std::deque<std::unique_ptr<Req>> queue;
  std::deque<Group *> finished;  // groups whose host callback ran
  std::deque<rs_completion> completions;
  bool stop = false;
  bool kicked = false;  // new submissions since the scheduler last looked
  std::thread worker;

  int slots_used = 0;
  uint64_t head_skips = 0;
  rs_server_stats st{};
};

namespace rsb {

struct Group {
  rs_server *srv = nullptr;
  std::vector<std::unique_ptr<Req>> reqs;
  int area = -1;  // group descriptor area index
  uint64_t done_ns = 0;
  int status = RS_OK;
  size_t launches = 0;
};

static void CUDART_CB group_done(void *p) {
  Group *g = static_cast<Group *>(p);
  g->done_ns = now_ns();
  rs_server *s = g->srv;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->finished.push_back(g);
  }
  s->cv_work.notify_all();
}

// Bytes a request needs besides its table: pinned/uploaded descriptor image and
// device-only scratch (decode rows, Lagrange intermediates).
static void size_request(Req &q, bool new_table) {
  const rs_request &r = q.r;
  const size_t k = r.data_shards, m = r.parity_shards, e = q.targets.size();
  size_t up = 0, dev = 0;
  if (r.field == 8) {
    if (r.op != RS_BATCH_ENCODE) {
      up += up256(k * 2) + up256(m * 2) + up256(2);  // survivors | targets | count
      dev += up256(m * k) + up256(sizeof(int));      // decode rows | status
    }
    if (new_table) up += up256(k * m);  // generator rows staged for upload
  } else {
    if (r.op == RS_BATCH_ENCODE && q.fft16) {
      if (new_table) up += up256(fft16_table_bytes(*q.fft16));  // constants staged for upload
      dev += up256(fft16_scratch_bytes(*q.fft16, 1, r.row_len, q.scratch_budget));
    } else if (r.op == RS_BATCH_ENCODE) {
      if (new_table) {
        up += up256(k * 2) + up256(m * 2);                 // nodes | targets
        dev += up256(k * 2) + up256(m * 2) + up256(m * 4);  // w | ell | hit
      }
    } else if (q.dec) {
      // constants | target points | pointer table; decode scratch
      up += up256(q.dec->cols.size() * 2) + up256(e * 4) + up256((k + m) * sizeof(void *));
      dev += up256(fft16_decode_scratch_bytes(*q.dec, r.row_len, q.scratch_budget));
    } else {
      up += up256(k * 2) + up256(e * 2) + up256((k + e) * sizeof(void *));  // nodes | targets | ptrs
      dev += up256(k * 2) + up256(e * 2) + up256(e * 4) + up256(e * k * 4);  // w | ell | hit | rows
    }
  }
  q.up_bytes = up;
  q.dev_bytes = dev;
}

static size_t payload_bytes(const rs_request &r) {
  return r.rows_on_host ? (r.data_shards + r.parity_shards) * r.row_len : 0;
}

static bool take(SpanAllocator &a, size_t bytes, Span &s) {
  if (!bytes) {
    s = Span{};
    return true;
  }
  size_t off;
  if (!a.alloc(bytes, off)) return false;
  s.off = off;
  s.bytes = bytes;
  s.live = true;
  return true;
}

static void give(SpanAllocator &a, Span &s) {
  if (s.live) a.release(s.off, s.bytes);
  s = Span{};
}

// Evicts idle tables, least recently used first, until `bytes` could fit or none is left.
static bool evict_for(rs_server *s, size_t bytes) {
  for (;;) {
    Span probe;
    if (take(s->dev_alloc, bytes, probe)) {
      give(s->dev_alloc, probe);
      return true;
    }
    Table *victim = nullptr;
    for (auto &kv : s->tables)
      if (kv.second->refs == 0 && (!victim || kv.second->last_use < victim->last_use)) victim = kv.second.get();
    if (!victim) return false;
    give(s->dev_alloc, victim->span);
    if (victim->ready) s->dead_events.push_back(victim->ready);
    s->tables.erase(victim->key);
    s->st.evictions++;
  }
}

// Reserves a request's working set; false (nothing held) if it does not fit now.
static bool reserve(rs_server *s, Req &q) {
  const rs_request &r = q.r;
  uint64_t key = table_key(r.field, r.data_shards, r.parity_shards);
  auto it = s->tables.find(key);
  if (it != s->tables.end() && it->second->stale && it->second->refs == 0) {
    give(s->dev_alloc, it->second->span);
    if (it->second->ready) s->dead_events.push_back(it->second->ready);
    s->tables.erase(it);
    it = s->tables.end();
  }
  if (it != s->tables.end() && it->second->stale) return false;
  bool need_table = r.field == 8 || r.op == RS_BATCH_ENCODE;
  bool new_table = need_table && it == s->tables.end();
  q.fft16.reset();
  q.scratch_budget = std::min<size_t>(kFft16ScratchBudget, s->cfg.arena_bytes / 8);
  if (r.field == 16 && r.op == RS_BATCH_ENCODE) {
    if (!new_table) {
      q.fft16 = it->second->fft16;
    } else {
      q.fft16 = q.candidate;
      // The FFT route must fit the arena on its own; otherwise the matrix route.
      if (q.fft16) {
        size_request(q, true);
        if (up256(q.up_bytes) + up256(q.dev_bytes) + up256(fft16_table_bytes(*q.fft16)) > s->cfg.arena_bytes)
          q.fft16.reset();
      }
    }
  }
  if (r.field == 16 && r.op != RS_BATCH_ENCODE) {
    q.dec = q.dec_candidate;
    if (q.dec) {
      size_request(q, false);
      if (up256(q.up_bytes) + up256(q.dev_bytes) > s->cfg.arena_bytes) q.dec.reset();
    }
  }
  size_request(q, new_table);
  size_t tb = !new_table ? 0
              : q.fft16 ? fft16_table_bytes(*q.fft16)
                        : table_bytes(r.field, r.data_shards, r.parity_shards);
  size_t total = up256(payload_bytes(r)) + up256(q.up_bytes) + up256(q.dev_bytes) + up256(tb);
  if (!evict_for(s, total)) return false;
  Span pay, up, dev, host, tab;
  if (!take(s->dev_alloc, payload_bytes(r), pay)) return false;
  if (!take(s->dev_alloc, q.up_bytes, up) || !take(s->dev_alloc, q.dev_bytes, dev) ||
      !take(s->dev_alloc, tb, tab) || !take(s->host_alloc, q.up_bytes, host)) {
    give(s->dev_alloc, pay);
    give(s->dev_alloc, up);
    give(s->dev_alloc, dev);
    give(s->dev_alloc, tab);
    give(s->host_alloc, host);
    return false;
  }
  q.payload = pay;
  q.up = up;
  q.dev = dev;
  q.host = host;
  if (need_table) {
    if (new_table) {
      auto t = std::make_unique<Table>();
      t->key = key;
      t->field = r.field;
      t->k = r.data_shards;
      t->m = r.parity_shards;
      t->span = tab;
      t->fft16 = q.fft16;
      it = s->tables.emplace(key, std::move(t)).first;
      q.builds_table = true;
      s->st.table_builds++;
    } else {
      s->st.table_hits++;
    }
    q.table = it->second.get();
    q.table->refs++;
    q.table->last_use = now_ns();
  }
  return true;
}

static void release_request(rs_server *s, Req &q) {
  give(s->dev_alloc, q.payload);
  give(s->dev_alloc, q.up);
  give(s->dev_alloc, q.dev);
  give(s->host_alloc, q.host);
  if (q.table) {
    q.table->refs--;
    q.table = nullptr;
  }
}

// Launch helpers ------------------------------------------------------------------

static int launch_gf16_server(const Apply16Args &a, cudaStream_t st) {
  if (a.n_sym == 0 || a.rows == 0 || a.n_stripes == 0) return RS_OK;
  Apply16Args b = a;
  dim3 grid;
  unsigned threads;
  gf16_launch_shape(b, sm_count(), grid, threads);
  gf16_matrix_kernel<4, false><<<grid, threads, 0, st>>>(b);
  g_launches++;
  RSB_CU(cudaGetLastError());
  return RS_OK;
}

// Lagrange rows (nodes -> targets) as split constants into `out`; scratch from `w`,
// `ell`, `hit`. The node/target index arrays are already on the device.
static int lagrange16_enqueue(const uint16_t *d_nodes, uint32_t k, const uint16_t *d_t, uint32_t nt, uint16_t *w,
                              uint16_t *ell, uint32_t *hit, uint32_t *out, cudaStream_t st) {
  if (!k || !nt) return RS_OK;
  lagrange16_weights<<<(k + 255) / 256, 256, 0, st>>>(d_nodes, k, w);
  lagrange16_ell<<<(nt + 255) / 256, 256, 0, st>>>(d_nodes, k, d_t, nt, ell, hit);
  uint64_t n = (uint64_t)k * nt;
  lagrange16_rows<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_nodes, k, d_t, nt, w, ell, hit, out, nullptr);
  g_launches += 3;
  RSB_CU(cudaGetLastError());
  return RS_OK;
}

static uint8_t *rows_of(rs_server *s, const Req &q) {
  return q.r.rows_on_host ? s->arena + q.payload.off : q.r.rows;
}

static int stage_in(rs_server *s, const Req &q, cudaStream_t st) {
  if (!q.r.rows_on_host) return RS_OK;
  const rs_request &r = q.r;
  size_t n = r.data_shards + r.parity_shards;
  size_t rows = r.op == RS_BATCH_ENCODE ? r.data_shards : n;
  RSB_CU(cudaMemcpyAsync(rows_of(s, q), r.rows, rows * r.row_len, cudaMemcpyHostToDevice, st));
  return RS_OK;
}

static int stage_out(rs_server *s, const Req &q, cudaStream_t st) {
  if (!q.r.rows_on_host) return RS_OK;
  const rs_request &r = q.r;
  uint8_t *d = rows_of(s, q);
  if (r.op == RS_BATCH_ENCODE) {
    size_t off = r.data_shards * r.row_len;
    RSB_CU(cudaMemcpyAsync(r.rows + off, d + off, r.parity_shards * r.row_len, cudaMemcpyDeviceToHost, st));
    return RS_OK;
  }
  for (uint32_t t : q.targets)
    RSB_CU(cudaMemcpyAsync(r.rows + (size_t)t * r.row_len, d + (size_t)t * r.row_len, r.row_len,
                           cudaMemcpyDeviceToHost, st));
  return RS_OK;
}

// Uploads a request's pinned descriptor image into its device span.
static int upload(rs_server *s, const Req &q, cudaStream_t st) {
  if (!q.up_bytes) return RS_OK;
  RSB_CU(cudaMemcpyAsync(s->arena + q.up.off, s->pinned + q.host.off, q.up_bytes, cudaMemcpyHostToDevice, st));
  return RS_OK;
}

static int wait_table(const Req &q, cudaStream_t st) {
  if (q.table && !q.builds_table && q.table->ready) RSB_CU(cudaStreamWaitEvent(st, q.table->ready, 0));
  return RS_OK;
}

// Called by the table's builder, before any other request can wait on it (those are
// enqueued later, in admission order). CUDA calls stay outside the server mutex.
static int mark_table(const Req &q, cudaStream_t st) {
  if (!q.builds_table) return RS_OK;
  if (!q.table->ready) RSB_CU(cudaEventCreateWithFlags(&q.table->ready, cudaEventDisableTiming));
  RSB_CU(cudaEventRecord(q.table->ready, st));
  return RS_OK;
}

// The launch configuration of one FFT launch group from the server's cost model (none:
// the library's automatic choice): the FFT configuration with the least predicted
// total time for `count` stripes of (K, K) with rows of about `bytes` bytes, where that
// is predicted at least 10% faster than the automatic choice (as rs_batch_choose).
// Decisions are cached per (K, alignment, half-octave of bytes, octave of count): one
// model evaluation per new bucket, on the scheduler thread.
static std::pair<int, int> fft_config(rs_server *s, const FftShape &sh, size_t bytes, size_t count, bool aligned) {
  if (!s->cfg.model || sh.gen) return {-1, -1};
  const int lb = (int)std::lround(2.0 * std::log2((double)std::max<size_t>(bytes, 1)));
  const int lc = (int)std::lround(std::log2((double)std::max<size_t>(count, 1)));
  const uint64_t key = ((uint64_t)sh.k << 32) | ((uint64_t)aligned << 24) | ((uint64_t)lb << 8) | (uint64_t)lc;
  auto it = s->fft_cfg.find(key);
  if (it != s->fft_cfg.end()) return it->second;
  std::pair<int, int> pick{-1, -1};
  float x[kTuneFeatures], *d = nullptr;
  const size_t row = (size_t)std::exp2(lb / 2.0);
  tune_features(sh.k, sh.m, row, 0, tune_batch(sh.k, sh.m, row, (size_t)1 << lc), aligned, x);
  std::vector<float> pred(kTuneConfigCount);
  if (cudaMalloc(&d, sizeof(float) * (kTuneFeatures + kTuneConfigCount)) == cudaSuccess) {
    if (cudaMemcpy(d, x, sizeof x, cudaMemcpyHostToDevice) == cudaSuccess &&
        rs_mlp_predict(s->cfg.model, d, 1, d + kTuneFeatures) == RS_OK &&
        cudaMemcpy(pred.data(), d + kTuneFeatures, sizeof(float) * kTuneConfigCount, cudaMemcpyDeviceToHost) ==
            cudaSuccess) {
      float best = 0;
      for (int c = 0; c < kTuneConfigCount; c++)
        if (kTuneConfigs[c].route == kTuneFft && (pick.first < 0 || pred[c] < best)) {
          best = pred[c];
          pick = {kTuneConfigs[c].p0, kTuneConfigs[c].p1};
        }
      const int auto_cfg = fft_auto_config(sh, aligned);
      if (auto_cfg >= 0 && std::exp((double)best) > 0.9 * std::exp((double)pred[auto_cfg])) pick = {-1, -1};
    }
    cudaFree(d);
  }
  cudaGetLastError();  // a failed evaluation leaves the automatic choice
  s->fft_cfg[key] = pick;
  return pick;
}

// One GF(2^8) launch group: tables, plans, then one FFT launch per K and one ragged
// matrix launch for the rest.
static int enqueue_gf8(rs_server *s, Group &g, cudaStream_t st) {
  uint8_t *gd = s->group_dev + (size_t)g.area * s->group_area;
  uint8_t *gh = s->group_host + (size_t)g.area * s->group_area;
  // Host images: GF(2^8) generator rows for new tables, plan index lists.
  for (auto &qp : g.reqs) {
    Req &q = *qp;
    uint8_t *h = s->pinned + q.host.off;
    size_t off = 0;
    const size_t k = q.r.data_shards, m = q.r.parity_shards;
    if (q.r.op != RS_BATCH_ENCODE) {
      uint16_t *surv = reinterpret_cast<uint16_t *>(h);
      uint16_t *targ = reinterpret_cast<uint16_t *>(h + up256(k * 2));
      uint16_t *nt = reinterpret_cast<uint16_t *>(h + up256(k * 2) + up256(m * 2));
      for (size_t t = 0; t < k; t++) surv[t] = (uint16_t)q.surv[t];
      for (size_t t = 0; t < q.targets.size(); t++) targ[t] = (uint16_t)q.targets[t];
      *nt = (uint16_t)q.targets.size();
      off = up256(k * 2) + up256(m * 2) + up256(2);
    }
    if (q.builds_table) {
      std::vector<uint8_t> rows;
      parity_rows<F8>(k, m, rows);
      memcpy(h + off, rows.data(), k * m);
      q.table_host_off = off;
    }
  }
  for (auto &qp : g.reqs) {
    Req &q = *qp;
    RSB_TRY(stage_in(s, q, st));
    RSB_TRY(upload(s, q, st));
    if (q.builds_table) {
      RSB_CU(cudaMemcpyAsync(s->arena + q.table->span.off, s->arena + q.up.off + q.table_host_off,
                             q.r.data_shards * q.r.parity_shards, cudaMemcpyDeviceToDevice, st));
      RSB_TRY(mark_table(q, st));
    }
    RSB_TRY(wait_table(q, st));
  }
  // Decode rows of every reconstruct (device Gauss-Jordan, first-nonzero pivot).
  for (auto &qp : g.reqs) {
    Req &q = *qp;
    if (q.r.op == RS_BATCH_ENCODE || q.targets.empty()) continue;
    const size_t k = q.r.data_shards, m = q.r.parity_shards;
    uint8_t *u = s->arena + q.up.off;
    uint8_t *d = s->arena + q.dev.off;
    PlanArgs pa{};
    pa.gen = s->arena + q.table->span.off;
    pa.k = (uint32_t)k;
    pa.m = (uint32_t)m;
    pa.survivors = reinterpret_cast<const uint16_t *>(u);
    pa.targets = reinterpret_cast<const uint16_t *>(u + up256(k * 2));
    pa.n_targets = reinterpret_cast<const uint16_t *>(u + up256(k * 2) + up256(m * 2));
    pa.max_rows = (uint32_t)m;
    pa.out = d;
    pa.status = reinterpret_cast<int *>(d + up256(m * k));
    size_t smem = plan_smem((uint32_t)k).total;
    if (smem > 48 * 1024)
      RSB_CU(cudaFuncSetAttribute(gf8_plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    gf8_plan_kernel<<<1, 256, smem, st>>>(pa);
    g_launches++;
    g.launches++;
    RSB_CU(cudaGetLastError());
  }
  // Item arrays in the group's descriptor area: FFT / generator items per compiled
  // shape, then ragged items.
  std::map<const FftShape *, std::vector<FftItem>> ffts;
  std::vector<RaggedItem> ragged;
  uint32_t max_k = 1;
  uint64_t blocks = 0;
  for (auto &qp : g.reqs) {
    Req &q = *qp;
    const size_t k = q.r.data_shards, m = q.r.parity_shards, L = q.r.row_len;
    uint8_t *rows = rows_of(s, q);
    if (q.fft) {
      auto &v = ffts[find_fft_shape(k, m)];
      FftItem f{};
      f.in_base = rows;
      f.out_base = rows + k * L;
      f.row_stride = L;
      f.len = L;
      f.group_begin = v.empty() ? 0 : v.back().group_begin + (v.back().len + 31) / 32;
      v.push_back(f);
      continue;
    }
    if (q.r.op != RS_BATCH_ENCODE && q.targets.empty()) continue;
    RaggedItem r{};
    r.base = rows;
    r.row_stride = L;
    r.len = L;
    r.k = (uint32_t)k;
    if (q.r.op == RS_BATCH_ENCODE) {
      r.coeffs = s->arena + q.table->span.off;
      r.rows = (uint32_t)m;
    } else {
      uint8_t *u = s->arena + q.up.off;
      r.coeffs = s->arena + q.dev.off;
      r.in_rows = reinterpret_cast<const uint16_t *>(u);
      r.out_rows = reinterpret_cast<const uint16_t *>(u + up256(k * 2));
      r.rows = (uint32_t)q.targets.size();
    }
    r.col_tiles = (uint32_t)((L + kTileBytes - 1) / kTileBytes);
    r.block_begin = (uint32_t)blocks;
    blocks += (uint64_t)r.col_tiles * ((r.rows + kRowChunk - 1) / kRowChunk);
    max_k = std::max<uint32_t>(max_k, r.k);
    ragged.push_back(r);
  }
  size_t off = 0;
  for (auto &kv : ffts) {
    size_t bytes = kv.second.size() * sizeof(FftItem);
    memcpy(gh + off, kv.second.data(), bytes);
    off = up256(off + bytes);
  }
  size_t ragged_off = off;
  uint64_t ragged_blocks[2];
  const uint32_t n_ragged0 = ragged_split(ragged, ragged_blocks);
  memcpy(gh + off, ragged.data(), ragged.size() * sizeof(RaggedItem));
  off += ragged.size() * sizeof(RaggedItem);
  if (off) RSB_CU(cudaMemcpyAsync(gd, gh, off, cudaMemcpyHostToDevice, st));
  off = 0;
  for (auto &kv : ffts) {
    const auto &v = kv.second;
    uint64_t groups = v.back().group_begin + (v.back().len + 31) / 32;
    uintptr_t align = 0;
    for (const FftItem &f : v) align |= reinterpret_cast<uintptr_t>(f.in_base) | f.row_stride;
    const std::pair<int, int> cfg = fft_config(s, *kv.first, groups * 32 / v.size(), v.size(), (align & 15) == 0);
    RSB_TRY(launch_fft8_items(*kv.first, reinterpret_cast<const FftItem *>(gd + off), (uint32_t)v.size(), groups, st,
                              nullptr, (align & 15) != 0, cfg.first, cfg.second));
    g.launches++;
    off = up256(off + v.size() * sizeof(FftItem));
  }
  if (!ragged.empty()) {
    size_t smem = 8192 + (size_t)kRowChunk * max_k;
    if (smem > 48 * 1024)
      RSB_CU(cudaFuncSetAttribute(gf8_ragged_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    RSB_CU(launch_ragged(reinterpret_cast<const RaggedItem *>(gd + ragged_off), n_ragged0, (uint32_t)ragged.size(),
                         ragged_blocks, smem, st));
    g_launches += ragged_launches(ragged_blocks);
    g.launches += ragged_launches(ragged_blocks);
  }
  for (auto &qp : g.reqs) RSB_TRY(stage_out(s, *qp, st));
  return RS_OK;
}

// One GF(2^16) request: generator (if new) or decode rows by device Lagrange, then
// the tower matrix kernel.
static int enqueue_gf16(rs_server *s, Group &g, cudaStream_t st) {
  Req &q = *g.reqs[0];
  const rs_request &r = q.r;
  const size_t k = r.data_shards, m = r.parity_shards, n = k + m, e = q.targets.size();
  uint8_t *h = s->pinned + q.host.off;
  uint8_t *u = s->arena + q.up.off;
  uint8_t *d = s->arena + q.dev.off;
  uint8_t *rows = rows_of(s, q);
  RSB_TRY(stage_in(s, q, st));
  Apply16Args a{};
  a.n_sym = r.row_len / 2;
  a.n_stripes = 1;
  a.k = (uint32_t)k;
  if (r.op == RS_BATCH_ENCODE && q.fft16) {
    const Fft16Program &p = *q.fft16;
    if (q.builds_table) {
      memcpy(h, p.cols.data(), fft16_table_bytes(p));
      RSB_CU(cudaMemcpyAsync(s->arena + q.table->span.off, h, fft16_table_bytes(p), cudaMemcpyHostToDevice, st));
      RSB_TRY(mark_table(q, st));
    }
    RSB_TRY(wait_table(q, st));
    const uint64_t before = g_launches.load();
    RSB_TRY(fft16_run(p, reinterpret_cast<const uint16_t *>(s->arena + q.table->span.off), d, q.dev.bytes, rows,
                      r.row_len, 0, rows + k * r.row_len, r.row_len, 0, nullptr, 1, r.row_len, st));
    g.launches += g_launches.load() - before;
    return stage_out(s, q, st);
  }
  if (r.op == RS_BATCH_ENCODE) {
    if (q.builds_table) {
      uint16_t *nodes = reinterpret_cast<uint16_t *>(h), *tg = reinterpret_cast<uint16_t *>(h + up256(k * 2));
      for (size_t i = 0; i < k; i++) nodes[i] = (uint16_t)i;
      for (size_t j = 0; j < m; j++) tg[j] = (uint16_t)(k + j);
      RSB_TRY(upload(s, q, st));
      RSB_TRY(lagrange16_enqueue(reinterpret_cast<uint16_t *>(u), (uint32_t)k,
                                 reinterpret_cast<uint16_t *>(u + up256(k * 2)), (uint32_t)m,
                                 reinterpret_cast<uint16_t *>(d), reinterpret_cast<uint16_t *>(d + up256(k * 2)),
                                 reinterpret_cast<uint32_t *>(d + up256(k * 2) + up256(m * 2)),
                                 reinterpret_cast<uint32_t *>(s->arena + q.table->span.off), st));
      g.launches += 3;
      RSB_TRY(mark_table(q, st));
    }
    RSB_TRY(wait_table(q, st));
    a.in_base = rows;
    a.in_row_stride = r.row_len;
    a.out_base = rows + k * r.row_len;
    a.out_row_stride = r.row_len;
    a.coeffs = reinterpret_cast<const uint32_t *>(s->arena + q.table->span.off);
    a.rows = (uint32_t)m;
  } else if (q.dec) {
    if (e == 0) return RS_OK;
    const Fft16Decode &dd = *q.dec;
    const size_t cb = up256(dd.cols.size() * 2), tb = up256(e * 4);
    memcpy(h, dd.cols.data(), dd.cols.size() * 2);
    uint32_t *tg = reinterpret_cast<uint32_t *>(h + cb);
    for (size_t j = 0; j < e; j++) tg[j] = q.targets[j];
    uint8_t **ptrs = reinterpret_cast<uint8_t **>(h + cb + tb);
    for (size_t i = 0; i < n; i++) ptrs[i] = rows + i * r.row_len;
    RSB_TRY(upload(s, q, st));
    const uint64_t before = g_launches.load();
    RSB_TRY(fft16_decode_run(dd, reinterpret_cast<const uint16_t *>(u), d, q.dev.bytes,
                             reinterpret_cast<uint8_t *const *>(u + cb + tb), reinterpret_cast<const uint32_t *>(u + cb),
                             e, r.row_len, st));
    g.launches += g_launches.load() - before;
    return stage_out(s, q, st);
  } else {
    if (e == 0) return RS_OK;
    uint16_t *nodes = reinterpret_cast<uint16_t *>(h), *tg = reinterpret_cast<uint16_t *>(h + up256(k * 2));
    uint8_t **ptrs = reinterpret_cast<uint8_t **>(h + up256(k * 2) + up256(e * 2));
    for (size_t i = 0; i < k; i++) {
      nodes[i] = (uint16_t)q.surv[i];
      ptrs[i] = rows + (size_t)q.surv[i] * r.row_len;
    }
    for (size_t j = 0; j < e; j++) {
      tg[j] = (uint16_t)q.targets[j];
      ptrs[k + j] = rows + (size_t)q.targets[j] * r.row_len;
    }
    (void)n;
    RSB_TRY(upload(s, q, st));
    uint32_t *coeffs = reinterpret_cast<uint32_t *>(d + up256(k * 2) + up256(e * 2) + up256(e * 4));
    RSB_TRY(lagrange16_enqueue(reinterpret_cast<uint16_t *>(u), (uint32_t)k,
                               reinterpret_cast<uint16_t *>(u + up256(k * 2)), (uint32_t)e,
                               reinterpret_cast<uint16_t *>(d), reinterpret_cast<uint16_t *>(d + up256(k * 2)),
                               reinterpret_cast<uint32_t *>(d + up256(k * 2) + up256(e * 2)), coeffs, st));
    g.launches += 3;
    uint8_t *const *dptrs = reinterpret_cast<uint8_t *const *>(u + up256(k * 2) + up256(e * 2));
    a.in_ptrs = reinterpret_cast<const uint8_t *const *>(dptrs);
    a.out_ptrs = dptrs + k;
    a.coeffs = coeffs;
    a.rows = (uint32_t)e;
  }
  RSB_TRY(launch_gf16_server(a, st));
  g.launches++;
  return stage_out(s, q, st);
}

static void complete_group(rs_server *s, Group *g) {
  std::lock_guard<std::mutex> lock(s->mu);
  for (auto &qp : g->reqs) {
    Req &q = *qp;
    rs_completion c{};
    c.tag = q.r.tag;
    c.status = g->status ? g->status : q.status;
    c.submit_ns = q.submit_ns;
    c.admit_ns = q.admit_ns;
    c.done_ns = g->done_ns ? g->done_ns : now_ns();
    c.bytes = q.bytes;
    c.group_size = (uint32_t)g->reqs.size();
    if (g->status && q.builds_table) q.table->stale = true;
    release_request(s, q);
    s->completions.push_back(c);
    s->st.completed++;
    if (c.status == RS_OK) s->st.bytes += c.bytes;
  }
  if (g->area >= 0) s->free_group_areas.push_back(g->area);
  s->slots_used -= (int)g->reqs.size();
  s->st.groups++;
  s->st.launches += g->launches;
  if (g->reqs.size() > 1) s->st.merged += g->reqs.size();
  delete g;
}

static void launch_group(rs_server *s, Group *g) {
  cudaStream_t st = s->streams[s->next_stream++ % s->streams.size()];
  uint64_t t = now_ns();
  for (auto &q : g->reqs) q->admit_ns = t;
  int rc = g->reqs[0]->r.field == 8 ? enqueue_gf8(s, *g, st) : enqueue_gf16(s, *g, st);
  if (rc == RS_OK) {
    cudaError_t e = cudaLaunchHostFunc(st, group_done, g);
    if (e == cudaSuccess) return;
    set_cuda_error(e, "cudaLaunchHostFunc");
    rc = RS_ERR_CUDA;
  }
  // Failed while enqueuing: drain what was enqueued, then complete with the error.
  cudaStreamSynchronize(st);
  cudaGetLastError();
  g->status = rc;
  complete_group(s, g);
}

static bool route_fft(const rs_server *s, const rs_request &r) {
  const FftShape *sh = find_fft_shape(r.data_shards, r.parity_shards);
  if (!sh || r.op != RS_BATCH_ENCODE) return false;
  if (sh->gen) return r.row_len >= 64;  // no per-size hints for generator shapes
  int kl = 0;
  while ((1 << (kl + 1)) <= sh->k) kl++;
  int bl = 0;
  while (bl < 31 && ((size_t)2 << bl) <= r.row_len) bl++;
  uint8_t hint = s->fft_route[kl - 1][bl];
  if (hint == 1) return false;
  if (hint == 2) return true;
  return r.row_len >= 64;
}

static void scheduler(rs_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    std::vector<Group *> done;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv_work.wait_for(lock, std::chrono::milliseconds(2), [&] {
        return s->kicked || !s->finished.empty() || (s->stop && s->slots_used == 0);
      });
      s->kicked = false;
      while (!s->finished.empty()) {
        done.push_back(s->finished.front());
        s->finished.pop_front();
      }
      if (s->stop && s->slots_used == 0 && done.empty()) return;
    }
    for (Group *g : done) complete_group(s, g);
    if (!done.empty()) s->cv_done.notify_all();

    // Admission in FIFO order. Requests behind one that does not fit are admitted only
    // within the lookahead window, and not once the blocked head has been passed over
    // 8 x slots times (so a large request is not starved by a stream of small ones).
    Group *g8 = nullptr;
    std::vector<Group *> ready;
    std::vector<cudaEvent_t> dead;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      if (s->stop) continue;
      size_t passed = 0;
      const uint64_t starve = 8 * (uint64_t)s->cfg.slots;
      for (auto it = s->queue.begin(); it != s->queue.end();) {
        if (s->slots_used >= s->cfg.slots) break;
        if (passed && (passed > (size_t)s->cfg.lookahead || s->head_skips >= starve)) break;
        Req &q = **it;
        if (q.r.field == 8 && !g8 && s->free_group_areas.empty()) break;
        if (!reserve(s, q)) {
          passed++;
          ++it;
          continue;
        }
        if (passed)
          s->head_skips++;
        else
          s->head_skips = 0;
        std::unique_ptr<Req> req = std::move(*it);
        it = s->queue.erase(it);
        s->slots_used++;
        if (req->r.field == 8) {
          req->fft = route_fft(s, req->r);
          if (!g8) {
            g8 = new Group();
            g8->srv = s;
            g8->area = s->free_group_areas.back();
            s->free_group_areas.pop_back();
          }
          g8->reqs.push_back(std::move(req));
          if (g8->reqs.size() >= (size_t)s->cfg.max_batch) {
            ready.push_back(g8);
            g8 = nullptr;
          }
        } else {
          Group *g = new Group();
          g->srv = s;
          g->reqs.push_back(std::move(req));
          ready.push_back(g);
        }
      }
      if (g8) ready.push_back(g8);
      dead.swap(s->dead_events);
    }
    for (cudaEvent_t e : dead) cudaEventDestroy(e);
    for (Group *g : ready) launch_group(s, g);
  }
}

static int validate(const rs_request &r, Req &q) {
  if (!r.rows || (r.field != 8 && r.field != 16) || r.op < 0 || r.op > 2) return RS_ERR_INVALID_ARGUMENT;
  const size_t k = r.data_shards, m = r.parity_shards, n = k + m;
  if (k == 0) return RS_TOO_FEW_DATA_SHARDS;
  if (m == 0) return RS_TOO_FEW_PARITY_SHARDS;
  if (n > (r.field == 8 ? 256u : 65536u)) return RS_TOO_MANY_SHARDS;
  if (r.row_len == 0) return RS_EMPTY_SHARD;
  if (r.field == 16 && (r.row_len % 2)) return RS_INCORRECT_SHARD_SIZE;
  q.bytes = n * r.row_len;
  if (r.op == RS_BATCH_ENCODE) return RS_OK;
  if (!r.present) return RS_ERR_INVALID_ARGUMENT;
  q.present.assign(r.present, r.present + n);
  size_t cnt = 0;
  for (size_t i = 0; i < n; i++) cnt += q.present[i] ? 1 : 0;
  if (cnt < k) return RS_TOO_FEW_SHARDS_PRESENT;
  // Survivors: the first k present; rebuilt: missing data, then (unless data only)
  // missing parity (src/reedsolomon.rs:550-566).
  for (size_t i = 0; i < n; i++)
    if (q.present[i] && q.surv.size() < k) q.surv.push_back((uint32_t)i);
  for (size_t i = 0; i < k; i++)
    if (!q.present[i]) q.targets.push_back((uint32_t)i);
  if (r.op == RS_BATCH_RECONSTRUCT)
    for (size_t i = k; i < n; i++)
      if (!q.present[i]) q.targets.push_back((uint32_t)i);
  q.bytes = (k + q.targets.size()) * r.row_len;
  return RS_OK;
}

}  // namespace rsb

extern "C" {

int rs_server_create(const rs_server_config *config, rs_server_t **out) {
  if (!out) return RS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int dev = 0;
  RSB_TRY(ensure_device(&dev));
  std::unique_ptr<rs_server> s(new (std::nothrow) rs_server());
  if (!s) return RS_ERR_ALLOC;
  if (config) s->cfg = *config;
  if (!s->cfg.arena_bytes) s->cfg.arena_bytes = (size_t)1 << 30;
  if (!s->cfg.pinned_bytes) s->cfg.pinned_bytes = (size_t)64 << 20;
  if (s->cfg.slots <= 0) s->cfg.slots = 64;
  if (s->cfg.streams <= 0) s->cfg.streams = 4;
  if (s->cfg.max_batch <= 0) s->cfg.max_batch = 64;
  if (s->cfg.lookahead < 0) s->cfg.lookahead = 0;
  s->device = dev;
  RSB_CU(cudaSetDevice(dev));
  size_t free_b = 0, total_b = 0;
  RSB_CU(cudaMemGetInfo(&free_b, &total_b));
  if (s->cfg.arena_bytes + ((size_t)256 << 20) > free_b) return RS_ERR_TOO_LARGE;
  s->cfg.arena_bytes = up256(s->cfg.arena_bytes);
  s->cfg.pinned_bytes = up256(s->cfg.pinned_bytes);
  if (cudaMalloc(&s->arena, s->cfg.arena_bytes) != cudaSuccess) {
    cudaGetLastError();
    return RS_ERR_ALLOC;
  }
  if (cudaMallocHost(&s->pinned, s->cfg.pinned_bytes) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(s->arena);
    return RS_ERR_ALLOC;
  }
  s->group_area = up256((size_t)s->cfg.max_batch * (sizeof(RaggedItem) + sizeof(FftItem)) + 8 * 256);
  size_t areas = (size_t)s->cfg.slots;
  bool ok = cudaMalloc(&s->group_dev, areas * s->group_area) == cudaSuccess &&
            cudaMallocHost(&s->group_host, areas * s->group_area) == cudaSuccess;
  for (int i = 0; ok && i < s->cfg.streams; i++) {
    cudaStream_t st;
    ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) s->streams.push_back(st);
  }
  if (!ok) {
    cudaGetLastError();
    for (auto st : s->streams) cudaStreamDestroy(st);
    if (s->group_dev) cudaFree(s->group_dev);
    if (s->group_host) cudaFreeHost(s->group_host);
    cudaFree(s->arena);
    cudaFreeHost(s->pinned);
    return RS_ERR_ALLOC;
  }
  for (size_t i = 0; i < areas; i++) s->free_group_areas.push_back((int)(areas - 1 - i));
  s->dev_alloc.reset(s->cfg.arena_bytes);
  s->host_alloc.reset(s->cfg.pinned_bytes);
  s->st.arena_bytes = s->cfg.arena_bytes;
  rs_server *raw = s.get();
  s->worker = std::thread([raw] { scheduler(raw); });
  *out = s.release();
  return RS_OK;
}

int rs_server_submit(rs_server_t *s, const rs_request *reqs, size_t n, int *statuses) {
  if (!s || (!reqs && n)) return RS_ERR_INVALID_ARGUMENT;
  std::vector<std::unique_ptr<Req>> accepted;
  std::vector<rs_completion> immediate;
  uint64_t t = now_ns();
  for (size_t i = 0; i < n; i++) {
    auto q = std::make_unique<Req>();
    q->r = reqs[i];
    q->submit_ns = t;
    int st = validate(reqs[i], *q);
    // A GF(2^16) request with k + m <= 256 has all its coefficients in the GF(2^8)
    // subfield, which scales the two byte planes alike: after the tower's own checks it
    // runs as the GF(2^8) request of its shape (and shares that shape's table and
    // launch groups).
    if (st == RS_OK && q->r.field == 16 && q->r.data_shards + q->r.parity_shards <= 256) q->r.field = 8;
    if (st == RS_OK) {
      // Largest working set it could ever need (building its table) must fit an empty
      // arena on at least one route.
      const rs_request &r = q->r;
      size_request(*q, true);
      size_t tb = (r.field == 8 || r.op == RS_BATCH_ENCODE) ? table_bytes(r.field, r.data_shards, r.parity_shards)
                                                             : 0;
      size_t need = up256(payload_bytes(r)) + up256(q->up_bytes) + up256(q->dev_bytes) + up256(tb);
      bool fits = need <= s->cfg.arena_bytes && up256(q->up_bytes) <= s->cfg.pinned_bytes;
      if (r.field == 16 && r.op == RS_BATCH_ENCODE) {
        auto p = std::make_shared<Fft16Program>();
        if (fft16_build(r.data_shards, r.parity_shards, *p) && fft16_faster(*p, r.row_len, 1)) {
          q->candidate = p;
          q->fft16 = p;
          q->scratch_budget = std::min<size_t>(kFft16ScratchBudget, s->cfg.arena_bytes / 8);
          size_request(*q, true);
          size_t need_fft = up256(payload_bytes(r)) + up256(q->up_bytes) + up256(q->dev_bytes) +
                            up256(fft16_table_bytes(*p));
          fits = fits || (need_fft <= s->cfg.arena_bytes && up256(q->up_bytes) <= s->cfg.pinned_bytes);
          q->fft16.reset();
        }
      }
      if (r.field == 16 && r.op != RS_BATCH_ENCODE && !q->targets.empty()) {
        auto dd = std::make_shared<Fft16Decode>();
        if (fft16_decode_build(r.data_shards, r.parity_shards, q->surv, q->targets, *dd) &&
            fft16_decode_preferred(*dd, r.data_shards)) {
          q->dec_candidate = dd;
          q->dec = dd;
          q->scratch_budget = std::min<size_t>(kFft16ScratchBudget, s->cfg.arena_bytes / 8);
          size_request(*q, false);
          size_t need_dec = up256(payload_bytes(r)) + up256(q->up_bytes) + up256(q->dev_bytes);
          fits = fits || (need_dec <= s->cfg.arena_bytes && up256(q->up_bytes) <= s->cfg.pinned_bytes);
          q->dec.reset();
        }
      }
      if (!fits) st = RS_ERR_TOO_LARGE;
    }
    if (statuses) statuses[i] = st;
    if (st != RS_OK) {
      std::lock_guard<std::mutex> lock(s->mu);
      s->st.rejected++;
      continue;
    }
    if (reqs[i].op != RS_BATCH_ENCODE && q->targets.empty()) {
      rs_completion c{};  // nothing to rebuild
      c.tag = reqs[i].tag;
      c.submit_ns = c.admit_ns = c.done_ns = t;
      c.group_size = 0;
      immediate.push_back(c);
      continue;
    }
    accepted.push_back(std::move(q));
  }
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->st.submitted += accepted.size() + immediate.size();
    for (auto &c : immediate) {
      s->completions.push_back(c);
      s->st.completed++;
    }
    for (auto &q : accepted) s->queue.push_back(std::move(q));
    s->kicked = true;
  }
  s->cv_work.notify_all();
  if (!immediate.empty()) s->cv_done.notify_all();
  return RS_OK;
}

int rs_server_poll(rs_server_t *s, rs_completion *out, size_t cap, size_t *n_out, int timeout_ms) {
  if (!s || !n_out || (!out && cap)) return RS_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lock(s->mu);
  if (s->completions.empty() && timeout_ms != 0) {
    auto pred = [&] { return !s->completions.empty(); };
    if (timeout_ms < 0)
      s->cv_done.wait(lock, pred);
    else
      s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), pred);
  }
  size_t n = std::min(cap, s->completions.size());
  for (size_t i = 0; i < n; i++) {
    out[i] = s->completions.front();
    s->completions.pop_front();
  }
  *n_out = n;
  return RS_OK;
}

int rs_server_set_fft_route(rs_server_t *s, size_t k, int log2_bytes, int route) {
  if (!s || route < 0 || route > 2 || log2_bytes < 0 || log2_bytes > 31) return RS_ERR_INVALID_ARGUMENT;
  const FftShape *sh = find_fft_shape(k, k);
  if (!sh || sh->gen) return RS_ERR_INVALID_ARGUMENT;
  int kl = 0;
  while ((1 << (kl + 1)) <= sh->k) kl++;
  std::lock_guard<std::mutex> lock(s->mu);
  s->fft_route[kl - 1][log2_bytes] = (uint8_t)route;
  return RS_OK;
}

int rs_server_stats_get(rs_server_t *s, rs_server_stats *out) {
  if (!s || !out) return RS_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  *out = s->st;
  out->queued = s->queue.size();
  out->in_flight = (size_t)s->slots_used;
  out->arena_used = s->dev_alloc.used;
  out->arena_peak = s->dev_alloc.peak;
  out->resident_tables = s->tables.size();
  return RS_OK;
}

void rs_server_free(rs_server_t *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
    // Requests not yet admitted are dropped.
    s->queue.clear();
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->device);
  for (auto st : s->streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (auto &kv : s->tables)
    if (kv.second->ready) cudaEventDestroy(kv.second->ready);
  for (cudaEvent_t e : s->dead_events) cudaEventDestroy(e);
  cudaFree(s->group_dev);
  cudaFreeHost(s->group_host);
  cudaFree(s->arena);
  cudaFreeHost(s->pinned);
  delete s;
}

}  // extern "C"
