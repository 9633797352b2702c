// Shared runtime pieces of the rs_b200 library: status handling, device buffers,
// per-codec execution contexts, presence masks and the decode-plan cache.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "rs_b200.h"

namespace rsb {

extern std::atomic<uint64_t> g_launches;
void set_cuda_error(cudaError_t e, const char *what);
int ensure_device(int *device_out);

#define RSB_CU(call)                          \
  do {                                        \
    cudaError_t e_ = (call);                  \
    if (e_ != cudaSuccess) {                  \
      ::rsb::set_cuda_error(e_, #call);       \
      return RS_ERR_CUDA;                     \
    }                                         \
  } while (0)

#define RSB_TRY(expr)           \
  do {                          \
    int st_ = (expr);           \
    if (st_ != RS_OK) return st_; \
  } while (0)

// Stream-ordered scratch from a pool this library owns on the current device. The pool
// keeps up to 1 GiB mapped between calls (the default pool returns memory at every
// synchronisation, so large per-call scratch would be mapped again on each call).
cudaError_t scratch_alloc(void **p, size_t bytes, cudaStream_t st);
inline void scratch_free(void *p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}

// Grow-only device allocation owned by one execution context.
struct DeviceBuf {
  uint8_t *ptr = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return RS_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    size_t want = std::max(bytes, (size_t)1 << 20);
    if (cudaMalloc(&ptr, want) != cudaSuccess) {
      cudaGetLastError();
      return RS_ERR_ALLOC;
    }
    cap = want;
    return RS_OK;
  }
  ~DeviceBuf() {
    if (ptr) cudaFree(ptr);
  }
};

// Pinned host staging for a call's small upload (index lists, work items), two buffers
// used in turn: a buffer is refilled only once the copy that last read it has run, so a
// call does not wait for the previous call's device work, and its upload is one
// asynchronous copy from pinned memory instead of several from pageable memory.
struct HostStage {
  struct Buf {
    uint8_t *ptr = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
    bool pending = false;
  };
  Buf b[2];
  int next = 0;
  // The next buffer, grown to at least `bytes` and free to be written.
  int acquire(size_t bytes, Buf *&out) {
    Buf &x = b[next];
    next ^= 1;
    if (x.pending) {
      RSB_CU(cudaEventSynchronize(x.ev));
      x.pending = false;
    }
    if (bytes > x.cap) {
      if (x.ptr) cudaFreeHost(x.ptr);
      x.ptr = nullptr;
      x.cap = 0;
      const size_t want = std::max(bytes, (size_t)1 << 20);
      RSB_CU(cudaMallocHost(&x.ptr, want));
      x.cap = want;
    }
    if (!x.ev) RSB_CU(cudaEventCreateWithFlags(&x.ev, cudaEventDisableTiming));
    out = &x;
    return RS_OK;
  }
  // After the copy that reads x has been enqueued on st.
  int release(Buf &x, cudaStream_t st) {
    RSB_CU(cudaEventRecord(x.ev, st));
    x.pending = true;
    return RS_OK;
  }
  ~HostStage() {
    for (Buf &x : b) {
      if (x.pending) cudaEventSynchronize(x.ev);
      if (x.ptr) cudaFreeHost(x.ptr);
      if (x.ev) cudaEventDestroy(x.ev);
    }
  }
};

// Pinned host memory that grows on demand and is kept for later calls.
struct PinnedBuf {
  uint8_t *ptr = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return RS_OK;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
    RSB_CU(cudaMallocHost(&ptr, bytes));
    cap = bytes;
    return RS_OK;
  }
  ~PinnedBuf() {
    if (ptr) cudaFreeHost(ptr);
  }
};

// Host copies of `count` pieces (copy_piece(i) for i < count), on up to
// host_copy_threads() host threads (the caller's included) when there are at least
// 8 MiB to move, where one thread's memcpy rate (about 11 GB/s on the B200 boxes' hosts)
// would bound the call. A thread that cannot be started leaves its share to the others.
inline std::atomic<int> &host_copy_threads() {
  static std::atomic<int> t{8};
  return t;
}
template <class F>
inline void host_copy_pieces(size_t count, size_t total_bytes, const F &copy_piece) {
  const unsigned hw = std::thread::hardware_concurrency();
  const size_t maxt = (size_t)std::max(1, host_copy_threads().load());
  size_t nt = total_bytes >= (8u << 20) ? std::min<size_t>(std::min<size_t>(maxt, hw ? hw : 1), count) : 1;
  if (nt <= 1) {
    for (size_t i = 0; i < count; i++) copy_piece(i);
    return;
  }
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (size_t i = next.fetch_add(1); i < count; i = next.fetch_add(1)) copy_piece(i);
  };
  std::vector<std::thread> ts;
  try {
    ts.reserve(nt - 1);
    for (size_t t = 1; t < nt; t++) ts.emplace_back(work);
  } catch (...) {
  }
  work();
  for (auto &t : ts) t.join();
}

// Rows of `len` bytes between host buffers and pinned staging `pitch` apart, by host
// threads in pieces of at most 1 MiB: gather copies row i from src(i) to h + i * pitch,
// scatter copies h + i * pitch to dst(i).
template <class SrcF>
inline void gather_rows(uint8_t *h, size_t pitch, size_t count, size_t len, const SrcF &src) {
  const size_t piece = std::min<size_t>(len, 1u << 20), per = (len + piece - 1) / piece;
  host_copy_pieces(count * per, count * len, [&](size_t i) {
    const size_t r = i / per, off = (i % per) * piece;
    memcpy(h + r * pitch + off, src(r) + off, std::min(piece, len - off));
  });
}
template <class DstF>
inline void scatter_rows(const uint8_t *h, size_t pitch, size_t count, size_t len, const DstF &dst) {
  const size_t piece = std::min<size_t>(len, 1u << 20), per = (len + piece - 1) / piece;
  host_copy_pieces(count * per, count * len, [&](size_t i) {
    const size_t r = i / per, off = (i % per) * piece;
    memcpy(dst(r) + off, h + r * pitch + off, std::min(piece, len - off));
  });
}

// Host-pointer calls whose rows crossing the link stay within this size are staged
// through pinned memory (PinnedBuf, gather_rows / scatter_rows) in one copy each way.
constexpr size_t kStagedCallBytes = 256u << 20;

// Whether host-pointer calls stage through pinned memory (rs_set_host_staging; on by
// default), and whether a call moving `bytes` across the link does.
inline std::atomic<int> &host_staging_on() {
  static std::atomic<int> on{1};
  return on;
}
inline bool host_staged(size_t bytes) { return host_staging_on().load() != 0 && bytes <= kStagedCallBytes; }

// Serialises host-pointer calls on one codec and owns their staging memory.
struct Exec {
  static constexpr int kPipe = 3;  // streams of the pipelined host batch path
  int device = 0;
  std::mutex mu;
  DeviceBuf buf;
  DeviceBuf aux;
  DeviceBuf pipe_buf;
  HostStage stage;  // uploads of the batched device calls
  PinnedBuf io;     // host-pointer encodes: the stripe gathered into pinned memory
  cudaStream_t stream = nullptr;
  cudaStream_t pipe[kPipe] = {nullptr, nullptr, nullptr};
  ~Exec() {
    if (stream) cudaStreamDestroy(stream);
    for (auto s : pipe)
      if (s) cudaStreamDestroy(s);
  }
  int pipe_streams() {
    for (auto &s : pipe)
      if (!s) RSB_CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return RS_OK;
  }
  int init(int dev) {
    device = dev;
    RSB_CU(cudaSetDevice(dev));
    RSB_CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    return RS_OK;
  }
};

inline int make_exec(int device, std::shared_ptr<Exec> &out) {
  auto e = std::make_shared<Exec>();
  RSB_TRY(e->init(device));
  out = e;
  return RS_OK;
}

// Which shard slots are present, one bit per index (src/reedsolomon.rs:103-115).
struct Presence {
  std::vector<uint64_t> bits;
  explicit Presence(size_t n = 0) : bits((n + 63) / 64, 0) {}
  void set(size_t i) { bits[i / 64] |= 1ull << (i % 64); }
  bool get(size_t i) const { return (bits[i / 64] >> (i % 64)) & 1; }
  bool operator==(const Presence &o) const { return bits == o.bits; }
  bool operator!=(const Presence &o) const { return bits != o.bits; }
};

// One erasure pattern's plan: survivors (first k present, ascending), the missing
// indexes (data ascending, then parity ascending) and device rows mapping the
// survivors to each missing shard, in that order.
struct Fft16Decode;

struct Plan {
  Presence presence;
  std::vector<uint32_t> survivors, missing_data, missing_parity;
  int device = 0;
  void *d_rows = nullptr;  // rows x k coefficients (u8 for GF(2^8), split u32 for the tower)
  // Tower patterns decoded on the FFT route instead: the decode program; d_rows then
  // holds its constants followed by its target points (u32).
  std::shared_ptr<const Fft16Decode> fft16;
  uint64_t fft16_targets_off = 0;  // byte offset of the target points in d_rows
  ~Plan() {
    if (d_rows) {
      cudaSetDevice(device);
      cudaFree(d_rows);
    }
  }
};

// Recently used plans, most recent first, at most 64 (src/reedsolomon.rs:24,592-613).
struct PlanCache {
  static constexpr size_t kLimit = 64;
  std::shared_mutex mu;
  std::vector<std::pair<Presence, std::shared_ptr<const Plan>>> list;
  std::shared_ptr<const Plan> find(const Presence &p) {
    std::shared_lock<std::shared_mutex> lock(mu);
    for (auto &e : list)
      if (e.first == p) return e.second;
    return nullptr;
  }
  std::shared_ptr<const Plan> insert(const Presence &p, std::shared_ptr<const Plan> plan) {
    std::unique_lock<std::shared_mutex> lock(mu);
    for (auto &e : list)
      if (e.first == p) return e.second;  // a racing thread won; reuse its plan
    list.insert(list.begin(), {p, plan});
    if (list.size() > kLimit) list.resize(kLimit);
    return plan;
  }
  void copy_from(PlanCache &o) {
    std::shared_lock<std::shared_mutex> lock(o.mu);
    list = o.list;
  }
};

// Presence scan of reconstruct, src/reedsolomon.rs:801-821 (GF(2^8)) and
// src/reedsolomon16.rs:690-703 (tower: even lengths only).
inline int scan_shards(const size_t *lens, const uint8_t *present, size_t n, bool even,
                       Presence &pres, size_t &n_present, size_t &shard_len) {
  pres = Presence(n);
  n_present = 0;
  shard_len = 0;
  for (size_t i = 0; i < n; i++) {
    if (!present[i]) continue;
    size_t len = lens[i];
    if (len == 0) return RS_EMPTY_SHARD;
    if (even && (len % 2)) return RS_INCORRECT_SHARD_SIZE;
    if (shard_len && shard_len != len) return RS_INCORRECT_SHARD_SIZE;
    shard_len = len;
    pres.set(i);
    n_present++;
  }
  return RS_OK;
}

// Survivors and missing lists of a pattern, src/reedsolomon.rs:550-566.
inline void split_pattern(const Presence &p, size_t k, size_t n, std::vector<uint32_t> &surv,
                          std::vector<uint32_t> &md, std::vector<uint32_t> &mp) {
  surv.clear();
  md.clear();
  mp.clear();
  for (size_t i = 0; i < n; i++) {
    if (p.get(i)) {
      if (surv.size() < k) surv.push_back((uint32_t)i);
    } else if (i < k) {
      md.push_back((uint32_t)i);
    } else {
      mp.push_back((uint32_t)i);
    }
  }
}

// Buffer gather of reconstruct_with_plan, src/reedsolomon.rs:837-864: an absent
// buffer that will be written must already have the shard length (absent parity
// buffers are skipped when only data is rebuilt).
inline int check_absent_buffers(const size_t *lens, const uint8_t *present, size_t n, size_t k,
                                size_t shard_len, bool data_only) {
  for (size_t i = 0; i < n; i++) {
    if (present[i]) continue;
    if (i >= k && data_only) continue;
    if (lens[i] != shard_len) return RS_INCORRECT_SHARD_SIZE;
  }
  return RS_OK;
}

}  // namespace rsb
