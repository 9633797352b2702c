// Persistent work queue: one long-running launch that codes stripes while the host keeps
// adding them (include/rs_b200.h, rs_queue_*). No counterpart in the reference.
//
// The host cuts every stripe (any GF(2^8) shape, shard length and erasure pattern) into
// units of at most kUnitBlocks blocks of the ragged matrix kernel's work (a block is one
// row chunk x one 4 KiB column tile of one stripe) and appends the units to a descriptor
// array in mapped pinned host memory, then raises the published count there. The
// persistent kernel's CTAs claim unit indexes from a device counter and wait for each to
// be published before running it. Every wait is bounded: a CTA that has waited
// `timeout_ns` on the device's global timer for its unit (a producer that stopped
// without closing the queue) sets RS_ERR_TIMEOUT in the queue's status and returns, and
// so does every CTA that sees that status; the kernel issues no asynchronous copies, so
// nothing is in flight when it returns. The launch is captured once into a CUDA graph and
// each session replays it.
//
// Memory ordering: the host writes a unit's descriptor, then a release fence, then the
// published count; the device reads the count with ld.acquire.sys and only then the
// descriptor. Coefficient rows of reconstruct units are copied to device memory and that
// copy is waited for before the units are published.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include "codec8.hpp"
#include "gf_host.hpp"
#include "kernels_batch.cuh"
#include "kernels_bits.cuh"
#include "runtime.hpp"

namespace rsb {

constexpr uint32_t kUnitBlocks = 16;

struct QueueUnit {
  RaggedItem item;  // block_begin unused
  uint32_t b0, b1;  // blocks [b0, b1) of the item
};

struct QueueCtl {  // mapped pinned host memory, written by the host
  unsigned long long published;  // units [0, published) are valid
  unsigned int closed;           // 1: nothing comes after `published`
  unsigned int pad;
};

struct QueueDev {  // device memory
  unsigned long long next;  // claim counter
  unsigned long long done;  // finished units
  int status;               // RS_OK, or RS_ERR_TIMEOUT when a wait gave up
  int pad;
};

__device__ __forceinline__ unsigned long long ld_acquire_sys(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned int ld_acquire_sys_u32(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// A unit's blocks run on the lookup kernel's ragged block (kernels_bits.cuh), with the
// 8-row output tile for units of at most 8 output rows.
__global__ void __launch_bounds__(kLutThreads)
    gf8_queue_kernel(const QueueUnit *units, const QueueCtl *ctl, QueueDev *dev, unsigned long long timeout_ns) {
  __shared__ __align__(16) LutShared sh;
  __shared__ QueueUnit s_unit;
  __shared__ int s_state;  // 0 run s_unit, 1 stop
  lut_init(sh);
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned long long u = atomicAdd(&dev->next, 1ull);
      const unsigned long long t0 = global_ns();
      unsigned int nap = 2000;  // ns between polls of host memory, doubling to 64 us
      int state = 0;
      for (;;) {
        // `closed` first: the host sets it after the last `published`, so once it is seen
        // the count read next is final.
        const unsigned int closed = ld_acquire_sys_u32(&ctl->closed);
        if (u < ld_acquire_sys(&ctl->published)) break;
        if (closed || atomicAdd(&dev->status, 0) != RS_OK) {
          state = 1;
          break;
        }
        if (global_ns() - t0 > timeout_ns) {
          atomicCAS(&dev->status, RS_OK, RS_ERR_TIMEOUT);
          state = 1;
          break;
        }
        __nanosleep(nap);
        nap = nap < 64000 ? 2 * nap : nap;
      }
      if (!state) s_unit = units[u];
      s_state = state;
    }
    __syncthreads();
    if (s_state) return;
    if (s_unit.item.rows <= 8)
      for (uint32_t b = s_unit.b0; b < s_unit.b1; b++) ragged_block_lut<8>(s_unit.item, b, sh);
    else
      for (uint32_t b = s_unit.b0; b < s_unit.b1; b++) ragged_block_lut<16>(s_unit.item, b, sh);
    __syncthreads();  // every thread is done with s_unit before thread 0 claims the next
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&dev->done, 1ull);
    }
  }
}

}  // namespace rsb

using namespace rsb;

struct rs_queue {
  int device = 0;
  size_t max_units = 0;
  unsigned long long timeout_ns = 0;
  QueueUnit *units_h = nullptr, *units_d = nullptr;
  QueueCtl *ctl_h = nullptr, *ctl_d = nullptr;
  QueueDev *dev = nullptr;
  DeviceBuf arena;  // coefficient rows and index lists of reconstruct units
  size_t arena_used = 0;
  unsigned long long published = 0;
  cudaStream_t stream = nullptr, aux = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool running = false;
  std::vector<std::shared_ptr<const Gen8>> gens;  // keeps generator tables alive
  std::mutex mu;
  ~rs_queue() {
    cudaSetDevice(device);
    if (running) {
      ctl_h->closed = 1;
      cudaStreamSynchronize(stream);
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (stream) cudaStreamDestroy(stream);
    if (aux) cudaStreamDestroy(aux);
    if (units_h) cudaFreeHost(units_h);
    if (ctl_h) cudaFreeHost(ctl_h);
    if (dev) cudaFree(dev);
  }
};

namespace rsb {

// Two 128-thread CTAs per SM (fewer if they do not fit): enough to keep the matrix
// work's loads in flight, while idle CTAs stay few, each polling host memory from one
// thread. The persistent launch must leave every SM room for the kernels that pushes
// enqueue while it runs (a new erasure pattern's plan kernel): three CTAs of this kernel
// take all of an SM's registers, and a push then waited for a plan kernel that could
// not start until the queue gave up.
static int queue_blocks() {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gf8_queue_kernel, kLutThreads, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return sm_count() * std::min(per_sm, 2);
}

}  // namespace rsb

extern "C" {

int rs_queue_create(size_t max_units, size_t arena_bytes, uint64_t timeout_ns, rs_queue_t **out) {
  if (!out || max_units == 0) return RS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int dev = 0;
  RSB_TRY(ensure_device(&dev));
  std::unique_ptr<rs_queue> q(new (std::nothrow) rs_queue());
  if (!q) return RS_ERR_ALLOC;
  q->device = dev;
  q->max_units = max_units;
  q->timeout_ns = timeout_ns ? timeout_ns : 1000000000ull;
  RSB_CU(cudaSetDevice(dev));
  RSB_CU(cudaHostAlloc(&q->units_h, max_units * sizeof(QueueUnit), cudaHostAllocMapped));
  RSB_CU(cudaHostAlloc(&q->ctl_h, sizeof(QueueCtl), cudaHostAllocMapped));
  RSB_CU(cudaHostGetDevicePointer((void **)&q->units_d, q->units_h, 0));
  RSB_CU(cudaHostGetDevicePointer((void **)&q->ctl_d, q->ctl_h, 0));
  RSB_CU(cudaMalloc(&q->dev, sizeof(QueueDev)));
  RSB_TRY(q->arena.ensure(arena_bytes ? arena_bytes : (64u << 20)));
  RSB_CU(cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking));
  RSB_CU(cudaStreamCreateWithFlags(&q->aux, cudaStreamNonBlocking));
  // The persistent launch, captured once; each session replays the graph.
  const int blocks = queue_blocks();
  RSB_CU(cudaStreamBeginCapture(q->stream, cudaStreamCaptureModeThreadLocal));
  gf8_queue_kernel<<<blocks, kLutThreads, 0, q->stream>>>(q->units_d, q->ctl_d, q->dev,
                                                                          q->timeout_ns);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(q->stream, &graph);
  if (e != cudaSuccess) {
    set_cuda_error(e, "cudaStreamEndCapture");
    return RS_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&q->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    set_cuda_error(e, "cudaGraphInstantiate");
    return RS_ERR_CUDA;
  }
  *out = q.release();
  return RS_OK;
}

int rs_queue_start(rs_queue_t *q) {
  if (!q) return RS_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(q->mu);
  if (q->running) return RS_ERR_INVALID_ARGUMENT;
  RSB_CU(cudaSetDevice(q->device));
  q->published = 0;
  q->arena_used = 0;
  q->gens.clear();
  std::memset(q->ctl_h, 0, sizeof(QueueCtl));
  std::atomic_thread_fence(std::memory_order_seq_cst);
  RSB_CU(cudaMemsetAsync(q->dev, 0, sizeof(QueueDev), q->stream));
  RSB_CU(cudaGraphLaunch(q->exec, q->stream));
  g_launches++;
  q->running = true;
  return RS_OK;
}

int rs_queue_push(rs_queue_t *q, const rs_batch_item *items, size_t n_items, int *statuses) {
  if (!q || (!items && n_items)) return RS_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(q->mu);
  if (!q->running) return RS_ERR_INVALID_ARGUMENT;
  RSB_CU(cudaSetDevice(q->device));
  struct Pending {
    RaggedItem item;
    size_t coef_off, rows_off;  // arena offsets (reconstruct), or SIZE_MAX
  };
  std::vector<Pending> pend;
  std::vector<uint8_t> host;  // arena image for this push, placed at q->arena_used
  auto put = [&](const void *p, size_t n) {
    size_t off = (host.size() + 255) & ~size_t(255);
    host.resize(off + n);
    std::memcpy(host.data() + off, p, n);
    return off;
  };
  size_t n_units = 0;
  for (size_t i = 0; i < n_items; i++) {
    const rs_batch_item &it = items[i];
    int st = RS_OK;
    if (!it.codec || !it.d_rows || it.op < 0 || it.op > 2 || it.codec->gen->device != q->device)
      st = RS_ERR_INVALID_ARGUMENT;
    else if (it.row_len == 0)
      st = RS_EMPTY_SHARD;
    else if (it.row_stride < it.row_len)
      st = RS_INCORRECT_SHARD_SIZE;
    if (st) {
      if (statuses) statuses[i] = st;
      continue;
    }
    const Gen8 &g = *it.codec->gen;
    const size_t k = g.k, n = g.k + g.m;
    RaggedItem r{};
    r.base = it.d_rows;
    r.row_stride = it.row_stride;
    r.len = it.row_len;
    r.k = (uint32_t)k;
    Pending pd{r, SIZE_MAX, SIZE_MAX};
    if (it.op == RS_BATCH_ENCODE) {
      pd.item.coeffs = g.d_rows;
      pd.item.rows = (uint32_t)g.m;
    } else {
      if (!it.present) {
        if (statuses) statuses[i] = RS_ERR_INVALID_ARGUMENT;
        continue;
      }
      Presence pres(n);
      size_t cnt = 0;
      for (size_t x = 0; x < n; x++)
        if (it.present[x]) {
          pres.set(x);
          cnt++;
        }
      if (cnt < k) {
        if (statuses) statuses[i] = RS_TOO_FEW_SHARDS_PRESENT;
        continue;
      }
      std::vector<uint32_t> surv, md, mp;
      split_pattern(pres, k, n, surv, md, mp);
      std::vector<size_t> nodes(surv.begin(), surv.end()), targets(md.begin(), md.end());
      if (it.op == RS_BATCH_RECONSTRUCT) targets.insert(targets.end(), mp.begin(), mp.end());
      if (cnt == n || targets.empty()) {
        if (statuses) statuses[i] = RS_OK;
        continue;
      }
      // Decode rows in closed form: the Lagrange basis on the survivor points evaluated
      // at each missing point (the reference's inverse-then-compose, src/reedsolomon.rs:
      // 550-585, as one matrix).
      std::vector<uint8_t> rows;
      lagrange_rows<F8>(nodes, targets, rows);
      std::vector<uint16_t> idx(k + targets.size());
      for (size_t t = 0; t < k; t++) idx[t] = (uint16_t)nodes[t];
      for (size_t t = 0; t < targets.size(); t++) idx[k + t] = (uint16_t)targets[t];
      pd.coef_off = put(rows.data(), rows.size());
      pd.rows_off = put(idx.data(), idx.size() * 2);
      pd.item.rows = (uint32_t)targets.size();
    }
    pd.item.col_tiles = (uint32_t)((it.row_len + kTileBytes - 1) / kTileBytes);
    const uint64_t blocks = (uint64_t)pd.item.col_tiles * ((pd.item.rows + kRowChunk - 1) / kRowChunk);
    n_units += (size_t)((blocks + kUnitBlocks - 1) / kUnitBlocks);
    pend.push_back(pd);
    if (statuses) statuses[i] = RS_OK;
  }
  if (q->published + n_units > q->max_units) return RS_ERR_TOO_LARGE;
  const size_t base_off = (q->arena_used + 255) & ~size_t(255);
  if (base_off + host.size() > q->arena.cap) return RS_ERR_TOO_LARGE;
  if (!host.empty()) {
    RSB_CU(cudaMemcpyAsync(q->arena.ptr + base_off, host.data(), host.size(), cudaMemcpyHostToDevice, q->aux));
    RSB_CU(cudaStreamSynchronize(q->aux));  // the rows are on the device before any unit names them
    q->arena_used = base_off + host.size();
  }
  unsigned long long u = q->published;
  for (Pending &pd : pend) {
    if (pd.coef_off != SIZE_MAX) {
      pd.item.coeffs = q->arena.ptr + base_off + pd.coef_off;
      pd.item.in_rows = reinterpret_cast<const uint16_t *>(q->arena.ptr + base_off + pd.rows_off);
      pd.item.out_rows = pd.item.in_rows + pd.item.k;
    }
    const uint32_t blocks = pd.item.col_tiles * ((pd.item.rows + kRowChunk - 1) / kRowChunk);
    for (uint32_t b0 = 0; b0 < blocks; b0 += kUnitBlocks) {
      QueueUnit &qu = q->units_h[u++];
      qu.item = pd.item;
      qu.b0 = b0;
      qu.b1 = std::min(blocks, b0 + kUnitBlocks);
    }
  }
  for (size_t i = 0; i < n_items; i++)
    if (items[i].codec && (!statuses || statuses[i] == RS_OK)) q->gens.push_back(items[i].codec->gen);
  // Descriptors first, then the count that publishes them.
  std::atomic_thread_fence(std::memory_order_release);
  reinterpret_cast<std::atomic<unsigned long long> *>(&q->ctl_h->published)->store(u, std::memory_order_release);
  q->published = u;
  return RS_OK;
}

int rs_queue_progress(rs_queue_t *q, uint64_t *done_units, uint64_t *published_units) {
  if (!q) return RS_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(q->mu);
  RSB_CU(cudaSetDevice(q->device));
  QueueDev d{};
  RSB_CU(cudaMemcpyAsync(&d, q->dev, sizeof d, cudaMemcpyDeviceToHost, q->aux));
  RSB_CU(cudaStreamSynchronize(q->aux));
  if (done_units) *done_units = d.done;
  if (published_units) *published_units = q->published;
  return RS_OK;
}

static int queue_end(rs_queue_t *q, bool close) {
  if (!q) return RS_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(q->mu);
  if (!q->running) return RS_ERR_INVALID_ARGUMENT;
  RSB_CU(cudaSetDevice(q->device));
  if (close) {
    std::atomic_thread_fence(std::memory_order_release);
    reinterpret_cast<std::atomic<unsigned int> *>(&q->ctl_h->closed)->store(1u, std::memory_order_release);
  }
  RSB_CU(cudaStreamSynchronize(q->stream));
  q->running = false;
  QueueDev d{};
  RSB_CU(cudaMemcpy(&d, q->dev, sizeof d, cudaMemcpyDeviceToHost));
  return d.status;
}

int rs_queue_finish(rs_queue_t *q) { return queue_end(q, true); }

int rs_queue_wait(rs_queue_t *q) { return queue_end(q, false); }

void rs_queue_free(rs_queue_t *q) { delete q; }

}  // extern "C"
