// rs8_reconstruct_batch_noalloc: batched reconstruct that allocates nothing.
//
// Some callers cannot allocate device memory while they run: a latency-critical path
// that must not stall on the allocator, a process whose memory budget was fixed when
// it started, or a host whose device allocator belongs to another framework. For them
// this entry point keeps all of its working memory (the per-stripe survivor and
// target lists, the decode rows and the plan statuses) in one fixed file-scope device
// array, and stages its index lists through one fixed file-scope host buffer. It
// calls no cudaMalloc, cudaFree or allocating library routine.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "codec8.hpp"
#include "kernels_matrix.cuh"
#include "kernels_plan.cuh"
#include "runtime.hpp"

namespace rsb {

// Working area shared by every call in the process. Every GPU that loads this library
// holds it until the process exits.
constexpr size_t kNoAllocScratchBytes = 8u << 20;
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

// Host staging of the index lists, copied into the device area on each call.
static uint8_t g_noalloc_host[kNoAllocScratchBytes];
static std::mutex g_noalloc_mu;

// Device address of g_noalloc_scratch per device. In host code the array's name is
// only a host-side stand-in, so the address is looked up with cudaGetSymbolAddress,
// once per device, with that device current (on the first call there). With CUDA's
// lazy module loading that first lookup is also when this file's device module is
// loaded, which is when the 8 MiB array is reserved on the device: the first call on
// a device therefore does take device memory, once, and fails with RS_ERR_CUDA if the
// device has no 8 MiB left. Later calls take none.
constexpr int kMaxDevices = 64;
static void *g_noalloc_dev_ptr[kMaxDevices];

static int noalloc_scratch(int device, uint8_t **out) {
  if (device < 0 || device >= kMaxDevices) return RS_ERR_INVALID_ARGUMENT;
  if (!g_noalloc_dev_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
      return RS_ERR_CUDA;
    }
    g_noalloc_dev_ptr[device] = p;
  }
  *out = static_cast<uint8_t *>(g_noalloc_dev_ptr[device]);
  return RS_OK;
}

static size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// Upper bound on the stripes one call can take: every stripe needs k*m + 2*(k+m) + 8
// bytes of the working area, so any count above this is rejected before the layout's
// products are formed (they could otherwise wrap around on 64-bit sizes).
static size_t noalloc_max_stripes(size_t k, size_t m) {
  return kNoAllocScratchBytes / (k * m + 2 * (k + m) + 8);
}

}  // namespace rsb

using namespace rsb;

extern "C" {

size_t rs8_reconstruct_batch_noalloc_limit(size_t k, size_t m, size_t n_stripes) {
  // A stripe count that could not fit even one byte of working memory per entry is
  // reported as "more than any size" instead of a product that wraps around.
  if (n_stripes > noalloc_max_stripes(k, m)) return SIZE_MAX;
  return up256(n_stripes * k * 2) + up256(n_stripes * m * 2) + up256(n_stripes * 2) + up256(n_stripes * m * k) +
         up256(n_stripes * sizeof(int));
}

int rs8_reconstruct_batch_noalloc(rs8_t *c, uint8_t *d_rows, size_t stripe_stride, size_t n_stripes, size_t row_len,
                                  const uint8_t *present, int data_only, int *statuses, void *stream) {
  if (!c || !present) return RS_ERR_INVALID_ARGUMENT;
  if (n_stripes == 0) return RS_OK;
  if (row_len == 0) return RS_EMPTY_SHARD;
  if (!d_rows) return RS_ERR_INVALID_ARGUMENT;
  const Gen8 &g = *c->gen;
  const size_t k = g.k, m = g.m, n = k + m;
  if (n_stripes > noalloc_max_stripes(k, m)) return RS_ERR_TOO_LARGE;
  // Working-area layout: survivors | targets | target counts | decode rows | statuses.
  const size_t o_targ = up256(n_stripes * k * 2), o_nt = o_targ + up256(n_stripes * m * 2);
  const size_t o_rows = o_nt + up256(n_stripes * 2), o_stat = o_rows + up256(n_stripes * m * k);
  const size_t need = o_stat + up256(n_stripes * sizeof(int));
  if (need > kNoAllocScratchBytes) return RS_ERR_TOO_LARGE;
  cudaStream_t st = (cudaStream_t)stream;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  RSB_CU(cudaSetDevice(g.device));
  // The index lists are copied from g_noalloc_host, which the next call overwrites. A
  // copy recorded into a graph would read that buffer only when the graph runs, by
  // which time it may hold another call's lists, so a stream that is capturing is
  // refused.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  RSB_CU(cudaStreamIsCapturing(st, &cap));
  if (cap != cudaStreamCaptureStatusNone) return RS_ERR_INVALID_ARGUMENT;
  uint8_t *base = nullptr;
  RSB_TRY(noalloc_scratch(g.device, &base));
  uint16_t *surv = reinterpret_cast<uint16_t *>(g_noalloc_host);
  uint16_t *targ = reinterpret_cast<uint16_t *>(g_noalloc_host + o_targ);
  uint16_t *ntarg = reinterpret_cast<uint16_t *>(g_noalloc_host + o_nt);
  // Survivors are the first k present rows; targets the missing data rows, then
  // (unless data_only) the missing parity rows (src/reedsolomon.rs:550-566). Every
  // entry the kernels read is written here on each call, so nothing left over from
  // an earlier call is used.
  size_t live = 0;
  for (size_t s = 0; s < n_stripes; s++) {
    const uint8_t *p = present + s * n;
    size_t cnt = 0, ns = 0, nt = 0;
    for (size_t i = 0; i < n; i++) cnt += p[i] ? 1 : 0;
    const int status = cnt < k ? RS_TOO_FEW_SHARDS_PRESENT : RS_OK;
    if (cnt == n || cnt < k) {
      for (size_t t = 0; t < k; t++) surv[s * k + t] = (uint16_t)t;
    } else {
      for (size_t i = 0; i < n; i++) {
        if (p[i]) {
          if (ns < k) surv[s * k + ns++] = (uint16_t)i;
        } else if (i < k) {
          targ[s * m + nt++] = (uint16_t)i;
        }
      }
      if (!data_only)
        for (size_t i = k; i < n; i++)
          if (!p[i]) targ[s * m + nt++] = (uint16_t)i;
    }
    ntarg[s] = (uint16_t)nt;
    live += nt ? 1 : 0;
    if (statuses) statuses[s] = status;
  }
  if (!live) return RS_OK;
  RSB_CU(cudaMemcpyAsync(base, g_noalloc_host, o_rows, cudaMemcpyHostToDevice, st));
  PlanArgs pa{};
  pa.gen = g.d_rows;
  pa.k = (uint32_t)k;
  pa.m = (uint32_t)m;
  pa.survivors = reinterpret_cast<const uint16_t *>(base);
  pa.targets = reinterpret_cast<const uint16_t *>(base + o_targ);
  pa.n_targets = reinterpret_cast<const uint16_t *>(base + o_nt);
  pa.max_rows = (uint32_t)m;
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
  a.coeff_stripe_stride = (uint64_t)m * k;
  a.rows_per_stripe = pa.n_targets;
  a.in_map = pa.survivors;
  a.out_map = pa.targets;
  a.k = (uint32_t)k;
  a.rows = (uint32_t)m;
  a.len = row_len;
  a.n_stripes = (uint32_t)n_stripes;
  return launch_gf8(a, nullptr, false, st);
}

}  // extern "C"
