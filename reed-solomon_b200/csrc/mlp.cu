// The learned cost model: a small FP32 MLP trained and served on the GPU by the
// kernels in this file (include/rs_b200.h, rs_mlp_*). It maps a workload's features
// (k, m, log shard bytes, erasures, batch; normalised by the caller) to one predicted
// log-time per candidate launch configuration; the tuner takes the argmin. It never
// touches payload bytes, so coded output stays bit-exact whatever it predicts.
//
// Layers: in -> H (ReLU) -> H (ReLU) -> H (ReLU) -> out. Loss: masked mean squared
// error over the measured (sample, configuration) pairs. Optimiser: Adam.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <random>
#include <vector>

#include "runtime.hpp"

namespace rsb {

constexpr int kMlpLayers = 4;

struct MlpShape {
  int dims[kMlpLayers + 1];  // in, h, h, h, out
  size_t w_off[kMlpLayers], b_off[kMlpLayers], total;
  void init(int in, int hidden, int out) {
    dims[0] = in;
    for (int l = 1; l < kMlpLayers; l++) dims[l] = hidden;
    dims[kMlpLayers] = out;
    size_t off = 0;
    for (int l = 0; l < kMlpLayers; l++) {
      w_off[l] = off;
      off += (size_t)dims[l + 1] * dims[l];
      b_off[l] = off;
      off += dims[l + 1];
    }
    total = off;
  }
};

// out[b, n] = act(sum_k in[b, k] * W[n, k] + bias[n])
static __global__ void mlp_linear_fwd(const float *in, const float *W, const float *bias, float *out, int B,
                                      int K, int N, int relu) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B * N) return;
  int b = t / N, n = t % N;
  const float *x = in + (size_t)b * K;
  const float *w = W + (size_t)n * K;
  float acc = bias[n];
  for (int k = 0; k < K; k++) acc = fmaf(x[k], w[k], acc);
  out[t] = relu ? fmaxf(acc, 0.f) : acc;
}

// Masked MSE: g = 2 * mask * (pred - y) / count; loss partial sums per block.
static __global__ void mlp_loss_grad(const float *pred, const float *y, const float *mask, float *g, int n,
                                     float inv_count, float *loss_acc) {
  __shared__ float part[256];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (t < n) {
    float d = (pred[t] - y[t]) * mask[t];
    g[t] = 2.f * d * inv_count;
    l = d * d * inv_count;
  }
  part[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss_acc, part[0]);
}

// dW[n, k] = sum_b gout[b, n] * in[b, k]; db[n] = sum_b gout[b, n] (column k == K).
static __global__ void mlp_linear_bwd_w(const float *in, const float *gout, float *dW, float *db, int B, int K,
                                        int N) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N * (K + 1)) return;
  int n = t / (K + 1), k = t % (K + 1);
  float acc = 0.f;
  if (k < K) {
    for (int b = 0; b < B; b++) acc = fmaf(gout[(size_t)b * N + n], in[(size_t)b * K + k], acc);
    dW[(size_t)n * K + k] = acc;
  } else {
    for (int b = 0; b < B; b++) acc += gout[(size_t)b * N + n];
    db[n] = acc;
  }
}

// gin[b, k] = (sum_n gout[b, n] * W[n, k]) * (act_in[b, k] > 0) for a ReLU input.
static __global__ void mlp_linear_bwd_x(const float *gout, const float *W, const float *act_in, float *gin,
                                        int B, int K, int N) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B * K) return;
  int b = t / K, k = t % K;
  float acc = 0.f;
  for (int n = 0; n < N; n++) acc = fmaf(gout[(size_t)b * N + n], W[(size_t)n * K + k], acc);
  gin[t] = act_in[t] > 0.f ? acc : 0.f;
}

static __global__ void mlp_adam(float *p, const float *g, float *m1, float *m2, size_t n, float lr, float b1,
                                float b2, float eps, float c1, float c2) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float gi = g[t];
  float a = b1 * m1[t] + (1.f - b1) * gi;
  float v = b2 * m2[t] + (1.f - b2) * gi * gi;
  m1[t] = a;
  m2[t] = v;
  p[t] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

}  // namespace rsb

using namespace rsb;

struct rs_mlp {
  std::mutex mu;  // predict and training share the work buffers
  int device = 0;
  MlpShape shape;
  float *params = nullptr, *grads = nullptr, *m1 = nullptr, *m2 = nullptr;
  float *work = nullptr;  // activations and gradients
  size_t work_cap = 0;
  int steps = 0;
  cudaStream_t stream = nullptr;
  ~rs_mlp() {
    cudaSetDevice(device);
    cudaFree(params);
    cudaFree(grads);
    cudaFree(m1);
    cudaFree(m2);
    cudaFree(work);
    if (stream) cudaStreamDestroy(stream);
  }
  // activations a[0] = x (copied), a[1..L] layer outputs; gradient buffers alike
  int ensure(int B) {
    size_t per = 0;
    for (int l = 0; l <= kMlpLayers; l++) per += shape.dims[l];
    size_t need = 2 * per * (size_t)B + 1;
    if (need <= work_cap) return RS_OK;
    if (work) cudaFree(work);
    work = nullptr;
    RSB_CU(cudaMalloc(&work, need * sizeof(float)));
    work_cap = need;
    return RS_OK;
  }
  float *act(int l, int B) {
    size_t off = 0;
    for (int i = 0; i < l; i++) off += (size_t)shape.dims[i] * B;
    return work + off;
  }
  float *grad_act(int l, int B) {
    size_t per = 0;
    for (int i = 0; i <= kMlpLayers; i++) per += shape.dims[i];
    size_t off = per * B;
    for (int i = 0; i < l; i++) off += (size_t)shape.dims[i] * B;
    return work + off;
  }
  float *loss_slot() { return work + work_cap - 1; }
};

namespace rsb {

static int mlp_forward(rs_mlp *m, const float *d_x, int B) {
  RSB_TRY(m->ensure(B));
  cudaStream_t st = m->stream;
  RSB_CU(cudaMemcpyAsync(m->act(0, B), d_x, sizeof(float) * B * m->shape.dims[0], cudaMemcpyDeviceToDevice, st));
  for (int l = 0; l < kMlpLayers; l++) {
    int K = m->shape.dims[l], N = m->shape.dims[l + 1];
    int n = B * N;
    mlp_linear_fwd<<<(n + 255) / 256, 256, 0, st>>>(m->act(l, B), m->params + m->shape.w_off[l],
                                                    m->params + m->shape.b_off[l], m->act(l + 1, B), B, K, N,
                                                    l + 1 < kMlpLayers);
    g_launches++;
  }
  RSB_CU(cudaGetLastError());
  return RS_OK;
}

static int mlp_backward(rs_mlp *m, const float *d_y, const float *d_mask, int B, float count) {
  cudaStream_t st = m->stream;
  const int L = kMlpLayers, out = m->shape.dims[L];
  RSB_CU(cudaMemsetAsync(m->loss_slot(), 0, sizeof(float), st));
  int n = B * out;
  mlp_loss_grad<<<(n + 255) / 256, 256, 0, st>>>(m->act(L, B), d_y, d_mask, m->grad_act(L, B), n,
                                                 1.f / std::max(count, 1.f), m->loss_slot());
  g_launches++;
  for (int l = L - 1; l >= 0; l--) {
    int K = m->shape.dims[l], N = m->shape.dims[l + 1];
    int nw = N * (K + 1);
    mlp_linear_bwd_w<<<(nw + 255) / 256, 256, 0, st>>>(m->act(l, B), m->grad_act(l + 1, B),
                                                       m->grads + m->shape.w_off[l], m->grads + m->shape.b_off[l],
                                                       B, K, N);
    g_launches++;
    if (l > 0) {
      int nx = B * K;
      mlp_linear_bwd_x<<<(nx + 255) / 256, 256, 0, st>>>(m->grad_act(l + 1, B), m->params + m->shape.w_off[l],
                                                         m->act(l, B), m->grad_act(l, B), B, K, N);
      g_launches++;
    }
  }
  RSB_CU(cudaGetLastError());
  return RS_OK;
}

}  // namespace rsb

extern "C" {

int rs_mlp_create(int n_in, int hidden, int n_out, uint64_t seed, rs_mlp_t **out) {
  if (!out || n_in <= 0 || hidden <= 0 || n_out <= 0) return RS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int dev = 0;
  RSB_TRY(ensure_device(&dev));
  rs_mlp *m = new (std::nothrow) rs_mlp();
  if (!m) return RS_ERR_ALLOC;
  m->device = dev;
  m->shape.init(n_in, hidden, n_out);
  size_t n = m->shape.total;
  std::vector<float> host(n, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < kMlpLayers; l++) {  // He initialisation, zero biases
    int K = m->shape.dims[l], N = m->shape.dims[l + 1];
    std::normal_distribution<float> dist(0.f, std::sqrt(2.f / K));
    for (size_t i = 0; i < (size_t)N * K; i++) host[m->shape.w_off[l] + i] = dist(rng);
  }
  int st = RS_OK;
  if (cudaMalloc(&m->params, n * 4) != cudaSuccess || cudaMalloc(&m->grads, n * 4) != cudaSuccess ||
      cudaMalloc(&m->m1, n * 4) != cudaSuccess || cudaMalloc(&m->m2, n * 4) != cudaSuccess ||
      cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
    st = RS_ERR_ALLOC;
  if (!st && (cudaMemcpy(m->params, host.data(), n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
              cudaMemset(m->m1, 0, n * 4) != cudaSuccess || cudaMemset(m->m2, 0, n * 4) != cudaSuccess ||
              cudaMemset(m->grads, 0, n * 4) != cudaSuccess))
    st = RS_ERR_CUDA;
  if (st) {
    cudaGetLastError();
    delete m;
    return st;
  }
  *out = m;
  return RS_OK;
}

void rs_mlp_free(rs_mlp_t *m) { delete m; }

size_t rs_mlp_param_count(const rs_mlp_t *m) { return m ? m->shape.total : 0; }

int rs_mlp_get_params(const rs_mlp_t *m, float *out, size_t n) {
  if (!m || !out || n != m->shape.total) return RS_ERR_INVALID_ARGUMENT;
  RSB_CU(cudaSetDevice(m->device));
  RSB_CU(cudaMemcpy(out, m->params, n * 4, cudaMemcpyDeviceToHost));
  return RS_OK;
}

int rs_mlp_set_params(rs_mlp_t *m, const float *in, size_t n) {
  if (!m || !in || n != m->shape.total) return RS_ERR_INVALID_ARGUMENT;
  RSB_CU(cudaSetDevice(m->device));
  RSB_CU(cudaMemcpy(m->params, in, n * 4, cudaMemcpyHostToDevice));
  return RS_OK;
}

int rs_mlp_dims(const rs_mlp_t *m, int *n_in, int *hidden, int *n_out) {
  if (!m) return RS_ERR_INVALID_ARGUMENT;
  if (n_in) *n_in = m->shape.dims[0];
  if (hidden) *hidden = m->shape.dims[1];
  if (n_out) *n_out = m->shape.dims[kMlpLayers];
  return RS_OK;
}

// File: 8-byte magic "RSMLP\0\0\1", then int32 n_in, hidden, n_out, then the parameters
// as little-endian float32 in parameter order.
static const char kMlpMagic[8] = {'R', 'S', 'M', 'L', 'P', 0, 0, 1};

int rs_mlp_save(const rs_mlp_t *m, const char *path) {
  if (!m || !path) return RS_ERR_INVALID_ARGUMENT;
  std::vector<float> p(m->shape.total);
  RSB_TRY(rs_mlp_get_params(m, p.data(), p.size()));
  FILE *f = fopen(path, "wb");
  if (!f) return RS_ERR_INVALID_ARGUMENT;
  const int32_t dims[3] = {m->shape.dims[0], m->shape.dims[1], m->shape.dims[kMlpLayers]};
  bool ok = fwrite(kMlpMagic, 1, 8, f) == 8 && fwrite(dims, 4, 3, f) == 3 &&
            fwrite(p.data(), 4, p.size(), f) == p.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? RS_OK : RS_ERR_INVALID_ARGUMENT;
}

int rs_mlp_load(const char *path, rs_mlp_t **out) {
  if (!path || !out) return RS_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  FILE *f = fopen(path, "rb");
  if (!f) return RS_ERR_INVALID_ARGUMENT;
  char magic[8];
  int32_t dims[3];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, kMlpMagic, 8) != 0 || fread(dims, 4, 3, f) != 3 ||
      dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0 || dims[0] > 4096 || dims[1] > 4096 || dims[2] > 4096) {
    fclose(f);
    return RS_ERR_INVALID_ARGUMENT;
  }
  rs_mlp_t *m = nullptr;
  int st = rs_mlp_create(dims[0], dims[1], dims[2], 0, &m);
  if (st) {
    fclose(f);
    return st;
  }
  std::vector<float> p(m->shape.total);
  const bool ok = fread(p.data(), 4, p.size(), f) == p.size();
  fclose(f);
  if (!ok || (st = rs_mlp_set_params(m, p.data(), p.size())) != RS_OK) {
    delete m;
    return ok ? st : RS_ERR_INVALID_ARGUMENT;
  }
  *out = m;
  return RS_OK;
}

int rs_mlp_predict(rs_mlp_t *m, const float *d_x, int batch, float *d_out) {
  if (!m || !d_x || !d_out || batch <= 0) return RS_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(m->mu);
  RSB_CU(cudaSetDevice(m->device));
  RSB_TRY(mlp_forward(m, d_x, batch));
  RSB_CU(cudaMemcpyAsync(d_out, m->act(kMlpLayers, batch), sizeof(float) * batch * m->shape.dims[kMlpLayers],
                         cudaMemcpyDeviceToDevice, m->stream));
  RSB_CU(cudaStreamSynchronize(m->stream));
  return RS_OK;
}

int rs_mlp_gradients(rs_mlp_t *m, const float *d_x, const float *d_y, const float *d_mask, int batch,
                     float mask_count, float *grads_out, size_t n, float *loss) {
  if (!m || !d_x || !d_y || !d_mask || batch <= 0) return RS_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(m->mu);
  RSB_CU(cudaSetDevice(m->device));
  RSB_TRY(mlp_forward(m, d_x, batch));
  RSB_TRY(mlp_backward(m, d_y, d_mask, batch, mask_count));
  if (grads_out) {
    if (n != m->shape.total) return RS_ERR_INVALID_ARGUMENT;
    RSB_CU(cudaMemcpyAsync(grads_out, m->grads, n * 4, cudaMemcpyDeviceToHost, m->stream));
  }
  float l = 0.f;
  RSB_CU(cudaMemcpyAsync(&l, m->loss_slot(), 4, cudaMemcpyDeviceToHost, m->stream));
  RSB_CU(cudaStreamSynchronize(m->stream));
  if (loss) *loss = l;
  return RS_OK;
}

int rs_mlp_train_step(rs_mlp_t *m, const float *d_x, const float *d_y, const float *d_mask, int batch,
                      float mask_count, float lr, float *loss) {
  if (!m || !d_x || !d_y || !d_mask || batch <= 0) return RS_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(m->mu);
  RSB_CU(cudaSetDevice(m->device));
  RSB_TRY(mlp_forward(m, d_x, batch));
  RSB_TRY(mlp_backward(m, d_y, d_mask, batch, mask_count));
  m->steps++;
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1.f - std::pow(b1, (float)m->steps), c2 = 1.f - std::pow(b2, (float)m->steps);
  size_t n = m->shape.total;
  mlp_adam<<<(unsigned)((n + 255) / 256), 256, 0, m->stream>>>(m->params, m->grads, m->m1, m->m2, n, lr, b1, b2,
                                                              1e-8f, c1, c2);
  g_launches++;
  RSB_CU(cudaGetLastError());
  if (loss) {
    RSB_CU(cudaMemcpyAsync(loss, m->loss_slot(), 4, cudaMemcpyDeviceToHost, m->stream));
    RSB_CU(cudaStreamSynchronize(m->stream));
  }
  return RS_OK;
}

}  // extern "C"
