// Payload framing on either side of the coder: the steps the reference crate's callers
// take to turn a byte payload into stripes of shards and back.
//
// * Shred-style FEC sets (the reference's Agave test shape, RS(32,32) x 987-byte shards,
//   src/reedsolomon.rs:973): a payload is cut into fixed-size data shards, k per stripe,
//   every stripe is encoded, and a receiver that holds any k shards of a stripe rebuilds
//   its data shards and reassembles the payload.
// * The tape outer coder (benches/gf16-bench/src/bin/live.rs:1-16): a segment is cut into
//   k = ceil(groups / 3) data shards of ceil(segment_len / k) bytes rounded up to 64 (at
//   most 4 MiB) and coded with ReedSolomon16(k, groups - k).
//
// Layout. Byte p of the payload goes to stripe p / (k * shard_len), data shard
// (p / shard_len) % k, offset p % shard_len; the bytes after the payload in the last
// stripe are zero. Stripes are stored [stripe][k + m rows][shard_len] in device memory,
// so the k data rows of a stripe are k * shard_len consecutive payload bytes: splitting
// is one pitched copy, reassembly another, and the coding runs on the batched kernels.
#include <cuda_runtime.h>

#include <vector>

#include "rs_b200.h"
#include "runtime.hpp"

namespace rsb {
namespace {

constexpr size_t kOuterMaxShard = 4u << 20;  // the outer coder's largest shard

int frame_check(size_t k, size_t payload_len, size_t shard_len, size_t n_stripes) {
  if (shard_len == 0) return RS_EMPTY_SHARD;
  if (n_stripes != rs_frame_stripe_count(payload_len, k, shard_len)) return RS_INCORRECT_SHARD_SIZE;
  return RS_OK;
}

// Payload -> the data rows of every stripe, zeros after the payload.
int frame_split(const uint8_t *d_payload, size_t payload_len, size_t k, size_t n, size_t shard_len,
                uint8_t *d_stripes, size_t n_stripes, cudaStream_t st) {
  const size_t data_bytes = k * shard_len, stripe_bytes = n * shard_len;
  const size_t full = payload_len / data_bytes, rest = payload_len - full * data_bytes;
  if (full)
    RSB_CU(cudaMemcpy2DAsync(d_stripes, stripe_bytes, d_payload, data_bytes, data_bytes, full,
                             cudaMemcpyDeviceToDevice, st));
  if (full < n_stripes) {  // the last stripe: the payload's tail, then zeros
    uint8_t *last = d_stripes + full * stripe_bytes;
    if (rest) RSB_CU(cudaMemcpyAsync(last, d_payload + full * data_bytes, rest, cudaMemcpyDeviceToDevice, st));
    RSB_CU(cudaMemsetAsync(last + rest, 0, data_bytes - rest, st));
  }
  return RS_OK;
}

// The data rows of every stripe -> the payload.
int frame_join(const uint8_t *d_stripes, size_t k, size_t n, size_t shard_len, uint8_t *d_payload,
               size_t payload_len, cudaStream_t st) {
  const size_t data_bytes = k * shard_len, stripe_bytes = n * shard_len;
  const size_t full = payload_len / data_bytes, rest = payload_len - full * data_bytes;
  if (full)
    RSB_CU(cudaMemcpy2DAsync(d_payload, data_bytes, d_stripes, stripe_bytes, data_bytes, full,
                             cudaMemcpyDeviceToDevice, st));
  if (rest)
    RSB_CU(cudaMemcpyAsync(d_payload + full * data_bytes, d_stripes + full * stripe_bytes, rest,
                           cudaMemcpyDeviceToDevice, st));
  return RS_OK;
}

int first_error(const std::vector<int> &st, int *out) {
  int first = RS_OK;
  for (size_t s = 0; s < st.size(); s++) {
    if (out) out[s] = st[s];
    if (!first && st[s]) first = st[s];
  }
  return first;
}

}  // namespace
}  // namespace rsb

using namespace rsb;

extern "C" {

size_t rs_frame_stripe_count(size_t payload_len, size_t data_shards, size_t shard_len) {
  if (data_shards == 0 || shard_len == 0) return 0;
  const size_t per = data_shards * shard_len;
  return payload_len / per + (payload_len % per ? 1 : 0);
}

int rs8_frame_encode_dev(rs8_t *c, const uint8_t *d_payload, size_t payload_len, size_t shard_len,
                         uint8_t *d_stripes, size_t n_stripes, void *stream) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  const size_t k = rs8_data_shard_count(c), n = rs8_total_shard_count(c);
  RSB_TRY(frame_check(k, payload_len, shard_len, n_stripes));
  if (n_stripes == 0) return RS_OK;
  if (!d_payload || !d_stripes) return RS_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  RSB_TRY(frame_split(d_payload, payload_len, k, n, shard_len, d_stripes, n_stripes, st));
  return rs8_encode_batch_dev(c, d_stripes, n * shard_len, d_stripes + k * shard_len, n * shard_len, n_stripes,
                              shard_len, stream);
}

int rs8_frame_decode_dev(rs8_t *c, uint8_t *d_stripes, size_t n_stripes, size_t shard_len, const uint8_t *present,
                         uint8_t *d_payload, size_t payload_len, int *statuses, void *stream) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  const size_t k = rs8_data_shard_count(c), n = rs8_total_shard_count(c);
  RSB_TRY(frame_check(k, payload_len, shard_len, n_stripes));
  if (n_stripes == 0) return RS_OK;
  if (!d_payload || !d_stripes || !present) return RS_ERR_INVALID_ARGUMENT;
  std::vector<int> st(n_stripes, 0);
  RSB_TRY(rs8_reconstruct_batch_dev(c, d_stripes, n * shard_len, n_stripes, shard_len, present, 1, st.data(),
                                    stream));
  RSB_TRY(frame_join(d_stripes, k, n, shard_len, d_payload, payload_len, (cudaStream_t)stream));
  return first_error(st, statuses);
}

int rs16_frame_encode_dev(rs16_t *c, const uint8_t *d_payload, size_t payload_len, size_t shard_len,
                          uint8_t *d_stripes, size_t n_stripes, void *stream) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  const size_t k = rs16_data_shard_count(c), n = rs16_total_shard_count(c);
  RSB_TRY(frame_check(k, payload_len, shard_len, n_stripes));
  if (shard_len % 2) return RS_INCORRECT_SHARD_SIZE;  // even shards (src/reedsolomon16.rs:758-772)
  if (n_stripes == 0) return RS_OK;
  if (!d_payload || !d_stripes) return RS_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  RSB_TRY(frame_split(d_payload, payload_len, k, n, shard_len, d_stripes, n_stripes, st));
  return rs16_encode_batch_dev(c, d_stripes, n * shard_len, d_stripes + k * shard_len, n * shard_len, n_stripes,
                               shard_len, stream);
}

int rs16_frame_decode_dev(rs16_t *c, uint8_t *d_stripes, size_t n_stripes, size_t shard_len, const uint8_t *present,
                          uint8_t *d_payload, size_t payload_len, int *statuses, void *stream) {
  if (!c) return RS_ERR_INVALID_ARGUMENT;
  const size_t k = rs16_data_shard_count(c), n = rs16_total_shard_count(c);
  RSB_TRY(frame_check(k, payload_len, shard_len, n_stripes));
  if (shard_len % 2) return RS_INCORRECT_SHARD_SIZE;
  if (n_stripes == 0) return RS_OK;
  if (!d_payload || !d_stripes || !present) return RS_ERR_INVALID_ARGUMENT;
  std::vector<int> st(n_stripes, 0);
  std::vector<uint8_t *> rows(n);
  std::vector<size_t> lens(n, shard_len);
  for (size_t s = 0; s < n_stripes; s++) {
    for (size_t i = 0; i < n; i++) rows[i] = d_stripes + (s * n + i) * shard_len;
    st[s] = rs16_reconstruct_dev(c, rows.data(), lens.data(), present + s * n, n, 1, stream);
    if (st[s] >= 100) return st[s];  // a device error ends the call; shard errors are per stripe
  }
  RSB_TRY(frame_join(d_stripes, k, n, shard_len, d_payload, payload_len, (cudaStream_t)stream));
  return first_error(st, statuses);
}

int rs_outer_shape(size_t groups, size_t *data_shards, size_t *parity_shards) {
  if (!data_shards || !parity_shards) return RS_ERR_INVALID_ARGUMENT;
  const size_t k = (groups + 2) / 3, m = groups - k;
  if (k == 0) return RS_TOO_FEW_DATA_SHARDS;
  if (m == 0) return RS_TOO_FEW_PARITY_SHARDS;
  if (groups > 65536) return RS_TOO_MANY_SHARDS;
  *data_shards = k;
  *parity_shards = m;
  return RS_OK;
}

int rs_outer_shard_bytes(size_t segment_len, size_t data_shards, size_t *shard_bytes) {
  if (!shard_bytes) return RS_ERR_INVALID_ARGUMENT;
  if (data_shards == 0) return RS_TOO_FEW_DATA_SHARDS;
  size_t s = segment_len / data_shards + (segment_len % data_shards ? 1 : 0);
  s = s < 64 ? 64 : (s + 63) & ~size_t(63);
  if (s > kOuterMaxShard) return RS_ERR_TOO_LARGE;
  *shard_bytes = s;
  return RS_OK;
}

}  // extern "C"
