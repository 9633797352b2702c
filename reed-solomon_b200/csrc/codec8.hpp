// The GF(2^8) codec and decoder handles behind rs8_t / rs8_dec_t, shared by the
// single-stripe entry points (rs_abi.cu) and the mixed batches (rs_batch.cu).
#pragma once

#include <atomic>
#include <memory>
#include <vector>

#include "kernels_fft.cuh"
#include "kernels_matrix.cuh"
#include "runtime.hpp"

namespace rsb {

// Systematic generator of one (k, m) shape, resident on `device`.
struct Gen8 {
  int device = 0;
  size_t k = 0, m = 0;
  std::vector<uint8_t> rows;  // parity rows, m x k
  uint8_t *d_rows = nullptr;
  const FftShape *fft = nullptr;  // bitsliced FFT kernel for this shape, if any
  ~Gen8() {
    if (d_rows) {
      cudaSetDevice(device);
      cudaFree(d_rows);
    }
  }
};

}  // namespace rsb

struct rs8_codec {
  std::shared_ptr<const rsb::Gen8> gen;
  std::shared_ptr<rsb::PlanCache> plans;
  std::shared_ptr<rsb::Exec> exec;
  std::atomic<int> route{0};  // 0 automatic, 1 matrix, 2 FFT where available
};

struct rs8_decoder {
  std::shared_ptr<const rsb::Gen8> gen;
  std::shared_ptr<const rsb::Plan> plan;
  std::shared_ptr<rsb::Exec> exec;
};

namespace rsb {

bool use_fft8(const rs8_codec *c, size_t len);
// Whether regenerating `missing_parity` parity rows with the shape's compiled kernel
// beats applying them on the matrix route (route 2 forces it).
bool regen_parity_pays(const Gen8 &g, size_t missing_parity, int route);
int encode8_strided(rs8_codec *c, const uint8_t *in_base, uint64_t in_row, uint64_t in_stripe, uint8_t *out_base,
                    uint64_t out_row, uint64_t out_stripe, size_t n_stripes, size_t len, cudaStream_t st);
int launch_gf8(const ApplyArgs &a, const PtrTable *pt, bool verify, cudaStream_t st);

}  // namespace rsb
