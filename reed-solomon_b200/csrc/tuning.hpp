// Launch configurations that the autotuner times and the cost model chooses among, and
// the features the model reads. Configurations choose kernels and launch shapes only,
// never arithmetic: every one yields the same bytes.
#pragma once

#include <cmath>
#include <cstddef>

namespace rsb {

enum TuneRoute { kTuneMatrix = 0, kTuneFft = 1, kTuneGen = 2 };

struct TuneConfig {
  int route;  // TuneRoute
  int p0;     // matrix: tile variant; FFT: lane-group width (0 narrow, 1 wide)
  int p1;     // FFT: launch shape (index into kFftVariants)
};

// The order is the cost model's output order (reed-solomon_b200/tuner.py CONFIGS).
constexpr TuneConfig kTuneConfigs[] = {
    {kTuneMatrix, 0, 0}, {kTuneMatrix, 1, 0}, {kTuneMatrix, 2, 0}, {kTuneMatrix, 3, 0},
    {kTuneFft, 0, 0},    {kTuneFft, 0, 1},    {kTuneFft, 1, 0},    {kTuneFft, 1, 1},
    {kTuneFft, 0, 2},    {kTuneFft, 1, 2},    {kTuneFft, 0, 3},    {kTuneFft, 1, 3},
    {kTuneGen, 0, 0}};
constexpr int kTuneConfigCount = sizeof(kTuneConfigs) / sizeof(kTuneConfigs[0]);
constexpr int kTuneFeatures = 6;
// The autotuner times launches of 1 .. 512 stripes of at most 64 MiB in all; a larger
// launch group is scored as the largest launch of its stripes inside that envelope
// (tune_batch), where the kernels already fill the GPU, instead of extrapolating.
constexpr size_t kTuneMaxBatch = 512;
constexpr size_t kTuneMaxLaunchBytes = 64u << 20;

inline size_t tune_batch(size_t k, size_t m, size_t shard_bytes, size_t stripes) {
  const size_t per = (k + m) * (shard_bytes ? shard_bytes : 1);
  size_t fit = kTuneMaxLaunchBytes / per;
  fit = fit < 1 ? 1 : fit > kTuneMaxBatch ? kTuneMaxBatch : fit;
  return stripes < fit ? (stripes ? stripes : 1) : fit;
}

// Features of one launch of `batch` stripes of (k, m) with shard_bytes-byte rows,
// `erasures` rebuilt per stripe (0: encode), rows 16-byte aligned or not.
inline void tune_features(size_t k, size_t m, size_t shard_bytes, size_t erasures, size_t batch, bool aligned,
                          float *out) {
  out[0] = (float)(std::log2((double)k) / 8.0);
  out[1] = (float)(std::log2((double)m) / 8.0);
  out[2] = (float)(std::log2((double)shard_bytes) / 20.0);
  out[3] = (float)((double)erasures / (double)(m ? m : 1));
  batch = batch < 1 ? 1 : batch > kTuneMaxBatch ? kTuneMaxBatch : batch;
  out[4] = (float)(std::log2((double)batch) / 8.0);
  out[5] = aligned ? 0.f : 1.f;
}

}  // namespace rsb
