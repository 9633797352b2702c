// Instantiates the bitsliced FFT encode kernels for (K,K) with K = 64 (kernels_fft.cuh).
#include "kernels_fft.cuh"

namespace rsb {

RSB_FFT_DEFINE(64)

}  // namespace rsb
