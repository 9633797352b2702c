// Instantiates the bitsliced FFT encode kernels for (K,K) with K = 128 (kernels_fft.cuh).
#include "kernels_fft.cuh"

namespace rsb {

RSB_FFT_DEFINE(128)

}  // namespace rsb
