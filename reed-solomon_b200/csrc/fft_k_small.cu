// Instantiates the bitsliced FFT encode kernels for (K,K) with K = 2, 4, 8 (kernels_fft.cuh).
#include "kernels_fft.cuh"

namespace rsb {

RSB_FFT_DEFINE(2)
RSB_FFT_DEFINE(4)
RSB_FFT_DEFINE(8)

}  // namespace rsb
