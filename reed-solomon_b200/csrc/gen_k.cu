// Instantiates the compile-time generator kernels (kernels_gen.cuh) for the reference's
// other generated shapes and (20,12); the storage-code shapes are in gen_k_more.cu.
#include "kernels_gen.cuh"

namespace rsb {

// Launch shapes from a sweep on B200 (256 stripes of 1 MiB shards): 256-thread CTAs,
// one per SM where the data planes need more than 128 registers, beat 128-thread CTAs
// at 2-3 per SM by 6-10% (the SM's warps stay on nearby code of the straight-line
// body), as for the FFT kernels.
template <bool PTRS>
cudaError_t gen8_launch(int k, int m, const FftArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st) {
  if (k == 7 && m == 13) return launch_gen8_shape<7, 13, PTRS, 256, 2>(a, pt, st);
  if (k == 10 && m == 10) return launch_gen8_shape<10, 10, PTRS, 256, 1>(a, pt, st);
  if (k == 14 && m == 14) return launch_gen8_shape<14, 14, PTRS, 256, 1>(a, pt, st);
  if (k == 18 && m == 6) return launch_gen8_shape<18, 6, PTRS, 256, 1>(a, pt, st);
  if (k == 20 && m == 12) return launch_gen8_shape<20, 12, PTRS, 256, 1>(a, pt, st);
  return gen8_launch_more<PTRS>(k, m, a, pt, st);
}

template cudaError_t gen8_launch<false>(int, int, const FftArgs &, const PtrTableT<false> &, cudaStream_t);
template cudaError_t gen8_launch<true>(int, int, const FftArgs &, const PtrTableT<true> &, cudaStream_t);

}  // namespace rsb
