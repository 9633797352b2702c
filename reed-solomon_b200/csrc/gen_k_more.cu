// Instantiates the compile-time generator kernels (kernels_gen.cuh) for common storage
// codes beyond the reference's generated shapes: (4,2), (6,3), (8,4), (10,4), (12,4),
// (16,4), (17,3). Compiled apart from gen_k.cu so the two build in parallel.
#include "kernels_gen.cuh"

namespace rsb {

// Launch shapes: 256-thread CTAs, two per SM where the data planes fit 128 registers
// without spills, else one.
template <bool PTRS>
cudaError_t gen8_launch_more(int k, int m, const FftArgs &a, const PtrTableT<PTRS> &pt, cudaStream_t st) {
  if (k == 4 && m == 2) return launch_gen8_shape<4, 2, PTRS, 256, 2>(a, pt, st);
  if (k == 6 && m == 3) return launch_gen8_shape<6, 3, PTRS, 256, 2>(a, pt, st);
  if (k == 8 && m == 4) return launch_gen8_shape<8, 4, PTRS, 256, 2>(a, pt, st);
  if (k == 10 && m == 4) return launch_gen8_shape<10, 4, PTRS, 256, 2>(a, pt, st);
  if (k == 12 && m == 4) return launch_gen8_shape<12, 4, PTRS, 256, 1>(a, pt, st);
  if (k == 16 && m == 4) return launch_gen8_shape<16, 4, PTRS, 256, 1>(a, pt, st);
  if (k == 17 && m == 3) return launch_gen8_shape<17, 3, PTRS, 256, 1>(a, pt, st);
  return cudaErrorInvalidValue;
}

template cudaError_t gen8_launch_more<false>(int, int, const FftArgs &, const PtrTableT<false> &, cudaStream_t);
template cudaError_t gen8_launch_more<true>(int, int, const FftArgs &, const PtrTableT<true> &, cudaStream_t);

}  // namespace rsb
