// Densification statistics of the reference's training loop
// (gaussians_handler.py:116-118, called from GaussianTrainer.py:119 with the
// render's screen-space gradient and its visibility mask):
//
//   counter[visible] += 1
//   accum[visible] += || dL/dmean2D[visible, :2] ||
//
// The reference runs this as boolean-mask indexing in torch (a nonzero pass
// with a host synchronisation, gathers, a norm reduction and scatters); here
// it is one pass over the Gaussians that reads the gradient and the radii and
// updates both accumulators in place.  Visible means radius > 0.
#include "common.cuh"
#include "kernels.h"

namespace w2w {
namespace {

__global__ void __launch_bounds__(256)
densify_stats_kernel(long long P, const float* __restrict__ dL_dmeans2D, const int* __restrict__ radii,
                     float* __restrict__ accum, float* __restrict__ counter) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += stride) {
    if (radii[i] > 0) {
      const float gx = dL_dmeans2D[3 * i], gy = dL_dmeans2D[3 * i + 1];
      accum[i] = __fadd_rn(accum[i], __fsqrt_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy))));
      counter[i] = __fadd_rn(counter[i], 1.0f);
    }
  }
}

}  // namespace

void launch_densify_stats(long long P, const float* dL_dmeans2D, const int* radii, float* accum, float* counter,
                          cudaStream_t stream) {
  if (P <= 0) return;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (P + 255) / 256;
  const int grid = int(want > (long long)sms * 8 ? (long long)sms * 8 : want);
  stage_begin(kStOther, stream);
  densify_stats_kernel<<<grid, 256, 0, stream>>>(P, dL_dmeans2D, radii, accum, counter);
  stage_end(kStOther, stream, 1);
}

}  // namespace w2w
