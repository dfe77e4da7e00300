// The activation preamble of Renderer.render (reference Renderer.py:164-167)
// as one forward and one backward pass over the Gaussians:
//
//   opacity = sigmoid(opacity logit), scales = exp(svec),
//   rotations = normalize(quaternion), shs = cat(sh_dc, sh_ac)
//
// The reference runs these as separate torch operations (four forward
// kernels, a norm reduction among them, and about a dozen in the backward,
// each a full pass over its tensors, plus the SH concatenation's copy both
// ways).  The forward here is bit-identical to those torch operations on a
// B200 (checked over 2^24 random inputs): sigmoid is 1 / (1 + exp(-x)) with
// IEEE division, and the quaternion norm sums the squares as
// (w*w + y*y) + (x*x + z*z) with every product rounded, then sqrt, a 1e-12
// floor and an IEEE division per component.  The backward applies the same
// chain rule torch's autograd would (equal up to rounding).
#include "common.cuh"
#include "kernels.h"

namespace w2w {
namespace {

constexpr int kActThreads = 256;

// kRow: floats per SH row, 3 (K + 1), when known at compile time (0: a.K's);
// a constant row turns the element -> Gaussian division into a multiply.
template <int kRow>
__global__ void __launch_bounds__(kActThreads)
activate_kernel(ActivateArgs a) {
  const long long P = a.P;
  const int K = kRow > 0 ? kRow / 3 - 1 : a.K;  // rest coefficients per Gaussian (sh_ac rows)
  const int row = 3 * (K + 1);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += stride) {
    a.opacity[i] = act_sigmoid(a.opacity_logit[i]);
#pragma unroll
    for (int k = 0; k < 3; ++k) a.scales[3 * i + k] = expf(a.svec[3 * i + k]);
    const float4 r = act_normalize(a.quat[4 * i], a.quat[4 * i + 1], a.quat[4 * i + 2], a.quat[4 * i + 3]);
    a.rotations[4 * i] = r.x;
    a.rotations[4 * i + 1] = r.y;
    a.rotations[4 * i + 2] = r.z;
    a.rotations[4 * i + 3] = r.w;
  }
  // shs[i] = [sh_dc[i], sh_ac[i]]: consecutive threads write consecutive floats
  // (32-bit indices: the host checks P * row < 2^31)
  const uint32_t total = uint32_t(P) * uint32_t(row);
#pragma unroll 4
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += uint32_t(stride)) {
    const uint32_t i = j / uint32_t(row);
    const uint32_t c = j - i * uint32_t(row);
    a.shs[j] = c < 3u ? __ldg(a.sh_dc + 3u * i + c) : __ldg(a.sh_ac + i * uint32_t(3 * K) + (c - 3u));
  }
}

template <int kRow>
__global__ void __launch_bounds__(kActThreads)
activate_backward_kernel(ActivateBackwardArgs a) {
  const long long P = a.P;
  const int K = kRow > 0 ? kRow / 3 - 1 : a.K;
  const int row = 3 * (K + 1);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += stride) {
    // activated opacity and scales: kept by the forward, or recomputed from
    // the raw parameters (the fused-preamble path keeps none)
    const float y = a.opacity != nullptr ? a.opacity[i] : act_sigmoid(a.opacity_logit[i]);
    a.d_opacity_logit[i] = a.g_opacity[i] * (1.f - y) * y;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      a.d_svec[3 * i + k] = a.g_scales[3 * i + k] * (a.scales != nullptr ? a.scales[3 * i + k] : expf(a.svec[3 * i + k]));
    const float q[4] = {a.quat[4 * i], a.quat[4 * i + 1], a.quat[4 * i + 2], a.quat[4 * i + 3]};
    const float g[4] = {a.g_rotations[4 * i], a.g_rotations[4 * i + 1], a.g_rotations[4 * i + 2],
                        a.g_rotations[4 * i + 3]};
    const float n = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    if (n > 1e-12f) {
      // d(q / n) = (g - r (r . g)) / n with r = q / n
      const float inv = 1.f / n;
      const float rg = (q[0] * g[0] + q[1] * g[1] + q[2] * g[2] + q[3] * g[3]) * inv;
#pragma unroll
      for (int k = 0; k < 4; ++k) a.d_quat[4 * i + k] = (g[k] - q[k] * inv * rg) * inv;
    } else {  // the norm is clamped to 1e-12 there: q / 1e-12 is linear in q
#pragma unroll
      for (int k = 0; k < 4; ++k) a.d_quat[4 * i + k] = g[k] * 1e12f;
    }
  }
  const uint32_t total = uint32_t(P) * uint32_t(row);
#pragma unroll 4
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += uint32_t(stride)) {
    const uint32_t i = j / uint32_t(row);
    const uint32_t c = j - i * uint32_t(row);
    const float v = __ldg(a.g_shs + j);
    if (c < 3u) a.d_sh_dc[3u * i + c] = v;
    else a.d_sh_ac[i * uint32_t(3 * K) + (c - 3u)] = v;
  }
}

int act_grid(long long P, int row) {
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (P * row + kActThreads - 1) / kActThreads;
  return int(want < 1 ? 1 : (want > (long long)sms * 16 ? (long long)sms * 16 : want));
}

}  // namespace

void launch_activate(const ActivateArgs& a, cudaStream_t stream) {
  if (a.P <= 0) return;
  const int grid = act_grid(a.P, 3 * (a.K + 1));
  stage_begin(kStOther, stream);
  if (a.K == 15) activate_kernel<48><<<grid, kActThreads, 0, stream>>>(a);
  else activate_kernel<0><<<grid, kActThreads, 0, stream>>>(a);
  stage_end(kStOther, stream, 1);
}

void launch_activate_backward(const ActivateBackwardArgs& a, cudaStream_t stream) {
  if (a.P <= 0) return;
  const int grid = act_grid(a.P, 3 * (a.K + 1));
  stage_begin(kStOther, stream);
  if (a.K == 15) activate_backward_kernel<48><<<grid, kActThreads, 0, stream>>>(a);
  else activate_backward_kernel<0><<<grid, kActThreads, 0, stream>>>(a);
  stage_end(kStOther, stream, 1);
}

}  // namespace w2w
