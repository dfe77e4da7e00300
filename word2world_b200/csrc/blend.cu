// Per-tile front-to-back alpha blending (reference pixelGaussiansFull.cu:3-98,
// pixelGaussiansDev.cuh:5-96, gaussEval.h:7-29).
//
// One CTA per 16x16 tile, one thread per pixel.  The tile's sorted list is
// staged 256 Gaussians at a time into shared memory (64-byte records,
// gathered by id), double-buffered: the next batch's records are loaded into
// registers while the current batch is blended and stored to the other buffer
// afterwards.  The CTA stops as soon as every pixel of the tile has
// terminated (the reference keeps loading every batch of the tile).  Pairs
// that certainly fall below the alpha threshold are rejected with a
// quadratic-form test before the exact evaluation (BlendRecord::reject).
//
// Per pixel the arithmetic is the reference's, in its operation order: the
// Gaussian is evaluated from the 2-D covariance and its determinant
// (mahalanobis / det, negative -> 1000), alpha = min(0.99, o*g), entries with
// alpha < 1/255 are skipped, the pixel terminates before the entry that would
// take transmittance below 1e-4, colour accumulates with fma, and the
// contributor count is the 1-based index of the last blended entry.
#include "common.cuh"
#include "kernels.h"

namespace w2w {
namespace {

__device__ __forceinline__ float gauss_eval(float px, float py, float mx, float my, float cxx, float cxy, float cyy,
                                            float det) {
  using namespace fp;
  const float dx = sub(px, mx), dy = sub(py, my);
  const float tX = d2<BL_TX>(dx, cyy, dy, cxy);
  const float tY = s2<BL_TY>(-dx, cxy, dy, cxx);
  const float num = s2<BL_NUM>(tX, dx, tY, dy);
  float m = div(num, det);
  if (m < 0.0f) m = 1000.0f;
  return expf(mul(-0.5f, m));
}

// True when the pair certainly has alpha < 1/255 (see BlendRecord::reject).
__device__ __forceinline__ bool early_reject(float dx, float dy, float4 q3, float reject) {
  const float ax = q3.x * dx * dx, cy = q3.z * dy * dy, bxy = 2.0f * q3.y * dx * dy;
  const float qf = ax + cy + bxy;
  const float mag = ax + cy + fabsf(bxy);
  return qf - 1e-4f * mag > reject;
}

__global__ void __launch_bounds__(kBlendThreads) blend_kernel(BlendArgs a) {
  __shared__ float4 s_rec[2][kBatch * 4];
  const int gw = (a.W + kTile - 1) / kTile;
  const int tile = blockIdx.y * gw + blockIdx.x;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int px = blockIdx.x * kTile + tx, py = blockIdx.y * kTile + ty;
  const bool inside = px < a.W && py < a.H;
  const uint2 range = a.ranges[tile];
  const int n = int(range.y - range.x);
  const float pxf = float(px), pyf = float(py);
  const float4* rec = reinterpret_cast<const float4*>(a.record);

  float C0 = 0.f, C1 = 0.f, C2 = 0.f, Wt = 0.f, D = 0.f, T = 1.0f;
  uint32_t contributor = 0, last = 0;
  bool done = !inside;

  const int nb = (n + kBatch - 1) / kBatch;
  float4 r0, r1, r2, r3;
  // first batch
  if (nb > 0 && int(threadIdx.x) < min(kBatch, n)) {
    const uint32_t id = a.point_list[range.x + threadIdx.x];
    r0 = __ldg(rec + 4 * size_t(id));
    r1 = __ldg(rec + 4 * size_t(id) + 1);
    r2 = __ldg(rec + 4 * size_t(id) + 2);
    r3 = __ldg(rec + 4 * size_t(id) + 3);
    s_rec[0][4 * threadIdx.x] = r0;
    s_rec[0][4 * threadIdx.x + 1] = r1;
    s_rec[0][4 * threadIdx.x + 2] = r2;
    s_rec[0][4 * threadIdx.x + 3] = r3;
  }
  const float min_alpha = 1.0f / 255.0f;
  for (int b = 0; b < nb; ++b) {
    const int cur = b & 1;
    // barrier: batch b is in shared memory; all pixels finished batch b-1
    if (__syncthreads_count(done ? 1 : 0) == kBlendThreads) break;
    const int next_base = (b + 1) * kBatch;
    const bool has_next = (b + 1 < nb) && (next_base + int(threadIdx.x) < n);
    if (has_next) {
      const uint32_t id = a.point_list[range.x + next_base + threadIdx.x];
      r0 = __ldg(rec + 4 * size_t(id));
      r1 = __ldg(rec + 4 * size_t(id) + 1);
      r2 = __ldg(rec + 4 * size_t(id) + 2);
      r3 = __ldg(rec + 4 * size_t(id) + 3);
    }
    const int cnt = min(kBatch, n - b * kBatch);
    if (!done) {
      const float4* s = s_rec[cur];
      for (int j = 0; j < cnt; ++j) {
        ++contributor;
        const float4 q0 = s[4 * j];
        // q0 = (mx, my, cxx, cxy), q1 = (cyy, det, opacity, depth), q2 = (r, g, b, reject), q3 = conic
        if (early_reject(sub(pxf, q0.x), sub(pyf, q0.y), s[4 * j + 3], s[4 * j + 2].w)) continue;
        const float4 q1 = s[4 * j + 1];
        const float g = gauss_eval(pxf, pyf, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y);
        const float a_ = fminf(0.99f, mul(q1.z, g));
        if (a_ >= min_alpha) {
          const float nT = mul(T, sub(1.0f, a_));
          if (nT >= 0.0001f) {
            const float4 q2 = s[4 * j + 2];
            const float aT = mul(a_, T);
            C0 = fma(q2.x, aT, C0);
            C1 = fma(q2.y, aT, C1);
            C2 = fma(q2.z, aT, C2);
            Wt = add(Wt, aT);
            D = s1<fp::BL_DEPTH>(q1.w, aT, D);
            T = nT;
            last = contributor;
          } else {
            done = true;
            break;
          }
        }
      }
    }
    if (has_next) {
      float4* s = s_rec[cur ^ 1];
      s[4 * threadIdx.x] = r0;
      s[4 * threadIdx.x + 1] = r1;
      s[4 * threadIdx.x + 2] = r2;
      s[4 * threadIdx.x + 3] = r3;
    }
  }
  if (inside) {
    const size_t pix = size_t(py) * a.W + px;
    const size_t hw = size_t(a.W) * a.H;
    a.n_contrib[pix] = last;
    a.out_alpha[pix] = Wt;
    a.out_depth[pix] = D;
    a.T_final[pix] = T;
    a.out_color[pix] = fma(T, a.bg[0], C0);
    a.out_color[hw + pix] = fma(T, a.bg[1], C1);
    a.out_color[2 * hw + pix] = fma(T, a.bg[2], C2);
  }
  // largest contributor count in the tile (the backward starts there)
  __shared__ uint32_t s_max[kBlendThreads / 32];
  const uint32_t wm = __reduce_max_sync(0xffffffffu, last);
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = wm;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t m = 0;
    for (int w = 0; w < kBlendThreads / 32; ++w) m = max(m, s_max[w]);
    a.tile_max[tile] = m;
  }
}

}  // namespace

void launch_blend(const BlendArgs& a, cudaStream_t stream) {
  const dim3 grid((a.W + kTile - 1) / kTile, (a.H + kTile - 1) / kTile);
  if (grid.x == 0 || grid.y == 0) return;
  stage_begin(kStBlend, stream);
  blend_kernel<<<grid, kBlendThreads, 0, stream>>>(a);
  stage_end(kStBlend, stream, 1);
}

}  // namespace w2w
