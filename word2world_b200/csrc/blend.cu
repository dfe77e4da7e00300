// Per-tile front-to-back alpha blending (reference pixelGaussiansFull.cu:3-98,
// pixelGaussiansDev.cuh:5-96, gaussEval.h:7-29).
//
// One CTA per 16x16 tile, one thread per pixel, one warp per 8x4 pixel block
// (tile_walk.cuh).  Each warp walks only the list entries that can reach its
// block with alpha >= 1/255, two at a time: both entries' Gaussian values are
// evaluated before the two transmittance/colour updates, so the two
// evaluations overlap.  The CTA stops as soon as every pixel of the tile has
// terminated (the reference keeps loading every batch of the tile).
//
// Per pixel the arithmetic is the reference's, in its operation order: the
// Gaussian is evaluated from the 2-D covariance and its determinant
// (mahalanobis / det, negative -> 1000), alpha = min(0.99, o*g), entries with
// alpha < 1/255 are skipped, the pixel terminates before the entry that would
// take transmittance below 1e-4, colour accumulates with fma, and the
// contributor count is the 1-based index of the last blended entry.
#include "common.cuh"
#include "kernels.h"
#include "tile_walk.cuh"

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

struct BlendPixel {
  float C0 = 0.f, C1 = 0.f, C2 = 0.f, Wt = 0.f, D = 0.f, T = 1.0f;
  uint32_t last = 0;
  bool done;

  // Entry with alpha `al` (record words q1, q2), 1-based list position `pos`.
  __device__ __forceinline__ void step(float al, float4 q1, float4 q2, uint32_t pos) {
    if (done || !(al >= 1.0f / 255.0f)) return;
    const float nT = mul(T, sub(1.0f, al));
    if (nT < 0.0001f) {
      done = true;
      return;
    }
    const float aT = mul(al, T);
    C0 = fma(q2.x, aT, C0);
    C1 = fma(q2.y, aT, C1);
    C2 = fma(q2.z, aT, C2);
    Wt = add(Wt, aT);
    D = s1<fp::BL_DEPTH>(q1.w, aT, D);
    T = nT;
    last = pos;
  }
};

__global__ void __launch_bounds__(kBlendThreads) blend_kernel(BlendArgs a) {
  __shared__ TileWalkShared sm;
  const int gw = (a.W + kTile - 1) / kTile;
  const int tile = blockIdx.y * gw + blockIdx.x;
  const TilePixel tp;
  const bool inside = tp.px < a.W && tp.py < a.H;
  const uint2 range = a.ranges[tile];
  const int n = int(range.y - range.x);
  const float pxf = float(tp.px), pyf = float(tp.py);

  BlendPixel pix;
  pix.done = !inside;
  const int nb = (n + kBatch - 1) / kBatch;
  Staged st;
  if (nb > 0) {
    stage_load(st, a.record, a.point_list, range.x + threadIdx.x, int(threadIdx.x) < n);
    stage_store(sm, 0, st, tp.X0, tp.Y0);
  }
  for (int b = 0; b < nb; ++b) {
    const int cur = b & 1;
    // barrier: batch b is staged; every warp has finished batch b-1
    if (__syncthreads_count(pix.done ? 1 : 0) == kBlendThreads) break;
    const int next_base = (b + 1) * kBatch;
    if (b + 1 < nb) stage_load(st, a.record, a.point_list, range.x + next_base + threadIdx.x,
                               next_base + int(threadIdx.x) < n);
    if (!__all_sync(0xffffffffu, pix.done)) {
      const float4* s = sm.rec[cur];
      ListIter it(sm.bal[cur][tp.warp]);
      const uint32_t base = uint32_t(b * kBatch) + 1u;
      for (;;) {
        const int j0 = it.next();
        if (j0 < 0) break;
        const int j1r = it.next();
        const int j1 = j1r < 0 ? j0 : j1r;
        const float4 a0 = s[kRecVec * j0], a1 = s[kRecVec * j0 + 1];
        const float4 b0 = s[kRecVec * j1], b1 = s[kRecVec * j1 + 1];
        const float g0 = gauss_eval(pxf, pyf, a0.x, a0.y, a0.z, a0.w, a1.x, a1.y);
        const float g1 = gauss_eval(pxf, pyf, b0.x, b0.y, b0.z, b0.w, b1.x, b1.y);
        const float al0 = fminf(0.99f, mul(a1.z, g0));
        const float al1 = fminf(0.99f, mul(b1.z, g1));
        pix.step(al0, a1, s[kRecVec * j0 + 2], base + uint32_t(j0));
        if (j1r >= 0) pix.step(al1, b1, s[kRecVec * j1 + 2], base + uint32_t(j1));
        if (__all_sync(0xffffffffu, pix.done)) break;
      }
    }
    if (b + 1 < nb) stage_store(sm, cur ^ 1, st, tp.X0, tp.Y0);
  }
  if (inside) {
    const size_t p = size_t(tp.py) * a.W + tp.px;
    const size_t hw = size_t(a.W) * a.H;
    a.n_contrib[p] = pix.last;
    a.out_alpha[p] = pix.Wt;
    a.out_depth[p] = pix.D;
    a.T_final[p] = pix.T;
    a.out_color[p] = fma(pix.T, a.bg[0], pix.C0);
    a.out_color[hw + p] = fma(pix.T, a.bg[1], pix.C1);
    a.out_color[2 * hw + p] = fma(pix.T, a.bg[2], pix.C2);
  }
  // largest contributor count in the tile (the backward starts there)
  __shared__ uint32_t s_max[kBlendThreads / 32];
  const uint32_t wm = __reduce_max_sync(0xffffffffu, pix.last);
  if (tp.lane == 0) s_max[tp.warp] = wm;
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
