// Per-tile front-to-back alpha blending (reference pixelGaussiansFull.cu:3-98,
// pixelGaussiansDev.cuh:5-96, gaussEval.h:7-29).
//
// One CTA per 16x16 tile, one thread per pixel, one warp per 8x4 pixel block
// (tile_walk.cuh).  Each warp walks only the list entries that can reach its
// block with alpha >= 1/255, kBlendIlp at a time: all their Gaussian values are
// evaluated before the sequential transmittance/colour updates, so the
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

constexpr int kBlendIlp = 4;  // list entries evaluated together per warp (the list is read 4 bytes at a time)
static_assert(kBlendIlp == 4, "packed list read");

// The reference's Gaussian value (gaussEval.h:7-29) in two halves: the
// mahalanobis numerator, then exp(-0.5 * num / det) with negative distances
// mapped to 1000.
__device__ __forceinline__ float gauss_num(float px, float py, float mx, float my, float cxx, float cxy, float cyy) {
  using namespace fp;
  const float dx = sub(px, mx), dy = sub(py, my);
  const float tX = d2<BL_TX>(dx, cyy, dy, cxy);
  const float tY = s2<BL_TY>(-dx, cxy, dy, cxx);
  return s2<BL_NUM>(tX, dx, tY, dy);
}
__device__ __forceinline__ float gauss_from_m(float m) {
  if (m < 0.0f) m = 1000.0f;
  return expf(mul(-0.5f, m));
}

struct BlendPixel {
  float C0 = 0.f, C1 = 0.f, C2 = 0.f, Wt = 0.f, D = 0.f, T = 1.0f;
  uint32_t last = 0;
  bool done;

  // Entry with alpha `al` (record words q1, q2), 1-based list position `pos`.
  // Branch-free: the updates are selected, so a warp's lanes never diverge.
  __device__ __forceinline__ void step(float al, float4 q1, float4 q2, uint32_t pos) {
    const bool blend = !done && al >= 1.0f / 255.0f;
    const float nT = mul(T, sub(1.0f, al));
    const bool term = blend && nT < 0.0001f;
    const bool acc = blend && !term;
    const float aT = mul(al, T);
    C0 = acc ? fma(q2.x, aT, C0) : C0;
    C1 = acc ? fma(q2.y, aT, C1) : C1;
    C2 = acc ? fma(q2.z, aT, C2) : C2;
    Wt = acc ? add(Wt, aT) : Wt;
    D = acc ? s1<fp::BL_DEPTH>(q1.w, aT, D) : D;
    T = acc ? nT : T;
    last = acc ? pos : last;
    done = done || term;
  }
};

// Warps per CTA, kBlendWarps: 8 (one CTA per tile) or 4 (two CTAs per tile,
// upper and lower eight rows; see tile_walk.cuh), chosen at run time (the
// tuning knob W2W_TUNE_BLEND_WARPS).  Results are identical either way.
template <int kBlendWarps>
__global__ void __launch_bounds__(32 * kBlendWarps, 16 / kBlendWarps) blend_kernel(BlendArgs a) {
  constexpr int kBlendParts = 8 / kBlendWarps;  // CTAs per tile
  constexpr int kBlendCta = 32 * kBlendWarps;
  constexpr int kStagePer = kBatch / kBlendCta;  // entries each thread stages per batch
  static_assert(kBatch % kBlendCta == 0, "whole entries per thread");
  __shared__ TileWalkShared<kBlendWarps> sm;
  const int part = int(blockIdx.x) % kBlendParts;
  const int tile = int(a.order[blockIdx.x / kBlendParts]);
  // this tile's image: the call's, or its batch item's
  int W = a.W, H = a.H, ltile = tile;
  size_t pbase = 0;
  const float* bg = a.bg;
  if (a.items != nullptr) {
    const BatchItem& it = a.items[find_item_tile(a.items, a.num_items, uint32_t(tile))];
    W = it.W;
    H = it.H;
    ltile = tile - int(it.tile_base);
    pbase = size_t(it.pix_base);
    bg = it.bg;
  }
  const int gw = (W + kTile - 1) / kTile;
  const int warp = int(threadIdx.x >> 5), first_block = part * kBlendWarps;
  const TilePixel tp(ltile, gw, first_block + warp);
  const bool inside = tp.px < W && tp.py < H;
  const uint2 range = a.ranges[tile];
  const int n = int(range.y - range.x);
  const float pxf = float(tp.px), pyf = float(tp.py);

  BlendPixel pix;
  pix.done = !inside;
  const int nb = (n + kBatch - 1) / kBatch;
  Staged st[kStagePer];
  auto load = [&](int base) {
#pragma unroll
    for (int r = 0; r < kStagePer; ++r) {
      const int e = base + r * kBlendCta + int(threadIdx.x);
      stage_load(st[r], a.record, a.point_list, range.x + e, e < n, a.num_records);
    }
  };
  // block masks for the backward: the upper half's CTA (or the whole tile's)
  // writes the top array, the lower half's the bottom one
  uint8_t* lo_dst = a.mask_top == nullptr ? nullptr : (part == 0 ? a.mask_top : a.mask_bottom) + range.x;
  uint8_t* hi_dst = a.mask_top == nullptr || kBlendParts != 1 ? nullptr : a.mask_bottom + range.x;
  auto store = [&](int buf, int base) {
#pragma unroll
    for (int r = 0; r < kStagePer; ++r)
      stage_store(sm, buf, st[r], r * kBlendCta + int(threadIdx.x), tp.X0, tp.Y0, first_block,
                  lo_dst ? lo_dst + base : nullptr, hi_dst ? hi_dst + base : nullptr);
  };
  if (nb > 0) {
    load(0);
    store(0, 0);
  }
  for (int b = 0; b < nb; ++b) {
    const int cur = b & 1;
    // barrier: batch b is staged; every warp has finished batch b-1
    if (__syncthreads_count(pix.done ? 1 : 0) == kBlendCta) break;
    const int next_base = (b + 1) * kBatch;
    if (b + 1 < nb) load(next_base);
    if (!__all_sync(0xffffffffu, pix.done)) {
      const float4* s = sm.rec[cur];
      const int cnt = build_list(sm, cur, warp, tp.lane);
      const uint8_t* lst = sm.list[warp];
      const uint32_t base = uint32_t(b * kBatch) + 1u;
      for (int k0 = 0; k0 < cnt; k0 += kBlendIlp) {
        // kBlendIlp entries in flight: their Gaussian values are independent,
        // only the transmittance/colour updates are sequential
        const uint32_t packed = *reinterpret_cast<const uint32_t*>(lst + k0);
        int j[kBlendIlp];
#pragma unroll
        for (int k = 0; k < kBlendIlp; ++k) j[k] = k0 + k < cnt ? int((packed >> (8 * k)) & 255u) : -1;
        float al[kBlendIlp], num[kBlendIlp], m[kBlendIlp];
        float4 q1[kBlendIlp], q2[kBlendIlp];
        bool in_range = true;
#pragma unroll
        for (int k = 0; k < kBlendIlp; ++k) {
          const int jj = j[k] < 0 ? j[0] : j[k];
          const float4 q0 = s[kRecVec * jj];
          q1[k] = s[kRecVec * jj + 1];
          q2[k] = s[kRecVec * jj + 2];
          num[k] = gauss_num(pxf, pyf, q0.x, q0.y, q0.z, q0.w, q1[k].x);
          in_range = in_range && div_in_range(num[k], q1[k].y);
        }
        // the branch-free division when every lane's operands allow it
        if (__all_sync(0xffffffffu, in_range)) {
#pragma unroll
          for (int k = 0; k < kBlendIlp; ++k) m[k] = div_markstein(num[k], q1[k].y);
        } else {
#pragma unroll
          for (int k = 0; k < kBlendIlp; ++k) m[k] = div(num[k], q1[k].y);
        }
#pragma unroll
        for (int k = 0; k < kBlendIlp; ++k)
          al[k] = j[k] < 0 ? 0.0f : fminf(0.99f, mul(q1[k].z, gauss_from_m(m[k])));
#pragma unroll
        for (int k = 0; k < kBlendIlp; ++k) pix.step(al[k], q1[k], q2[k], base + uint32_t(j[k]));
        if (__all_sync(0xffffffffu, pix.done)) break;
      }
    }
    if (b + 1 < nb) store(cur ^ 1, next_base);
  }
  if (inside) {
    const size_t q = size_t(tp.py) * W + tp.px;
    const size_t p = pbase + q, cp = 3 * pbase + q;
    const size_t hw = size_t(W) * H;
    a.n_contrib[p] = pix.last;
    a.out_alpha[p] = pix.Wt;
    a.out_depth[p] = pix.D;
    a.T_final[p] = pix.T;
    a.out_color[cp] = fma(pix.T, bg[0], pix.C0);
    a.out_color[hw + cp] = fma(pix.T, bg[1], pix.C1);
    a.out_color[2 * hw + cp] = fma(pix.T, bg[2], pix.C2);
  }
  // largest contributor count in the tile (the backward starts there); the
  // tile's CTAs combine theirs (tile_max is cleared before the launch)
  __shared__ uint32_t s_max[kBlendWarps];
  const uint32_t wm = __reduce_max_sync(0xffffffffu, pix.last);
  if (tp.lane == 0) s_max[warp] = wm;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t mx = 0;
    for (int w = 0; w < kBlendWarps; ++w) mx = max(mx, s_max[w]);
    if (kBlendParts == 1) a.tile_max[tile] = mx;
    else atomicMax(&a.tile_max[tile], mx);
  }
}

}  // namespace

// Bucket sort of the tiles by decreasing list length (quarter-octave buckets;
// order within a bucket is arbitrary).  One CTA.
__global__ void __launch_bounds__(1024) tile_order_kernel(const uint2* ranges, const uint32_t* counts, int num_tiles,
                                                          uint32_t* order, uint32_t* zero) {
  constexpr int kBuckets = 130;
  __shared__ uint32_t s_cnt[kBuckets];
  __shared__ uint32_t s_pos[kBuckets];
  auto bucket = [](uint32_t n) -> int {
    if (n == 0) return 0;
    const int e = 31 - __clz(n);
    const uint32_t q = e >= 2 ? (n >> (e - 2)) & 3u : (n << (2 - e)) & 3u;
    return 1 + 4 * e + int(q);
  };
  for (int i = threadIdx.x; i < kBuckets; i += blockDim.x) s_cnt[i] = 0;
  if (zero != nullptr)
    for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) zero[t] = 0u;
  __syncthreads();
  auto weight = [&](int t) -> uint32_t {
    if (counts) return counts[t];
    const uint2 r = ranges[t];
    return r.y - r.x;
  };
  for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) atomicAdd(&s_cnt[bucket(weight(t))], 1u);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int b = kBuckets - 1; b >= 0; --b) {
      s_pos[b] = acc;
      acc += s_cnt[b];
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) order[atomicAdd(&s_pos[bucket(weight(t))], 1u)] = uint32_t(t);
}

void launch_blend(const BlendArgs& a, cudaStream_t stream) {
  const int tiles = a.items ? a.total_tiles : ((a.W + kTile - 1) / kTile) * ((a.H + kTile - 1) / kTile);
  if (tiles <= 0) return;
  const int warps = tune_value(kTuneBlendWarps);
  stage_begin(kStOther, stream);
  // with two CTAs per tile they combine their maxima with atomics: clear first
  tile_order_kernel<<<1, 1024, 0, stream>>>(a.ranges, nullptr, tiles, a.order, warps == 4 ? a.tile_max : nullptr);
  stage_end(kStOther, stream, 1);
  stage_begin(kStBlend, stream);
  if (warps == 4) blend_kernel<4><<<tiles * 2, 128, 0, stream>>>(a);
  else blend_kernel<8><<<tiles, 256, 0, stream>>>(a);
  stage_end(kStBlend, stream, 1);
  // the backward's order: by the largest contributor count the blend just found
  stage_begin(kStOther, stream);
  tile_order_kernel<<<1, 1024, 0, stream>>>(nullptr, a.tile_max, tiles, a.order_bwd, nullptr);
  stage_end(kStOther, stream, 1);
}

}  // namespace w2w
