// Backward pass.
//
// Per-pixel pass (reference backward.cu:521-665): one CTA per tile, pixels
// walk the tile's list back to front, recomputing each pair's alpha from the
// stored state (final transmittance and last-contributor index) instead of
// storing per-pair values.  Each entry's per-pixel contributions are summed
// across the warp with shuffles and added with one atomic per warp (the
// reference issues ten atomics per pixel-Gaussian pair).  A tile starts at its
// largest contributor count: entries past it are skipped by every pixel.
//
// Per-Gaussian pass: the reference's computeCov2DCUDA (backward.cu:27-227) and
// backwardPreprocessingKernel (backward.cu:229-519) fused into one thread per
// Gaussian.
//
// grad_mode 0 reproduces the reference's formulas, including where they are
// not the derivative of its forward (+0.3 on the 2-D covariance, a 1.3*tan box
// clamp, colour-clamp masks, SH_C2[2] = 0.3154 and all 16 SH bands).  grad_mode
// 1 is the exact derivative of the forward: the pair set is re-derived with the
// forward's own Gaussian evaluation and the forward's final transmittance.
#include "common.cuh"
#include "kernels.h"
#include "tile_walk.cuh"

namespace w2w {
namespace {

constexpr int kValues = 10;
// Heavy tiles: each warp's walk is cut into kSplitWays segments, one CTA per
// segment.  The CTA of a segment first replays the state recurrences of the
// entries behind it (alpha and the transmittance / suffix updates only: no
// gradients, no reduction, about kReplayCost of a full entry's work) to reach
// the state at its segment's end, then walks its segment in full.  All CTAs
// compute the state with the same code in the same order, so each starts from
// exactly the state a single walk would have reached; only the order of the
// atomic additions changes.  Segment lengths (from the back) make the
// segments' work equal: L_0 = W, L_i = W - kReplayCost * (L_0 + ... + L_{i-1}).
// kSplitWays (2 or 3) and the number of split tiles are run-time tuning
// knobs (W2W_TUNE_BWD_WAYS, W2W_TUNE_BWD_SPLIT); only the order of the atomic
// additions depends on them.
constexpr float kReplayCost = 0.22f;

// List positions [lo, hi) of segment k (0 = the back-most) of a walk of
// length `walk`.
template <int kSplitWays>
__device__ __forceinline__ void segment_of(int walk, int k, int& lo, int& hi) {
  float len[kSplitWays], before = 0.f, total = 0.f;
#pragma unroll
  for (int i = 0; i < kSplitWays; ++i) {
    len[i] = 1.0f - kReplayCost * before;
    before += len[i];
  }
  total = before;
  float b0 = 0.f, b1 = 0.f;
#pragma unroll
  for (int i = 0; i < kSplitWays; ++i) {
    if (i < k) b0 += len[i];
    if (i <= k) b1 += len[i];
  }
  hi = walk - int(float(walk) * (b0 / total));
  lo = k == kSplitWays - 1 ? 0 : walk - int(float(walk) * (b1 / total));
  lo = max(0, min(lo, hi));
}

// Where each of the ten per-entry sums goes: after the transposed reduction
// below, lane L (L even) holds the warp's sum of value (L >> 1); lanes 0..18
// each add one of them to its gradient array.
struct Target {
  float* base;
  int mult, off;
  bool active;
  bool second = false;  // flush_pair: the lane's value belongs to the second entry
};

// The gradient array and component of value idx (0..kValues-1).
__device__ __forceinline__ Target value_target(const BackwardArgs& a, int mode, int idx, bool active) {
  Target t{nullptr, 0, 0, active && idx >= 0 && idx < kValues};
  if (idx < 0) return t;
  if (idx < 3) t = Target{a.dL_dcolors, 3, idx, t.active};
  else if (idx == 3) t = Target{a.acc_depth, 1, 0, t.active};
  else if (idx < 6) t = Target{a.dL_dmean2D, 3, idx - 4, t.active};
  else if (idx < 9) t = Target{a.acc_cov, 4, mode == 0 ? (idx == 8 ? 3 : idx - 6) : idx - 6, t.active};
  else if (idx == 9) t = Target{a.dL_dopacity, 1, 0, t.active};
  return t;
}

__device__ __forceinline__ Target lane_target(const BackwardArgs& a, int mode) {
  const int lane = threadIdx.x & 31, idx = (lane >> 1) & 15;
  return value_target(a, mode, idx, (lane & 1) == 0);
}

// flush_pair's lane roles: lane bit 4 picks the entry; within it the 16 lanes
// of bits 0-3 hold values 5 * b3 + {0, 1, 2, 3, 4} at (b2, b1, b0) = (000,
// 001, 010, 100, 101), and the other three hold the tree's zero padding.
__device__ __forceinline__ Target lane_target_pair(const BackwardArgs& a, int mode) {
  const int lane = threadIdx.x & 31;
  const int b0 = lane & 1, b1 = (lane >> 1) & 1, b2 = (lane >> 2) & 1, b3 = (lane >> 3) & 1;
  const int sub = b2 ? (b1 ? -1 : 3 + b0) : (b1 && b0 ? -1 : 2 * b1 + b0);
  Target t = value_target(a, mode, sub < 0 ? -1 : 5 * b3 + sub, true);
  t.second = (lane & 16) != 0;
  return t;
}

// Sum ten values over the warp with 16 shuffles (each step exchanges the half
// of the partial sums a lane does not keep) and add each total with one
// atomic, issued by ten lanes at once.
__device__ __forceinline__ void flush(const float (&c)[kValues], bool any_contrib, uint32_t id, const Target& t) {
  if (!__any_sync(0xffffffffu, any_contrib)) return;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  float v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = k < kValues ? c[k] : 0.0f;
  float w8[8], w4[4], w2[2];
  bool b = lane & 16;
#pragma unroll
  for (int k = 0; k < 8; ++k) w8[k] = (b ? v[k + 8] : v[k]) + __shfl_xor_sync(full, b ? v[k] : v[k + 8], 16);
  b = lane & 8;
#pragma unroll
  for (int k = 0; k < 4; ++k) w4[k] = (b ? w8[k + 4] : w8[k]) + __shfl_xor_sync(full, b ? w8[k] : w8[k + 4], 8);
  b = lane & 4;
#pragma unroll
  for (int k = 0; k < 2; ++k) w2[k] = (b ? w4[k + 2] : w4[k]) + __shfl_xor_sync(full, b ? w4[k] : w4[k + 2], 4);
  b = lane & 2;
  float w1 = (b ? w2[1] : w2[0]) + __shfl_xor_sync(full, b ? w2[0] : w2[1], 2);
  w1 += __shfl_xor_sync(full, w1, 1);
  if (t.active) atomicAdd(t.base + size_t(t.mult) * id + t.off, w1);
}

// Two entries' sums at once: their 20 values halve over five exchange steps
// (10, 5, 3, 2 and 1 shuffles, the odd counts padded with a zero) instead of
// 16 shuffles per entry; 20 lanes then add one total each (lane_target_pair).
// An entry no lane contributes to is left out: the other goes alone (flush).
__device__ __forceinline__ void flush_pair(const float (&c0)[kValues], const float (&c1)[kValues], bool any0,
                                           bool any1, uint32_t id0, uint32_t id1, const Target& t,
                                           const Target& tp) {
  const bool has0 = __any_sync(0xffffffffu, any0), has1 = __any_sync(0xffffffffu, any1);
  if (!has0 || !has1) {
    if (has0) flush(c0, true, id0, t);
    if (has1) flush(c1, true, id1, t);
    return;
  }
  static_assert(kValues == 10, "pair tree layout");
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  float w10[10], w5[6], w3[4], w2[2];
  bool b = lane & 16;
#pragma unroll
  for (int k = 0; k < 10; ++k) w10[k] = (b ? c1[k] : c0[k]) + __shfl_xor_sync(full, b ? c0[k] : c1[k], 16);
  b = lane & 8;
#pragma unroll
  for (int k = 0; k < 5; ++k) w5[k] = (b ? w10[k + 5] : w10[k]) + __shfl_xor_sync(full, b ? w10[k] : w10[k + 5], 8);
  w5[5] = 0.0f;
  b = lane & 4;
#pragma unroll
  for (int k = 0; k < 3; ++k) w3[k] = (b ? w5[k + 3] : w5[k]) + __shfl_xor_sync(full, b ? w5[k] : w5[k + 3], 4);
  w3[3] = 0.0f;
  b = lane & 2;
#pragma unroll
  for (int k = 0; k < 2; ++k) w2[k] = (b ? w3[k + 2] : w3[k]) + __shfl_xor_sync(full, b ? w3[k] : w3[k + 2], 2);
  b = lane & 1;
  const float w1 = (b ? w2[1] : w2[0]) + __shfl_xor_sync(full, b ? w2[0] : w2[1], 1);
  if (tp.active) atomicAdd(tp.base + size_t(tp.mult) * (tp.second ? id1 : id0) + tp.off, w1);
}

// Pixel-loop prologue shared by both modes: this thread's pixel, its
// upstream gradients and contributor count, the tile's walk length.
struct BwdPixel {
  int tile;
  TilePixel tp;
  bool inside;
  size_t pix, hw;
  uint2 range;
  int walk;  // list positions [0, walk) may hold contributors of this warp's pixels
  uint32_t last, warp_last;
  float dLp0 = 0.f, dLp1 = 0.f, dLp2 = 0.f, dLd = 0.f, dLa = 0.f;
  int W, H;         // this tile's image size
  size_t pbase;     // its first pixel in the (packed) per-pixel buffers
  const float* bg;
  __device__ __forceinline__ BwdPixel(const BackwardArgs& a, int tile_, int local_tile, int W_, int H_, size_t pbase_,
                                      const float* bg_)
      : tile(tile_), tp(local_tile, (W_ + kTile - 1) / kTile), W(W_), H(H_), pbase(pbase_), bg(bg_) {
    inside = tp.px < W && tp.py < H;
    range = a.ranges[tile];
    hw = size_t(W) * H;
    pix = inside ? pbase + size_t(tp.py) * W + tp.px : 0;
    last = inside ? a.n_contrib[pix] : 0u;
    warp_last = __reduce_max_sync(0xffffffffu, last);
    walk = int(min(warp_last, range.y - range.x));
    if (inside) {
      // colour planes: an image's three planes sit together at 3 * pbase
      const size_t cp = 3 * pbase + (pix - pbase);
      dLp0 = a.dL_dcolor[cp];
      dLp1 = a.dL_dcolor[hw + cp];
      dLp2 = a.dL_dcolor[2 * hw + cp];
      dLd = a.dL_ddepth != nullptr ? a.dL_ddepth[pix] : 0.f;  // absent: no loss on depth / alpha
      dLa = a.dL_dalpha != nullptr ? a.dL_dalpha[pix] : 0.f;
    }
  }
};

// Reference formulas (backward.cu:552-663), per pixel, for one entry:
// q0 = (mx, my, conic a, conic b), q1 = (conic c, opacity, depth, r), q2 = (g, b, skip, _).
// kDA: a loss reaches depth or alpha.  Without one (dL/ddepth and dL/dalpha
// absent, read as zero) every depth and alpha term adds exactly zero, so
// RefChain<false> leaves them out (the suffix depth and alpha, their terms of
// dL/dopacity, the depth contribution): the same results with about 7 % fewer
// instructions per pair.
template <bool kDA>
struct RefChain {
  float T, T_final, bg_dot;
  float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc_d = 0.f, acc_a = 0.f;
  float last_alpha = 0.f, lc0 = 0.f, lc1 = 0.f, lc2 = 0.f, last_depth = 0.f;

  // The state after entry (opacity-weighted alpha `alpha`, colour in q1.w,
  // q2.x, q2.y, depth q1.z).  T in [~1e-4, 1] (the forward stops before
  // T < 1e-4) and 1 - alpha in [0.01, 1]: the division is in div_markstein's
  // range, which equals /.
  struct Next {
    float Tn, n0, n1, n2, nd, na, y;  // y: RN(1 / (1 - alpha)), shared by the step's two quotients
  };
  __device__ __forceinline__ Next next(float alpha) const {
    Next x;
    x.y = rcp_markstein(1.f - alpha);
    x.Tn = div_markstein_y(T, 1.f - alpha, x.y);
    x.n0 = last_alpha * lc0 + (1.f - last_alpha) * acc0;
    x.n1 = last_alpha * lc1 + (1.f - last_alpha) * acc1;
    x.n2 = last_alpha * lc2 + (1.f - last_alpha) * acc2;
    if constexpr (kDA) {
      x.nd = last_alpha * last_depth + (1.f - last_alpha) * acc_d;
      x.na = last_alpha + (1.f - last_alpha) * acc_a;
    } else {
      x.nd = 0.f;
      x.na = 0.f;
    }
    return x;
  }
  __device__ __forceinline__ void commit(bool ok, const Next& x, float4 q1, float4 q2, float alpha) {
    if (ok) {
      T = x.Tn;
      acc0 = x.n0; acc1 = x.n1; acc2 = x.n2;
      lc0 = q1.w; lc1 = q2.x; lc2 = q2.y;
      if constexpr (kDA) {
        acc_d = x.nd; acc_a = x.na;
        last_depth = q1.z;
      }
      last_alpha = alpha;
    }
  }
  // State only (the walk of a later segment's prefix, see render_ref_kernel).
  __device__ __forceinline__ void advance(bool ok, float4 q1, float4 q2, float alpha) {
    commit(ok, next(alpha), q1, q2, alpha);
  }

  // ok false: the entry is skipped (state unchanged, contributions zero).
  __device__ __forceinline__ void step(bool ok, const BwdPixel& p, float4 q0, float4 q1, float4 q2, float dx, float dy,
                                       float G, float alpha, float ddelx_dx, float ddely_dy, float (&c)[kValues]) {
    const Next x = next(alpha);
    const float Tn = x.Tn, n0 = x.n0, n1 = x.n1, n2 = x.n2, nd = x.nd, na = x.na;
    // a skipped entry's contributions are zeroed through three of their
    // factors: alpha <= 0.99 and T_final / T finite keep dL_dopa finite, and
    // the conic (inverse of a covariance with +0.3 on its diagonal) keeps dx,
    // dy and the products finite, so each contribution is exactly +-0
    const float dchdc = ok ? alpha * Tn : 0.f;
    float dL_dopa = 0.0f;
    dL_dopa += (q1.w - n0) * p.dLp0;
    dL_dopa += (q2.x - n1) * p.dLp1;
    dL_dopa += (q2.y - n2) * p.dLp2;
    if constexpr (kDA) {
      const float c_d = q1.z;
      dL_dopa += (c_d - nd) * p.dLd;
      dL_dopa += (1 - na) * p.dLa;
    }
    dL_dopa *= Tn;
    dL_dopa += div_markstein_y(-T_final, 1.f - alpha, x.y) * bg_dot;
    const float Gz = ok ? G : 0.f;  // G itself may be infinite where the entry is skipped
    const float dL_dG = ok ? q1.y * dL_dopa : 0.f;
    const float gdx = Gz * dx, gdy = Gz * dy;
    const float dG_ddelx = -gdx * q0.z - gdy * q0.w;
    const float dG_ddely = -gdy * q1.x - gdx * q0.w;
    c[0] = dchdc * p.dLp0;
    c[1] = dchdc * p.dLp1;
    c[2] = dchdc * p.dLp2;
    c[3] = kDA ? dchdc * p.dLd : 0.f;
    c[4] = dL_dG * dG_ddelx * ddelx_dx;
    c[5] = dL_dG * dG_ddely * ddely_dy;
    c[6] = -0.5f * gdx * dx * dL_dG;
    c[7] = -0.5f * gdx * dy * dL_dG;
    c[8] = -0.5f * gdy * dy * dL_dG;
    c[9] = Gz * dL_dopa;
    commit(ok, x, q1, q2, alpha);
  }
};

// The reference's pair test and Gaussian value: power from the conic, skipped
// when positive or (certainly) below alpha 1/255, alpha = min(0.99, o G).
__device__ __forceinline__ bool ref_eval(float4 q0, float4 q1, float4 q2, float pxf, float pyf, float& dx, float& dy,
                                         float& G, float& alpha) {
  dx = q0.x - pxf;
  dy = q0.y - pyf;
  const float power = -0.5f * (q0.z * dx * dx + q1.x * dy * dy) - q0.w * dx * dy;
  G = expf(power);
  alpha = fminf(0.99f, q1.y * G);
  return power <= 0.0f && power >= q2.z && alpha >= 1.0f / 255.0f;
}

// Walk list positions [lo, top) back to front, kChunk at a time; body(bits,
// hi) handles one staged chunk whose entry j is list position hi - 1 - j and
// whose set bits are the entries that may reach this warp's block.
// wmask / wbit: the warp's block-mask array and bit (the blend's masks), or null.
template <typename Body>
__device__ __forceinline__ void walk_back(const float* records, const uint32_t* point_list, uint32_t num_records,
                                          const uint8_t* wmask, int wbit, uint32_t base, int lo, int top,
                                          WarpChunk& wc, const TilePixel& tp, Body&& body) {
  const int len = top - lo;
  const int nc = len > 0 ? (len + kChunk - 1) / kChunk : 0;
  ChunkLoad ld;
  uint32_t reach = 0;
  if (nc > 0) {
    chunk_load(ld, records, point_list, base + top - 1 - tp.lane, tp.lane < len, num_records, wmask, wbit);
    reach = chunk_store(wc, ld, tp.bx, tp.by);
  }
  for (int c = 0; c < nc; ++c) {
    const int hi = top - c * kChunk;
    const int hn = hi - kChunk;
    const bool more = c + 1 < nc;
    if (more)
      chunk_load(ld, records, point_list, base + hn - 1 - tp.lane, hn - 1 - tp.lane >= lo, num_records, wmask,
                 wbit);
    body(reach, hi);
    if (more) {
      __syncwarp();
      reach = chunk_store(wc, ld, tp.bx, tp.by);
    }
  }
}

// CTA b's tile and segment: the first kSplitWays * split CTAs are the
// segments of the `split` heaviest tiles (segment 0..kSplitWays-1), the rest
// one whole tile each (segment -1), heaviest first.
// Pixel-loop prologue for CTA blockIdx.x: its tile's image (the call's, or its
// batch item's) and segment role.
__device__ __forceinline__ BwdPixel make_bwd_pixel(const BackwardArgs& a, int tile, const float*& bg) {
  if (a.items == nullptr) {
    bg = a.bg;
    return BwdPixel(a, tile, tile, a.W, a.H, 0, a.bg);
  }
  const BatchItem& it = a.items[find_item_tile(a.items, a.num_items, uint32_t(tile))];
  bg = it.bg;
  return BwdPixel(a, tile, tile - int(it.tile_base), it.W, it.H, size_t(it.pix_base), it.bg);
}

template <int kSplitWays>
__device__ __forceinline__ int cta_tile(const BackwardArgs& a, int& seg) {
  const int b = int(blockIdx.x);
  if (b < kSplitWays * a.split) {
    seg = b % kSplitWays;
    return int(a.order_bwd[b / kSplitWays]);
  }
  seg = -1;
  return int(a.order_bwd[b - (kSplitWays - 1) * a.split]);
}

template <int kSplitWays, bool kDA>
__global__ void __launch_bounds__(kBlendThreads, 2) render_ref_kernel(BackwardArgs a) {
  __shared__ WarpChunk s_chunk[kBlendThreads / 32];
  int role;
  const int gtile = cta_tile<kSplitWays>(a, role);
  const float* bgp;
  const BwdPixel p = make_bwd_pixel(a, gtile, bgp);
  RefChain<kDA> ch;
  ch.T_final = p.inside ? 1.0f - a.out_alpha[p.pix] : 0.0f;
  ch.T = ch.T_final;
  ch.bg_dot = bgp[0] * p.dLp0 + bgp[1] * p.dLp1 + bgp[2] * p.dLp2;
  const float ddelx_dx = 0.5f * float(p.W), ddely_dy = 0.5f * float(p.H);
  const float pxf = float(p.tp.px), pyf = float(p.tp.py);
  const Target tgt = lane_target(a, 0);
  const Target tgt2 = lane_target_pair(a, 0);
  WarpChunk& wc = s_chunk[threadIdx.x >> 5];
  // the blend's block masks, when this binning state has them: warps 0-3 read
  // the top array, 4-7 the bottom one, bit = block within that half
  const bool use_masks = a.masks_valid != nullptr && *a.masks_valid != 0u;
  const uint8_t* wmask = use_masks ? ((threadIdx.x >> 5) < 4 ? a.mask_top : a.mask_bottom) : nullptr;
  const int wbit = int(threadIdx.x >> 5) & 3;
  const float4* s = wc.rec;
  auto full = [&](uint32_t bits, int hi) {
    while (bits != 0u) {
      const int j0 = pop_entry(bits);
      const int j1r = pop_entry(bits);
      const bool has1 = j1r >= 0;
      const int j1 = has1 ? j1r : j0;
      const float4 a0 = s[kRecVec * j0], a1 = s[kRecVec * j0 + 1], a2 = s[kRecVec * j0 + 2];
      const float4 b0 = s[kRecVec * j1], b1 = s[kRecVec * j1 + 1], b2 = s[kRecVec * j1 + 2];
      float dx0, dy0, G0, al0, dx1, dy1, G1, al1;
      const bool ok0 = ref_eval(a0, a1, a2, pxf, pyf, dx0, dy0, G0, al0) && uint32_t(hi - 1 - j0) < p.last;
      const bool ok1 = ref_eval(b0, b1, b2, pxf, pyf, dx1, dy1, G1, al1) && has1 &&
                       uint32_t(hi - 1 - j1) < p.last;
      float c0[kValues], c1[kValues];
      ch.step(ok0, p, a0, a1, a2, dx0, dy0, G0, al0, ddelx_dx, ddely_dy, c0);
      ch.step(ok1, p, b0, b1, b2, dx1, dy1, G1, al1, ddelx_dx, ddely_dy, c1);
      flush_pair(c0, c1, ok0, ok1, wc.id[j0], wc.id[j1], tgt, tgt2);
    }
  };
  auto state_only = [&](uint32_t bits, int hi) {
    while (bits != 0u) {
      const int j0 = pop_entry(bits);
      const int j1r = pop_entry(bits);
      const bool has1 = j1r >= 0;
      const int j1 = has1 ? j1r : j0;
      const float4 a0 = s[kRecVec * j0], a1 = s[kRecVec * j0 + 1], a2 = s[kRecVec * j0 + 2];
      const float4 b0 = s[kRecVec * j1], b1 = s[kRecVec * j1 + 1], b2 = s[kRecVec * j1 + 2];
      float dx0, dy0, G0, al0, dx1, dy1, G1, al1;
      const bool ok0 = ref_eval(a0, a1, a2, pxf, pyf, dx0, dy0, G0, al0) && uint32_t(hi - 1 - j0) < p.last;
      const bool ok1 = ref_eval(b0, b1, b2, pxf, pyf, dx1, dy1, G1, al1) && has1 &&
                       uint32_t(hi - 1 - j1) < p.last;
      ch.advance(ok0, a1, a2, al0);
      ch.advance(ok1, b1, b2, al1);
    }
  };
  if (role < 0) {
    walk_back(a.bwd_record, a.point_list, uint32_t(a.P), wmask, wbit, p.range.x, 0, p.walk, wc, p.tp, full);
  } else {
    int lo, hi;
    segment_of<kSplitWays>(p.walk, role, lo, hi);
    walk_back(a.bwd_record, a.point_list, uint32_t(a.P), wmask, wbit, p.range.x, hi, p.walk, wc, p.tp, state_only);
    __syncwarp();
    walk_back(a.bwd_record, a.point_list, uint32_t(a.P), wmask, wbit, p.range.x, lo, hi, wc, p.tp, full);
  }
}

// The forward's Gaussian value (blend.cu), split at its division so that a
// warp's divisions can run branch-free together.
__device__ __forceinline__ float gauss_num_fwd(float px, float py, float mx, float my, float cxx, float cxy,
                                               float cyy) {
  using namespace fp;
  const float dx = sub(px, mx), dy = sub(py, my);
  const float tX = d2<BL_TX>(dx, cyy, dy, cxy);
  const float tY = s2<BL_TY>(-dx, cxy, dy, cxx);
  return s2<BL_NUM>(tX, dx, tY, dy);
}

// Exact derivative of the forward blend, per pixel, for one entry:
// q0 = (mx, my, cxx, cxy), q1 = (cyy, det, opacity, depth), q2 = (r, g, b, _).
struct ExactChain {
  float T;
  float S0, S1, S2, SD = 0.f, SW = 0.f;  // suffix sums behind the current entry (colour includes the background)

  // State only (the walk of a later segment's prefix).
  __device__ __forceinline__ void advance(bool ok, float4 q1, float4 q2, float a_) {
    const float ia = rcp_markstein(1.0f - a_);
    const float Tn = T * ia;
    const float aT = a_ * Tn;
    if (ok) {
      T = Tn;
      S0 += q2.x * aT;
      S1 += q2.y * aT;
      S2 += q2.z * aT;
      SD += q1.w * aT;
      SW += aT;
    }
  }

  // ok false: the entry is skipped (state unchanged, contributions zero).
  __device__ __forceinline__ void step(bool ok, const BwdPixel& p, float4 q0, float4 q1, float4 q2, float pxf,
                                       float pyf, float g, float og, float a_, float mahal, float hW, float hH,
                                       float (&c)[kValues]) {
    const float ia = rcp_markstein(1.0f - a_);  // 1 - alpha in [0.01, 1]
    const float Tn = T * ia;  // transmittance in front of this entry
    const float aT = a_ * Tn;
    float dLda = p.dLp0 * (q2.x * Tn - S0 * ia) + p.dLp1 * (q2.y * Tn - S1 * ia) + p.dLp2 * (q2.z * Tn - S2 * ia);
    dLda += p.dLd * (q1.w * Tn - SD * ia);
    dLda += p.dLa * (Tn - SW * ia);
    // skipped entries' contributions are zeroed through one factor each:
    // 1 - alpha >= 0.01, g <= 1, det >= 0.09 and the mahalanobis distance
    // (a quotient by det) keep every other factor finite
    const float aTz = ok ? aT : 0.f;
    c[0] = aTz * p.dLp0;
    c[1] = aTz * p.dLp1;
    c[2] = aTz * p.dLp2;
    c[3] = aTz * p.dLd;
    if (ok) {
      T = Tn;
      S0 += q2.x * aT;
      S1 += q2.y * aT;
      S2 += q2.z * aT;
      SD += q1.w * aT;
      SW += aT;
    }
    const bool unclamped = ok && og < 0.99f;
    c[9] = dLda * (unclamped ? g : 0.f);
    const bool inner = unclamped && mahal >= 0.0f;
    const float dLdm = inner ? dLda * q1.z * (-0.5f * g) : 0.f;
    const float cxx = q0.z, cxy = q0.w, cyy = q1.x, det = q1.y;
    const float dx = pxf - q0.x, dy = pyf - q0.y;
    // det >= 0.09 (the forward's +0.3 low-pass on a positive semi-definite
    // covariance), where rcp_markstein is the correctly rounded 1/det
    const float idet = rcp_markstein(det);
    const float num = mahal * det;
    c[4] = -dLdm * (2.f * cyy * dx - 2.f * cxy * dy) * idet * hW;
    c[5] = -dLdm * (2.f * cxx * dy - 2.f * cxy * dx) * idet * hH;
    c[6] = dLdm * (dy * dy * idet - num * cyy * idet * idet);
    c[7] = dLdm * (-2.f * dx * dy * idet + 2.f * num * cxy * idet * idet);
    c[8] = dLdm * (dx * dx * idet - num * cxx * idet * idet);
  }
};

template <int kSplitWays>
__global__ void __launch_bounds__(kBlendThreads, 2) render_exact_kernel(BackwardArgs a) {
  __shared__ WarpChunk s_chunk[kBlendThreads / 32];
  int role;
  const int gtile = cta_tile<kSplitWays>(a, role);
  const float* bgp;
  const BwdPixel p = make_bwd_pixel(a, gtile, bgp);
  ExactChain ch;
  const float Tf = p.inside ? a.T_final[p.pix] : 0.0f;
  ch.T = Tf;
  ch.S0 = Tf * bgp[0];
  ch.S1 = Tf * bgp[1];
  ch.S2 = Tf * bgp[2];
  const float hW = 0.5f * float(p.W), hH = 0.5f * float(p.H);
  const float pxf = float(p.tp.px), pyf = float(p.tp.py);
  const Target tgt = lane_target(a, 1);
  const Target tgt2 = lane_target_pair(a, 1);
  WarpChunk& wc = s_chunk[threadIdx.x >> 5];
  // the blend's block masks, when this binning state has them: warps 0-3 read
  // the top array, 4-7 the bottom one, bit = block within that half
  const bool use_masks = a.masks_valid != nullptr && *a.masks_valid != 0u;
  const uint8_t* wmask = use_masks ? ((threadIdx.x >> 5) < 4 ? a.mask_top : a.mask_bottom) : nullptr;
  const int wbit = int(threadIdx.x >> 5) & 3;
  const float4* s = wc.rec;
  // the forward's Gaussian values of two entries (same division as the blend)
  auto eval2 = [&](int j0, int j1, float& m0, float& m1, float& g0, float& g1) {
    const float4 a0 = s[kRecVec * j0], a1 = s[kRecVec * j0 + 1];
    const float4 b0 = s[kRecVec * j1], b1 = s[kRecVec * j1 + 1];
    const float n0 = gauss_num_fwd(pxf, pyf, a0.x, a0.y, a0.z, a0.w, a1.x);
    const float n1 = gauss_num_fwd(pxf, pyf, b0.x, b0.y, b0.z, b0.w, b1.x);
    if (__all_sync(0xffffffffu, div_in_range(n0, a1.y) && div_in_range(n1, b1.y))) {
      m0 = div_markstein(n0, a1.y);
      m1 = div_markstein(n1, b1.y);
    } else {
      m0 = div(n0, a1.y);
      m1 = div(n1, b1.y);
    }
    g0 = expf(mul(-0.5f, m0 < 0.0f ? 1000.0f : m0));
    g1 = expf(mul(-0.5f, m1 < 0.0f ? 1000.0f : m1));
  };
  auto full = [&](uint32_t bits, int hi) {
    while (bits != 0u) {
      const int j0 = pop_entry(bits);
      const int j1r = pop_entry(bits);
      const bool has1 = j1r >= 0;
      const int j1 = has1 ? j1r : j0;
      float m0, m1, g0, g1;
      eval2(j0, j1, m0, m1, g0, g1);
      const float4 a0 = s[kRecVec * j0], a1 = s[kRecVec * j0 + 1];
      const float4 b0 = s[kRecVec * j1], b1 = s[kRecVec * j1 + 1];
      const float og0 = mul(a1.z, g0), og1 = mul(b1.z, g1);
      const float al0 = fminf(0.99f, og0), al1 = fminf(0.99f, og1);
      const bool ok0 = al0 >= 1.0f / 255.0f && uint32_t(hi - 1 - j0) < p.last;
      const bool ok1 = al1 >= 1.0f / 255.0f && has1 && uint32_t(hi - 1 - j1) < p.last;
      float c0[kValues], c1[kValues];
      ch.step(ok0, p, a0, a1, s[kRecVec * j0 + 2], pxf, pyf, g0, og0, al0, m0, hW, hH, c0);
      ch.step(ok1, p, b0, b1, s[kRecVec * j1 + 2], pxf, pyf, g1, og1, al1, m1, hW, hH, c1);
      flush_pair(c0, c1, ok0, ok1, wc.id[j0], wc.id[j1], tgt, tgt2);
    }
  };
  auto state_only = [&](uint32_t bits, int hi) {
    while (bits != 0u) {
      const int j0 = pop_entry(bits);
      const int j1r = pop_entry(bits);
      const bool has1 = j1r >= 0;
      const int j1 = has1 ? j1r : j0;
      float m0, m1, g0, g1;
      eval2(j0, j1, m0, m1, g0, g1);
      const float4 a1 = s[kRecVec * j0 + 1], b1 = s[kRecVec * j1 + 1];
      const float al0 = fminf(0.99f, mul(a1.z, g0)), al1 = fminf(0.99f, mul(b1.z, g1));
      const bool ok0 = al0 >= 1.0f / 255.0f && uint32_t(hi - 1 - j0) < p.last;
      const bool ok1 = al1 >= 1.0f / 255.0f && has1 && uint32_t(hi - 1 - j1) < p.last;
      ch.advance(ok0, a1, s[kRecVec * j0 + 2], al0);
      ch.advance(ok1, b1, s[kRecVec * j1 + 2], al1);
    }
  };
  if (role < 0) {
    walk_back(a.record, a.point_list, uint32_t(a.P), wmask, wbit, p.range.x, 0, p.walk, wc, p.tp, full);
  } else {
    int lo, hi;
    segment_of<kSplitWays>(p.walk, role, lo, hi);
    walk_back(a.record, a.point_list, uint32_t(a.P), wmask, wbit, p.range.x, hi, p.walk, wc, p.tp, state_only);
    __syncwarp();
    walk_back(a.record, a.point_list, uint32_t(a.P), wmask, wbit, p.range.x, lo, hi, wc, p.tp, full);
  }
}

// ---------------------------------------------------------------------------
// Per-Gaussian passes: one thread per Gaussian, with the SH rows (up to 48
// floats each) moved between global and shared memory by the whole warp, so
// that global loads and stores are contiguous 128-byte runs instead of one
// 192-byte-strided row per thread.
// ---------------------------------------------------------------------------
constexpr int kGaussThreads = 128;

__device__ __forceinline__ int sh_stride(int M) {
  const int r = 3 * (M < 16 ? M : 16);
  return r | 1;
}

// Rows [i0, i0 + n) of shs ([P, M, 3]), first min(M, 16) coefficients, into
// s (row g at g * stride).  Warp-collective.
__device__ __forceinline__ void sh_stage_in(const float* shs, int M, int i0, int n, float* s, int stride) {
  constexpr int kInFlight = 8;  // loads issued before their stores
  const int rs = 3 * (M < 16 ? M : 16), rg = 3 * M, lane = threadIdx.x & 31;
  if (M == 16 && n == 32 && aligned16(shs)) {
    stage_span(shs + size_t(i0) * 48, 48, s, stride, 0);
    __syncwarp();
    return;
  }
  if (rs > 0) {
    const int total = n * rs;
    int g = 0, c = lane;
    while (c >= rs) { c -= rs; ++g; }
    for (int e0 = 0; e0 < total; e0 += 32 * kInFlight) {
      float v[kInFlight];
      int dst[kInFlight];
#pragma unroll
      for (int k = 0; k < kInFlight; ++k) {
        const bool ok = e0 + 32 * k + lane < total;
        v[k] = ok ? __ldg(shs + size_t(i0 + g) * rg + c) : 0.f;
        dst[k] = ok ? g * stride + c : -1;
        c += 32;
        while (c >= rs) { c -= rs; ++g; }
      }
#pragma unroll
      for (int k = 0; k < kInFlight; ++k)
        if (dst[k] >= 0) s[dst[k]] = v[k];
    }
  }
  __syncwarp();
}

// Write the span of 32 rows of `len` floats at dst: row g's element c is
// coefficient (c + off) / 3, channel (c + off) % 3 of Gaussian g, the product of
// its basis value and colour factor in s (row g at g * 21: 16 basis, 3 factors).
__device__ __forceinline__ void store_span(float* dst, int len, const float* s, int off) {
  const int lane = threadIdx.x & 31, nf = 8 * len;
  float4* q = reinterpret_cast<float4*>(dst);
  for (int f = lane; f < nf; f += 32) {
    int g = (4 * f) / len, c = 4 * f - g * len;
    float o[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const int e = c + off, k = e / 3, ch = e - 3 * k;
      o[w] = s[g * 21 + k] * s[g * 21 + 16 + ch];
      if (++c == len) {
        c = 0;
        ++g;
      }
    }
    q[f] = make_float4(o[0], o[1], o[2], o[3]);
  }
}

// dsh rows [i0, i0 + n) ([P, M, 3]) = basis[k] * cf[ch] (k < 16; 0 beyond),
// written contiguously; each thread's factors pass through s.  Warp-collective.
__device__ __forceinline__ void sh_store_outer(float* dsh, int M, int i0, int n, float* s, const float (&basis)[16],
                                               const float (&cf)[3], bool active) {
  constexpr int kRow = 21;  // 16 basis + 3 colour factors, odd stride
  const int lane = threadIdx.x & 31, rg = 3 * M;
  __syncwarp();  // the SH rows in s have been read
#pragma unroll
  for (int k = 0; k < 16; ++k) s[lane * kRow + k] = active ? basis[k] : 0.f;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) s[lane * kRow + 16 + ch] = active ? cf[ch] : 0.f;
  __syncwarp();
  if (M == 16 && n == 32 && aligned16(dsh)) {
    store_span(dsh + size_t(i0) * 48, 48, s, 0);
    return;
  }
  if (rg > 0) {
    constexpr int kInFlight = 8;
    const int total = n * rg;
    int g = 0, c = lane;
    while (c >= rg) { c -= rg; ++g; }
    for (int e0 = 0; e0 < total; e0 += 32 * kInFlight) {
      float v[kInFlight];
      size_t dst[kInFlight];
#pragma unroll
      for (int q = 0; q < kInFlight; ++q) {
        const int k = c / 3, ch = c - 3 * k;
        const bool ok = e0 + 32 * q + lane < total;
        v[q] = ok && k < 16 ? s[g * kRow + k] * s[g * kRow + 16 + ch] : 0.f;
        dst[q] = ok ? size_t(i0 + g) * rg + c : ~size_t(0);
        c += 32;
        while (c >= rg) { c -= rg; ++g; }
      }
#pragma unroll
      for (int q = 0; q < kInFlight; ++q)
        if (dst[q] != ~size_t(0)) dsh[dst[q]] = v[q];
    }
  }
}

// The raw path's SH rows: coefficient 0 from sh_dc ([P, 1, 3]), the rest from
// sh_ac ([P, M - 1, 3]).  Same staging as sh_stage_in.  Warp-collective.
__device__ __forceinline__ void sh_stage_in_raw(const float* dc, const float* ac, int M, int i0, int n, float* s,
                                                int stride) {
  constexpr int kInFlight = 8;
  const int rs = 3 * (M < 16 ? M : 16), ra = 3 * (M - 1), lane = threadIdx.x & 31;
  if (M == 16 && n == 32 && aligned16(dc) && aligned16(ac)) {
    stage_span(dc + size_t(i0) * 3, 3, s, stride, 0);
    stage_span(ac + size_t(i0) * 45, 45, s, stride, 3);
    __syncwarp();
    return;
  }
  if (rs > 0) {
    const int total = n * rs;
    int g = 0, c = lane;
    while (c >= rs) { c -= rs; ++g; }
    for (int e0 = 0; e0 < total; e0 += 32 * kInFlight) {
      float v[kInFlight];
      int dst[kInFlight];
#pragma unroll
      for (int k = 0; k < kInFlight; ++k) {
        const bool ok = e0 + 32 * k + lane < total;
        v[k] = !ok ? 0.f : c < 3 ? __ldg(dc + size_t(i0 + g) * 3 + c) : __ldg(ac + size_t(i0 + g) * ra + (c - 3));
        dst[k] = ok ? g * stride + c : -1;
        c += 32;
        while (c >= rs) { c -= rs; ++g; }
      }
#pragma unroll
      for (int k = 0; k < kInFlight; ++k)
        if (dst[k] >= 0) s[dst[k]] = v[k];
    }
  }
  __syncwarp();
}

// sh_store_outer for the raw path: coefficient 0 to ddc, the rest to dac.
__device__ __forceinline__ void sh_store_outer_raw(float* ddc, float* dac, int M, int i0, int n, float* s,
                                                   const float (&basis)[16], const float (&cf)[3], bool active) {
  constexpr int kRow = 21;
  const int lane = threadIdx.x & 31, rg = 3 * M, ra = 3 * (M - 1);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 16; ++k) s[lane * kRow + k] = active ? basis[k] : 0.f;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) s[lane * kRow + 16 + ch] = active ? cf[ch] : 0.f;
  __syncwarp();
  if (M == 16 && n == 32 && aligned16(ddc) && aligned16(dac)) {
    store_span(ddc + size_t(i0) * 3, 3, s, 0);
    store_span(dac + size_t(i0) * 45, 45, s, 3);
    return;
  }
  if (rg > 0) {
    constexpr int kInFlight = 8;
    const int total = n * rg;
    int g = 0, c = lane;
    while (c >= rg) { c -= rg; ++g; }
    for (int e0 = 0; e0 < total; e0 += 32 * kInFlight) {
      float v[kInFlight];
      float* dst[kInFlight];
#pragma unroll
      for (int q = 0; q < kInFlight; ++q) {
        const int k = c / 3, ch = c - 3 * k;
        const bool ok = e0 + 32 * q + lane < total;
        v[q] = ok && k < 16 ? s[g * kRow + k] * s[g * kRow + 16 + ch] : 0.f;
        dst[q] = !ok ? nullptr : c < 3 ? ddc + size_t(i0 + g) * 3 + c : dac + size_t(i0 + g) * ra + (c - 3);
        c += 32;
        while (c >= rg) { c -= rg; ++g; }
      }
#pragma unroll
      for (int q = 0; q < kInFlight; ++q)
        if (dst[q] != nullptr) *dst[q] = v[q];
    }
  }
}

// A batched call's SH rows of the warp's elements [i0, i0 + n): one scene's
// contiguous rows when all n belong to one item (sh_stage_in's spans), else
// each thread its own row (the warp spans scenes).  Warp-collective.
__device__ __forceinline__ void batch_sh_stage_in(const BackwardArgs& a, int i0, int n, float* s, int stride) {
  const int lane = threadIdx.x & 31;
  const int first = find_item_elem(a.items, a.num_items, uint32_t(i0));
  const int last = find_item_elem(a.items, a.num_items, uint32_t(i0 + n - 1));
  if (first == last) {
    const BatchItem& it = a.items[first];
    sh_stage_in(it.shs, a.M, i0 - int(it.elem_base), n, s, stride);
    return;
  }
  const int rs = 3 * (a.M < 16 ? a.M : 16);
  if (lane < n) {
    const int i = i0 + lane;
    const BatchItem& it = a.items[find_item_elem(a.items, a.num_items, uint32_t(i))];
    const float* row = it.shs + size_t(i - int(it.elem_base)) * 3 * a.M;
    for (int c = 0; c < rs; ++c) s[lane * stride + c] = __ldg(row + c);
  }
  __syncwarp();
}

// Per-Gaussian, reference formulas (backward.cu:27-227 then :229-519)
__constant__ float kSH_C2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                                -1.0925484305920792f, 0.5462742152960396f};
__constant__ float kSH_C3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                                0.3731763325901154f,  -0.4570457994644658f, 1.445305721320277f,
                                -0.5900435899266435f};

// The scene and camera of one element: the call's, or its batch item's.
struct GView {
  const float* means3D;
  const float* scales;
  const float* rotations;
  const float* mats;  // view (16), projection (16), camera position (3)
  int gi;             // index within the scene
  int W, degree;
  float h_x, h_y, tan_fovx, tan_fovy, focal_x, scale_modifier;
  const float* svec = nullptr;  // raw scales / quaternions (then scales / rotations are unused)
  const float* quat = nullptr;

  // the activated scale k and rotation (w, x, y, z).  The raw path's
  // rotation multiplies by the reciprocal of the clamped norm (the forward
  // divides, bit-exact with torch; here it only enters gradients, and the two
  // differ by at most an ulp)
  __device__ __forceinline__ float scale(int k) const {
    return svec != nullptr ? expf(__ldg(&svec[3 * gi + k])) : __ldg(&scales[3 * gi + k]);
  }
  __device__ __forceinline__ float4 rotation() const {
    if (quat != nullptr) {
      const float w = __ldg(&quat[4 * gi]), x = __ldg(&quat[4 * gi + 1]), y = __ldg(&quat[4 * gi + 2]),
                  z = __ldg(&quat[4 * gi + 3]);
      const float inv = __frcp_rn(fmaxf(sqrtf((w * w + y * y) + (x * x + z * z)), 1e-12f));
      return make_float4(w * inv, x * inv, y * inv, z * inv);
    }
    return make_float4(__ldg(&rotations[4 * gi]), __ldg(&rotations[4 * gi + 1]), __ldg(&rotations[4 * gi + 2]),
                       __ldg(&rotations[4 * gi + 3]));
  }
};

// Element i (global index) of batch item `it`.
__device__ __forceinline__ GView item_gview(const BatchItem& it, int i) {
  return GView{it.means3D, it.scales, it.rotations, it.view, i - int(it.elem_base), it.W, it.degree, it.h_x, it.h_y,
               it.tan_fovx, it.tan_fovy, it.h_x, it.scale_modifier};
}

__device__ __forceinline__ GView make_gview(const BackwardArgs& a, int i, const float* s_mats) {
  GView g;
  if (a.items == nullptr) {
    g = GView{a.means3D, a.scales, a.rotations, s_mats, i, a.W, a.degree, a.h_x, a.h_y, a.tan_fovx, a.tan_fovy,
              a.focal_x, a.scale_modifier};
    g.svec = a.svec;
    g.quat = a.quat;
  } else {
    g = item_gview(a.items[find_item_elem(a.items, a.num_items, uint32_t(i))], i);
  }
  return g;
}

// The per-Gaussian outputs of one element (kept in registers; the kernels
// store them, or sum them over a group's views).
struct GOut {
  float m3[3], cov[6], sc[3], rot[4];
};

__device__ __forceinline__ void store_gout(const BackwardArgs& a, int i, const GOut& o) {
  for (int k = 0; k < 3; ++k) a.dL_dmeans3D[3 * i + k] = o.m3[k];
  for (int k = 0; k < 6; ++k) a.dL_dcov3D[6 * i + k] = o.cov[k];
  for (int k = 0; k < 3; ++k) a.dL_dscales[3 * i + k] = o.sc[k];
  for (int k = 0; k < 4; ++k) a.dL_drotations[4 * i + k] = o.rot[k];
}

// One Gaussian (radius > 0) of the reference-formula pass: every output but
// dL_dsh, plus the SH basis and masked colour gradient dL_dsh is built from.
// sh_row: this Gaussian's SH coefficients (staged in shared memory).
__device__ __forceinline__ void ref_gaussian(const BackwardArgs& a, int i, const GView& gv, const float* sh_row, float (&basis)[16],
                                             float (&cf)[3], GOut& o) {
  const int M = a.M;
  const float* mats = gv.mats;
  const float* cam = mats + 32;
  const float* view = mats;
  const float* proj = mats + 16;
  const float cx = __ldg(&gv.means3D[3 * gv.gi]), cy = __ldg(&gv.means3D[3 * gv.gi + 1]), cz = __ldg(&gv.means3D[3 * gv.gi + 2]);
  const float* pc = a.cov3D + 6 * size_t(i);  // read with __ldg below

  // ---- computeCov2DCUDA ----
  float vx = view[0] * cx + view[4] * cy + view[8] * cz + view[12];
  float vy = view[1] * cx + view[5] * cy + view[9] * cz + view[13];
  float vz = view[2] * cx + view[6] * cy + view[10] * cz + view[14];
  const float vw = view[3] * cx + view[7] * cy + view[11] * cz + view[15];
  const float w_inv = 1.0f / (vw + 1e-8f);
  vx *= w_inv;
  vy *= w_inv;
  vz *= w_inv;
  const float bound_x = 1.3f * gv.tan_fovx, bound_y = 1.3f * gv.tan_fovy;
  const float proj_x = vx / vz, proj_y = vy / vz;
  const float cpx = fminf(bound_x, fmaxf(-bound_x, proj_x));
  const float cpy = fminf(bound_y, fmaxf(-bound_y, proj_y));
  const float px = cpx * vz, py = cpy * vz;
  const float mask_x = (proj_x >= -bound_x && proj_x <= bound_x) ? 1.0f : 0.0f;
  const float mask_y = (proj_y >= -bound_y && proj_y <= bound_y) ? 1.0f : 0.0f;
  const float z_inv = 1.0f / vz, z_inv2 = z_inv * z_inv;
  const float h_x = gv.h_x, h_y = gv.h_y;
  // J (glm column-major J[col][row]) and T = W * J
  const float J[3][3] = {{h_x * z_inv, 0.f, -h_x * px * z_inv2}, {0.f, h_y * z_inv, -h_y * py * z_inv2}, {0.f, 0.f, 0.f}};
  const float Wv[3][3] = {{view[0], view[4], view[8]}, {view[1], view[5], view[9]}, {view[2], view[6], view[10]}};
  const float Vk[3][3] = {{__ldg(pc + 0), __ldg(pc + 1), __ldg(pc + 2)}, {__ldg(pc + 1), __ldg(pc + 3), __ldg(pc + 4)}, {__ldg(pc + 2), __ldg(pc + 4), __ldg(pc + 5)}};
  float T[3][3], tmp[3][3], c2[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) T[c][r] = Wv[0][r] * J[c][0] + Wv[1][r] * J[c][1] + Wv[2][r] * J[c][2];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) tmp[c][r] = Vk[r][0] * T[c][0] + Vk[r][1] * T[c][1] + Vk[r][2] * T[c][2];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r) c2[c][r] = T[r][0] * tmp[c][0] + T[r][1] * tmp[c][1] + T[r][2] * tmp[c][2];
  c2[0][0] += 0.3f;
  c2[1][1] += 0.3f;
  const float ca = c2[0][0], cb = c2[0][1], cc = c2[1][1];
  const float den = ca * cc - cb * cb;
  const float dinv2 = 1.0f / (den * den + 1e-7f);
  const float gx = __ldg(&a.acc_cov[4 * i]), gy = __ldg(&a.acc_cov[4 * i + 1]), gz = __ldg(&a.acc_cov[4 * i + 3]);
  float ga = 0.f, gb = 0.f, gc = 0.f;
  float dc[6];
  if (dinv2 > 0) {
    ga = dinv2 * (-cc * cc * gx + 2.0f * cb * cc * gy + (den - ca * cc) * gz);
    gb = dinv2 * 2.0f * (cb * cc * gx - (den + 2.0f * cb * cb) * gy + ca * cb * gz);
    gc = dinv2 * (-ca * ca * gz + 2.0f * ca * cb * gy + (den - ca * cc) * gx);
    dc[0] = T[0][0] * T[0][0] * ga + T[0][0] * T[1][0] * gb + T[1][0] * T[1][0] * gc;
    dc[3] = T[0][1] * T[0][1] * ga + T[0][1] * T[1][1] * gb + T[1][1] * T[1][1] * gc;
    dc[5] = T[0][2] * T[0][2] * ga + T[0][2] * T[1][2] * gb + T[1][2] * T[1][2] * gc;
    dc[1] = 2.0f * (T[0][0] * T[0][1] * ga + (T[0][0] * T[1][1] + T[0][1] * T[1][0]) * gb * 0.5f + T[1][0] * T[1][1] * gc);
    dc[2] = 2.0f * (T[0][0] * T[0][2] * ga + (T[0][0] * T[1][2] + T[0][2] * T[1][0]) * gb * 0.5f + T[1][0] * T[1][2] * gc);
    dc[4] = 2.0f * (T[0][1] * T[0][2] * ga + (T[0][1] * T[1][2] + T[0][2] * T[1][1]) * gb * 0.5f + T[1][1] * T[1][2] * gc);
  } else {
    for (int k = 0; k < 6; ++k) dc[k] = 0.f;
  }
  for (int k = 0; k < 6; ++k) o.cov[k] = dc[k];
  const float gT00 = 2.0f * (T[0][0] * Vk[0][0] + T[0][1] * Vk[0][1] + T[0][2] * Vk[0][2]) * ga + (T[1][0] * Vk[0][0] + T[1][1] * Vk[0][1] + T[1][2] * Vk[0][2]) * gb;
  const float gT01 = 2.0f * (T[0][0] * Vk[1][0] + T[0][1] * Vk[1][1] + T[0][2] * Vk[1][2]) * ga + (T[1][0] * Vk[1][0] + T[1][1] * Vk[1][1] + T[1][2] * Vk[1][2]) * gb;
  const float gT02 = 2.0f * (T[0][0] * Vk[2][0] + T[0][1] * Vk[2][1] + T[0][2] * Vk[2][2]) * ga + (T[1][0] * Vk[2][0] + T[1][1] * Vk[2][1] + T[1][2] * Vk[2][2]) * gb;
  const float gT10 = 2.0f * (T[1][0] * Vk[0][0] + T[1][1] * Vk[0][1] + T[1][2] * Vk[0][2]) * gc + (T[0][0] * Vk[0][0] + T[0][1] * Vk[0][1] + T[0][2] * Vk[0][2]) * gb;
  const float gT11 = 2.0f * (T[1][0] * Vk[1][0] + T[1][1] * Vk[1][1] + T[1][2] * Vk[1][2]) * gc + (T[0][0] * Vk[1][0] + T[0][1] * Vk[1][1] + T[0][2] * Vk[1][2]) * gb;
  const float gT12 = 2.0f * (T[1][0] * Vk[2][0] + T[1][1] * Vk[2][1] + T[1][2] * Vk[2][2]) * gc + (T[0][0] * Vk[2][0] + T[0][1] * Vk[2][1] + T[0][2] * Vk[2][2]) * gb;
  const float gJ00 = Wv[0][0] * gT00 + Wv[0][1] * gT01 + Wv[0][2] * gT02;
  const float gJ02 = Wv[2][0] * gT00 + Wv[2][1] * gT01 + Wv[2][2] * gT02;
  const float gJ11 = Wv[1][0] * gT10 + Wv[1][1] * gT11 + Wv[1][2] * gT12;
  const float gJ12 = Wv[2][0] * gT10 + Wv[2][1] * gT11 + Wv[2][2] * gT12;
  const float z_inv3 = z_inv2 * z_inv;
  const float gvx = mask_x * (-h_x * z_inv2 * gJ02);
  const float gvy = mask_y * (-h_y * z_inv2 * gJ12);
  const float gvz = -h_x * z_inv2 * gJ00 - h_y * z_inv2 * gJ11 + 2.0f * h_x * px * z_inv3 * gJ02 +
                    2.0f * h_y * py * z_inv3 * gJ12;
  float sd[3] = {view[0] * gvx + view[1] * gvy + view[2] * gvz, view[4] * gvx + view[5] * gvy + view[6] * gvz,
                 view[8] * gvx + view[9] * gvy + view[10] * gvz};

  // ---- backwardPreprocessingKernel ----
  const float cw = proj[3] * cx + proj[7] * cy + proj[11] * cz + proj[15];
  const float iw = 1.0f / (cw + 1e-7f);
  const float iw2 = iw * iw;
  const float ptx = (proj[0] * cx + proj[4] * cy + proj[8] * cz + proj[12]) * iw2;
  const float pty = (proj[1] * cx + proj[5] * cy + proj[9] * cz + proj[13]) * iw2;
  const float g2x = __ldg(&a.dL_dmean2D[3 * i]), g2y = __ldg(&a.dL_dmean2D[3 * i + 1]);
  sd[0] += (proj[0] * iw - proj[3] * ptx) * g2x + (proj[1] * iw - proj[3] * pty) * g2y;
  sd[1] += (proj[4] * iw - proj[7] * ptx) * g2x + (proj[5] * iw - proj[7] * pty) * g2y;
  sd[2] += (proj[8] * iw - proj[11] * ptx) * g2x + (proj[9] * iw - proj[11] * pty) * g2y;
  const float vzz = view[2] * cx + view[6] * cy + view[10] * cz + view[14];
  const float gd = __ldg(&a.acc_depth[i]);
  sd[0] += (view[2] - view[3] * vzz) * gd;
  sd[1] += (view[6] - view[7] * vzz) * gd;
  sd[2] += (view[10] - view[11] * vzz) * gd;
  // SH (all 16 bands, colour-clamp masks)
  const float ox = cx - cam[0], oy = cy - cam[1], oz = cz - cam[2];
  const float msq = ox * ox + oy * oy + oz * oz;
  const float mag = sqrtf(msq + 1e-10f);
  const float im = 1.0f / mag;
  const float x = ox * im, y = oy * im, z = oz * im;
  const float x2 = x * x, y2 = y * y, z2 = z * z, xy = x * y, xz = x * z, yz = y * z;
  const float x2my2 = x2 - y2, tx2 = 3.0f * x2, ty2 = 3.0f * y2, fz2 = 4.0f * z2, wz2 = 2.0f * z2;
  for (int ch = 0; ch < 3; ++ch) cf[ch] = __ldg(&a.dL_dcolors[3 * i + ch]) * (__ldg(&a.clamped[3 * i + ch]) ? 0.0f : 1.0f);
  const float SH_C0 = 0.28209479177387814f, SH_C1 = 0.4886025119029199f;
  basis[0] = SH_C0; basis[1] = -SH_C1 * y; basis[2] = SH_C1 * z; basis[3] = -SH_C1 * x;
  basis[4] = kSH_C2[0] * xy; basis[5] = kSH_C2[1] * yz; basis[6] = kSH_C2[2] * (wz2 - x2 - y2);
  basis[7] = kSH_C2[3] * xz; basis[8] = kSH_C2[4] * x2my2;
  basis[9] = kSH_C3[0] * y * (tx2 - y2); basis[10] = kSH_C3[1] * xy * z; basis[11] = kSH_C3[2] * y * (fz2 - x2 - y2);
  basis[12] = kSH_C3[3] * z * (wz2 - tx2 - ty2); basis[13] = kSH_C3[4] * x * (fz2 - x2 - y2);
  basis[14] = kSH_C3[5] * z * x2my2; basis[15] = kSH_C3[6] * x * (x2 - ty2);
  auto SH = [&](int k, int ch) -> float { return k < M ? sh_row[3 * k + ch] : 0.0f; };
  float ag[3] = {0.f, 0.f, 0.f};
  auto dotc = [&](int k) { return SH(k, 0) * cf[0] + SH(k, 1) * cf[1] + SH(k, 2) * cf[2]; };
  ag[0] -= SH_C1 * dotc(3);
  ag[1] -= SH_C1 * dotc(1);
  ag[2] += SH_C1 * dotc(2);
  float d2x[3], d2y[3], d2z[3];
  for (int ch = 0; ch < 3; ++ch) {
    d2x[ch] = kSH_C2[0] * y * SH(4, ch) + kSH_C2[2] * (-2.0f * x) * SH(6, ch) + kSH_C2[3] * z * SH(7, ch) + kSH_C2[4] * (2.0f * x) * SH(8, ch);
    d2y[ch] = kSH_C2[0] * x * SH(4, ch) + kSH_C2[1] * z * SH(5, ch) + kSH_C2[2] * (-2.0f * y) * SH(6, ch) + kSH_C2[4] * (-2.0f * y) * SH(8, ch);
    d2z[ch] = kSH_C2[1] * y * SH(5, ch) + kSH_C2[2] * (4.0f * z) * SH(6, ch) + kSH_C2[3] * x * SH(7, ch);
  }
  ag[0] += d2x[0] * cf[0] + d2x[1] * cf[1] + d2x[2] * cf[2];
  ag[1] += d2y[0] * cf[0] + d2y[1] * cf[1] + d2y[2] * cf[2];
  ag[2] += d2z[0] * cf[0] + d2z[1] * cf[1] + d2z[2] * cf[2];
  const float f3x[7] = {kSH_C3[0] * 6.0f * xy, kSH_C3[1] * yz, kSH_C3[2] * (-2.0f * xy), kSH_C3[3] * (-6.0f * xz),
                        kSH_C3[4] * (fz2 - 3.0f * x2 - y2), kSH_C3[5] * 2.0f * xz, kSH_C3[6] * 3.0f * x2my2};
  const float f3y[7] = {kSH_C3[0] * 3.0f * (x2 - y2), kSH_C3[1] * xz, kSH_C3[2] * (fz2 - 3.0f * y2 - x2),
                        kSH_C3[3] * (-6.0f * yz), kSH_C3[4] * (-2.0f * xy), kSH_C3[5] * (-2.0f * yz),
                        kSH_C3[6] * (-6.0f * xy)};
  const float f3z[7] = {0.0f, kSH_C3[1] * xy, kSH_C3[2] * 8.0f * yz, kSH_C3[3] * 3.0f * (wz2 - x2 - y2),
                        kSH_C3[4] * 8.0f * xz, kSH_C3[5] * x2my2, 0.0f};
  float d3x[3] = {0.f, 0.f, 0.f}, d3y[3] = {0.f, 0.f, 0.f}, d3z[3] = {0.f, 0.f, 0.f};
  for (int k = 0; k < 7; ++k)
    for (int ch = 0; ch < 3; ++ch) {
      const float s = SH(9 + k, ch);
      d3x[ch] += f3x[k] * s;
      d3y[ch] += f3y[k] * s;
      d3z[ch] += f3z[k] * s;
    }
  ag[0] += d3x[0] * cf[0] + d3x[1] * cf[1] + d3x[2] * cf[2];
  ag[1] += d3y[0] * cf[0] + d3y[1] * cf[1] + d3y[2] * cf[2];
  ag[2] += d3z[0] * cf[0] + d3z[1] * cf[1] + d3z[2] * cf[2];
  const float im3 = im * im * im;
  const float rd[3] = {ox, oy, oz};
  for (int r = 0; r < 3; ++r) {
    float acc = 0.f;
    for (int c = 0; c < 3; ++c) acc += ((c == r ? msq : 0.0f) - rd[c] * rd[r]) * im3 * ag[c];
    sd[r] += acc;
  }
  o.m3[0] = sd[0];
  o.m3[1] = sd[1];
  o.m3[2] = sd[2];

  // ---- scale / rotation (backward.cu:446-518) ----
  const float4 qr = gv.rotation();
  const float qw = qr.x, qx = qr.y, qy = qr.z, qz = qr.w;
  const float xx = qx * qx, yy = qy * qy, zz = qz * qz;
  const float qxy = qx * qy, qxz = qx * qz, qyz = qy * qz;
  const float xw = qx * qw, yw = qy * qw, zw = qz * qw;
  const float sc[3] = {gv.scale(0), gv.scale(1), gv.scale(2)};
  const float sx = gv.scale_modifier * sc[0], sy = gv.scale_modifier * sc[1], sz = gv.scale_modifier * sc[2];
  const float m11 = sx * (1.f - 2.f * (yy + zz)), m12 = sx * 2.f * (qxy - zw), m13 = sx * 2.f * (qxz + yw);
  const float m21 = sy * 2.f * (qxy + zw), m22 = sy * (1.f - 2.f * (xx + zz)), m23 = sy * 2.f * (qyz - xw);
  const float m31 = sz * 2.f * (qxz - yw), m32 = sz * 2.f * (qyz + xw), m33 = sz * (1.f - 2.f * (xx + yy));
  const float g11 = dc[0], g12 = dc[1], g13 = dc[2], g22 = dc[3], g23 = dc[4], g33 = dc[5];
  const float a11 = 2.f * (m11 * g11 + m12 * g12 + m13 * g13);
  const float a12 = 2.f * (m11 * g12 + m12 * g22 + m13 * g23);
  const float a13 = 2.f * (m11 * g13 + m12 * g23 + m13 * g33);
  const float a21 = 2.f * (m21 * g11 + m22 * g12 + m23 * g13);
  const float a22 = 2.f * (m21 * g12 + m22 * g22 + m23 * g23);
  const float a23 = 2.f * (m21 * g13 + m22 * g23 + m23 * g33);
  const float a31 = 2.f * (m31 * g11 + m32 * g12 + m33 * g13);
  const float a32 = 2.f * (m31 * g12 + m32 * g22 + m33 * g23);
  const float a33 = 2.f * (m31 * g13 + m32 * g23 + m33 * g33);
  float ds[3] = {(1.f - 2.f * (yy + zz)) * a11 + 2.f * (qxy - zw) * a12 + 2.f * (qxz + yw) * a13,
                 2.f * (qxy + zw) * a21 + (1.f - 2.f * (xx + zz)) * a22 + 2.f * (qyz - xw) * a23,
                 2.f * (qxz - yw) * a31 + 2.f * (qyz + xw) * a32 + (1.f - 2.f * (xx + yy)) * a33};
  if (gv.svec != nullptr)  // raw path: scales = exp(svec)
    for (int k = 0; k < 3; ++k) ds[k] = ds[k] * sc[k];
  o.sc[0] = ds[0];
  o.sc[1] = ds[1];
  o.sc[2] = ds[2];
  float4 dq;
  dq.x = 4.f * (-sz * (a31 * yw - a32 * xw + a33 * qxy) + sy * (a21 * zw - a22 * qxz + a23 * yy) + sx * (a12 * zw - a13 * yw - a11 * qyz));
  dq.y = 4.f * (sz * (a31 * zw + a32 * zz - a33 * qyz) - sy * (a21 * yw + a22 * qxy + a23 * xx) + sx * (a12 * yy + a13 * zw + a11 * qxz));
  dq.z = 4.f * (-sz * (a31 * xx + a32 * xw + a33 * qxz) + sy * (a21 * zw + a22 * yy + a23 * yw) - sx * (a12 * xw + a13 * xx + a11 * qxy));
  dq.w = 4.f * (sz * (a31 * xw - a32 * xx + a33 * qxy) - sy * (a21 * qxz - a22 * zw + a23 * qyz) + sx * (a12 * qyz - a13 * zz + a11 * yy));
  if (gv.quat != nullptr) {  // raw path: rotation = q / max(|q|, 1e-12)
    const float q0 = __ldg(&gv.quat[4 * gv.gi]), q1 = __ldg(&gv.quat[4 * gv.gi + 1]),
                q2 = __ldg(&gv.quat[4 * gv.gi + 2]), q3 = __ldg(&gv.quat[4 * gv.gi + 3]);
    const float n = sqrtf(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
    if (n > 1e-12f) {  // (g - r (r . g)) / n with r = q / n
      const float inv = __frcp_rn(n);
      const float rg = (q0 * dq.x + q1 * dq.y + q2 * dq.z + q3 * dq.w) * inv;
      dq = make_float4((dq.x - q0 * inv * rg) * inv, (dq.y - q1 * inv * rg) * inv, (dq.z - q2 * inv * rg) * inv,
                       (dq.w - q3 * inv * rg) * inv);
    } else {  // the norm is clamped to 1e-12 there: q / 1e-12 is linear in q
      dq = make_float4(dq.x * 1e12f, dq.y * 1e12f, dq.z * 1e12f, dq.w * 1e12f);
    }
  }
  o.rot[0] = dq.x;
  o.rot[1] = dq.y;
  o.rot[2] = dq.z;
  o.rot[3] = dq.w;
}

// 8 CTAs per SM (64 registers, no spills; shared memory allows 9): more
// Gaussians' loads in flight (0.452 -> 0.415 ms per 4-view step against the
// default 6 CTAs at 80 registers).
__global__ void __launch_bounds__(kGaussThreads, 8) gaussians_ref_kernel(BackwardArgs a) {
  __shared__ float s_sh[kGaussThreads / 32][32 * kShStride];
  // view, projection, camera position: shared memory is never aliased by the
  // outputs, so these stay in place across the output stores
  __shared__ float s_mats[35];
  if (a.items == nullptr) {  // a batched call's matrices live in its item table
    if (threadIdx.x < 16) s_mats[threadIdx.x] = a.view[threadIdx.x];
    else if (threadIdx.x < 32) s_mats[threadIdx.x] = a.proj[threadIdx.x - 16];
    else if (threadIdx.x < 35) s_mats[threadIdx.x] = a.campos[threadIdx.x - 32];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  float* sw = s_sh[threadIdx.x >> 5];
  const int i0 = blockIdx.x * kGaussThreads + (threadIdx.x & ~31);
  if (i0 >= a.P) return;  // warp-uniform
  const int n = min(32, a.P - i0);
  const int i = i0 + lane;
  const int stride = sh_stride(a.M);
  const GView gv = make_gview(a, lane < n ? i : i0, s_mats);
  if (a.items == nullptr) {
    if (a.sh_dc != nullptr) sh_stage_in_raw(a.sh_dc, a.sh_ac, a.M, i0, n, sw, stride);
    else sh_stage_in(a.shs, a.M, i0, n, sw, stride);
  } else {
    batch_sh_stage_in(a, i0, n, sw, stride);
  }
  float basis[16], cf[3] = {0.f, 0.f, 0.f};
  const bool active = lane < n && a.radii[i] > 0;
  if (active) {
    GOut o;
    ref_gaussian(a, i, gv, sw + lane * stride, basis, cf, o);
    store_gout(a, i, o);
  } else if (lane < n) {
    for (int k = 0; k < 3; ++k) a.dL_dmeans3D[3 * i + k] = 0.f;
    for (int k = 0; k < 6; ++k) a.dL_dcov3D[6 * i + k] = 0.f;
    for (int k = 0; k < 3; ++k) a.dL_dscales[3 * i + k] = 0.f;
    for (int k = 0; k < 4; ++k) a.dL_drotations[4 * i + k] = 0.f;
  }
  // raw path: the accumulated opacity gradient through opacity = sigmoid(logit)
  if (a.logit != nullptr && lane < n) {
    const float y = __frcp_rn(1.f + expf(-__ldg(&a.logit[i])));  // sigmoid, within an ulp of the forward's
    a.dL_dopacity[i] = a.dL_dopacity[i] * (1.f - y) * y;
  }
  // densification statistics (gaussians_handler.py:116-118) in this pass, not
  // one of their own; atomic, because views on other streams may add too
  if (a.dens_accum != nullptr && lane < n && a.radii[i] > 0) {
    const float gx = a.dL_dmean2D[3 * i], gy = a.dL_dmean2D[3 * i + 1];
    atomicAdd(&a.dens_accum[i], __fsqrt_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy))));
    atomicAdd(&a.dens_counter[i], 1.0f);
  }
  // dL_dsh[k][ch] = basis[k] * cf[ch] for the first min(M, 16) bands, 0 beyond
  if (a.dL_dsh_dc != nullptr) sh_store_outer_raw(a.dL_dsh_dc, a.dL_dsh_ac, a.M, i0, n, sw, basis, cf, active);
  else sh_store_outer(a.dL_dsh, a.M, i0, n, sw, basis, cf, active);
}

// Per-Gaussian, exact derivative of the forward.
// One Gaussian (radius > 0) of the exact-derivative pass: every output but
// dL_dsh, plus the outer-product factors of dL_dsh (see ref_gaussian).
__device__ __forceinline__ void exact_gaussian(const BackwardArgs& a, int i, const GView& gv, const float* sh_row,
                                               float (&basis)[16], float (&cf)[3], GOut& o) {
  const int M = a.M;
  const float* mats = gv.mats;
  const float* cam = mats + 32;
  const float* V = mats;
  const float* PM = mats + 16;
  const float m0 = __ldg(&gv.means3D[3 * gv.gi]), m1 = __ldg(&gv.means3D[3 * gv.gi + 1]), m2 = __ldg(&gv.means3D[3 * gv.gi + 2]);
  float gm[3] = {0.f, 0.f, 0.f};
  // screen position / depth: ndc = clip.xyz / (clip.w + 1e-5); dL_dmean2D already holds dL/dNDC
  float clip[4];
  for (int r = 0; r < 4; ++r) clip[r] = PM[r] * m0 + PM[4 + r] * m1 + PM[8 + r] * m2 + PM[12 + r];
  const float wi = 1.0f / (clip[3] + 1e-5f);
  const float gn0 = __ldg(&a.dL_dmean2D[3 * i]), gn1 = __ldg(&a.dL_dmean2D[3 * i + 1]), gn2 = __ldg(&a.acc_depth[i]);
  const float gcl[4] = {gn0 * wi, gn1 * wi, gn2 * wi, -(gn0 * clip[0] + gn1 * clip[1] + gn2 * clip[2]) * wi * wi};
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 4; ++r) gm[c] += PM[4 * c + r] * gcl[r];
  // covariance chain
  float t[3];
  for (int r = 0; r < 3; ++r) t[r] = V[r] * m0 + V[4 + r] * m1 + V[8 + r] * m2 + V[12 + r];
  const float L = float(gv.W) / (2.0f * gv.focal_x);
  const float rx = t[0] / t[2], ry = t[1] / t[2];
  const float nn = sqrtf(rx * rx + ry * ry) / L;
  const bool clampd = nn > 1.0f;
  float txp = t[0], typ = t[1];
  if (clampd) { txp = rx / nn * t[2]; typ = ry / nn * t[2]; }
  const float tz = t[2], f = gv.focal_x;
  const float rgt[3] = {V[0], V[4], V[8]}, upv[3] = {V[1], V[5], V[9]}, fw[3] = {V[2], V[6], V[10]};
  float jx[3], jy[3];
  for (int k = 0; k < 3; ++k) {
    jx[k] = f * (rgt[k] / tz - txp * fw[k] / (tz * tz));
    jy[k] = f * (upv[k] / tz - typ * fw[k] / (tz * tz));
  }
  const float* pc = a.cov3D + 6 * size_t(i);  // read with __ldg below
  const float S[3][3] = {{__ldg(pc + 0), __ldg(pc + 1), __ldg(pc + 2)}, {__ldg(pc + 1), __ldg(pc + 3), __ldg(pc + 4)}, {__ldg(pc + 2), __ldg(pc + 4), __ldg(pc + 5)}};
  const float gxx = __ldg(&a.acc_cov[4 * i]), gxy = __ldg(&a.acc_cov[4 * i + 1]), gyy = __ldg(&a.acc_cov[4 * i + 2]);
  float Gf[3][3];
  for (int p = 0; p < 3; ++p)
    for (int q = 0; q < 3; ++q) Gf[p][q] = gxx * jx[p] * jx[q] + gyy * jy[p] * jy[q] + gxy * jx[p] * jy[q];
  o.cov[0] = Gf[0][0];
  o.cov[1] = Gf[0][1] + Gf[1][0];
  o.cov[2] = Gf[0][2] + Gf[2][0];
  o.cov[3] = Gf[1][1];
  o.cov[4] = Gf[1][2] + Gf[2][1];
  o.cov[5] = Gf[2][2];
  float Sjx[3], Sjy[3];
  for (int p = 0; p < 3; ++p) {
    Sjx[p] = S[p][0] * jx[0] + S[p][1] * jx[1] + S[p][2] * jx[2];
    Sjy[p] = S[p][0] * jy[0] + S[p][1] * jy[1] + S[p][2] * jy[2];
  }
  float gtxp = 0.f, gtyp = 0.f, gtz = 0.f;
  for (int k = 0; k < 3; ++k) {
    const float gjx = 2.f * gxx * Sjx[k] + gxy * Sjy[k];
    const float gjy = 2.f * gyy * Sjy[k] + gxy * Sjx[k];
    gtxp += gjx * (-f * fw[k] / (tz * tz));
    gtyp += gjy * (-f * fw[k] / (tz * tz));
    gtz += gjx * f * (-rgt[k] / (tz * tz) + 2.f * txp * fw[k] / (tz * tz * tz));
    gtz += gjy * f * (-upv[k] / (tz * tz) + 2.f * typ * fw[k] / (tz * tz * tz));
  }
  float gt[3];
  if (!clampd) {
    gt[0] = gtxp; gt[1] = gtyp; gt[2] = gtz;
  } else {
    const float r2 = t[0] * t[0] + t[1] * t[1], r1 = sqrtf(r2), r3 = r2 * r1;
    const float dxx = L * tz * t[1] * t[1] / r3, dxy = -L * tz * t[0] * t[1] / r3, dxz = L * t[0] / r1;
    const float dyx = -L * tz * t[0] * t[1] / r3, dyy = L * tz * t[0] * t[0] / r3, dyz = L * t[1] / r1;
    gt[0] = gtxp * dxx + gtyp * dyx;
    gt[1] = gtxp * dxy + gtyp * dyy;
    gt[2] = gtz + gtxp * dxz + gtyp * dyz;
  }
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) gm[c] += V[4 * c + r] * gt[r];
  // Sigma = M M^T, M = R diag(s)
  const float4 qr = gv.rotation();
  const float w = qr.x, x = qr.y, y = qr.z, z = qr.w;
  const float R[3][3] = {{1.f - 2.f * (y * y + z * z), 2.f * (x * y - w * z), 2.f * (x * z + w * y)},
                         {2.f * (x * y + w * z), 1.f - 2.f * (x * x + z * z), 2.f * (y * z - w * x)},
                         {2.f * (x * z - w * y), 2.f * (y * z + w * x), 1.f - 2.f * (x * x + y * y)}};
  const float s[3] = {gv.scale(0), gv.scale(1), gv.scale(2)};
  float dM[3][3];
  for (int p = 0; p < 3; ++p)
    for (int k = 0; k < 3; ++k) {
      float acc = 0.f;
      for (int q = 0; q < 3; ++q) acc += 0.5f * (Gf[p][q] + Gf[q][p]) * R[q][k] * s[k];
      dM[p][k] = 2.f * acc;
    }
  for (int k = 0; k < 3; ++k) {
    float acc = 0.f;
    for (int p = 0; p < 3; ++p) acc += dM[p][k] * R[p][k];
    o.sc[k] = acc;
  }
  float dR[3][3];
  for (int p = 0; p < 3; ++p)
    for (int k = 0; k < 3; ++k) dR[p][k] = dM[p][k] * s[k];
  o.rot[0] = dR[0][1] * (-2.f * z) + dR[0][2] * (2.f * y) + dR[1][0] * (2.f * z) + dR[1][2] * (-2.f * x) +
                           dR[2][0] * (-2.f * y) + dR[2][1] * (2.f * x);
  o.rot[1] = dR[0][1] * (2.f * y) + dR[0][2] * (2.f * z) + dR[1][0] * (2.f * y) + dR[1][1] * (-4.f * x) +
                               dR[1][2] * (-2.f * w) + dR[2][0] * (2.f * z) + dR[2][1] * (2.f * w) + dR[2][2] * (-4.f * x);
  o.rot[2] = dR[0][0] * (-4.f * y) + dR[0][1] * (2.f * x) + dR[0][2] * (2.f * w) + dR[1][0] * (2.f * x) +
                               dR[1][2] * (2.f * z) + dR[2][0] * (-2.f * w) + dR[2][1] * (2.f * z) + dR[2][2] * (-4.f * y);
  o.rot[3] = dR[0][0] * (-4.f * z) + dR[0][1] * (-2.f * w) + dR[0][2] * (2.f * x) + dR[1][0] * (2.f * w) +
                               dR[1][1] * (-4.f * z) + dR[1][2] * (2.f * y) + dR[2][0] * (2.f * x) + dR[2][1] * (2.f * y);
  // colour: rgb = sum_k basis_k(dir) sh_k + 0.5 with the forward's constants
  const float v0 = m0 - cam[0], v1 = m1 - cam[1], v2 = m2 - cam[2];
  const float vn = sqrtf(v0 * v0 + v1 * v1 + v2 * v2);
  const float X = v0 / vn, Y = v1 / vn, Z = v2 / vn;
  const float gc0 = __ldg(&a.dL_dcolors[3 * i]), gc1 = __ldg(&a.dL_dcolors[3 * i + 1]), gc2 = __ldg(&a.dL_dcolors[3 * i + 2]);
  const float C1 = 0.4886025119029199f, C2a = 1.0925484305920792f, C2e = 0.5462742152960396f;
  const float C30 = 0.5900435899266435f, C31 = 2.890611442640554f, C32 = 0.4570457994644658f;
  const float C33 = 0.3731763325901154f, C35 = 1.445305721320277f;
  const float xx = X * X, yy = Y * Y, zz = Z * Z;
  float b[16], db[16][3];
  for (int k = 0; k < 16; ++k) db[k][0] = db[k][1] = db[k][2] = 0.f;
  b[0] = 0.28209479177387814f;
  b[1] = -C1 * Y; db[1][1] = -C1;
  b[2] = C1 * Z; db[2][2] = C1;
  b[3] = -C1 * X; db[3][0] = -C1;
  b[4] = C2a * X * Y; db[4][0] = C2a * Y; db[4][1] = C2a * X;
  b[5] = -C2a * Y * Z; db[5][1] = -C2a * Z; db[5][2] = -C2a * Y;
  b[6] = 0.3f * (2.f * zz - xx - yy); db[6][0] = -0.6f * X; db[6][1] = -0.6f * Y; db[6][2] = 1.2f * Z;
  b[7] = -C2a * X * Z; db[7][0] = -C2a * Z; db[7][2] = -C2a * X;
  b[8] = C2e * (xx - yy); db[8][0] = 2.f * C2e * X; db[8][1] = -2.f * C2e * Y;
  b[9] = -C30 * Y * (3.f * xx - yy); db[9][0] = -6.f * C30 * X * Y; db[9][1] = -C30 * (3.f * xx - 3.f * yy);
  b[10] = C31 * X * Y * Z; db[10][0] = C31 * Y * Z; db[10][1] = C31 * X * Z; db[10][2] = C31 * X * Y;
  b[11] = -C32 * Y * (4.f * zz - xx - yy); db[11][0] = 2.f * C32 * X * Y; db[11][1] = -C32 * (4.f * zz - xx - 3.f * yy); db[11][2] = -8.f * C32 * Y * Z;
  b[12] = C33 * Z * (2.f * zz - 3.f * xx - 3.f * yy); db[12][0] = -6.f * C33 * X * Z; db[12][1] = -6.f * C33 * Y * Z; db[12][2] = C33 * (6.f * zz - 3.f * xx - 3.f * yy);
  b[13] = -C32 * X * (4.f * zz - xx - yy); db[13][0] = -C32 * (4.f * zz - 3.f * xx - yy); db[13][1] = 2.f * C32 * X * Y; db[13][2] = -8.f * C32 * X * Z;
  b[14] = C35 * Z * (xx - yy); db[14][0] = 2.f * C35 * X * Z; db[14][1] = -2.f * C35 * Y * Z; db[14][2] = C35 * (xx - yy);
  b[15] = -C30 * X * (xx - 3.f * yy); db[15][0] = -C30 * (3.f * xx - 3.f * yy); db[15][1] = 6.f * C30 * X * Y;
  int de = gv.degree > 3 ? 3 : gv.degree;
  while (de > 0 && (de + 1) * (de + 1) > M) --de;
  const int nb = (de + 1) * (de + 1);
  const float* shd = sh_row;
  float gdir[3] = {0.f, 0.f, 0.f};
  for (int k = 0; k < nb; ++k) {
    const float sdot = shd[3 * k] * gc0 + shd[3 * k + 1] * gc1 + shd[3 * k + 2] * gc2;
    gdir[0] += sdot * db[k][0];
    gdir[1] += sdot * db[k][1];
    gdir[2] += sdot * db[k][2];
  }
  // dL_dsh = b[k] * gc for the bands the forward used, 0 beyond
  for (int k = 0; k < 16; ++k) basis[k] = k < nb ? b[k] : 0.f;
  cf[0] = gc0;
  cf[1] = gc1;
  cf[2] = gc2;
  const float dd[3] = {X, Y, Z};
  const float dot = dd[0] * gdir[0] + dd[1] * gdir[1] + dd[2] * gdir[2];
  for (int p = 0; p < 3; ++p) gm[p] += (gdir[p] - dd[p] * dot) / vn;
  o.m3[0] = gm[0];
  o.m3[1] = gm[1];
  o.m3[2] = gm[2];
}

__global__ void __launch_bounds__(kGaussThreads) gaussians_exact_kernel(BackwardArgs a) {
  __shared__ float s_sh[kGaussThreads / 32][32 * kShStride];
  // view, projection, camera position: shared memory is never aliased by the
  // outputs, so these stay in place across the output stores
  __shared__ float s_mats[35];
  if (a.items == nullptr) {  // a batched call's matrices live in its item table
    if (threadIdx.x < 16) s_mats[threadIdx.x] = a.view[threadIdx.x];
    else if (threadIdx.x < 32) s_mats[threadIdx.x] = a.proj[threadIdx.x - 16];
    else if (threadIdx.x < 35) s_mats[threadIdx.x] = a.campos[threadIdx.x - 32];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  float* sw = s_sh[threadIdx.x >> 5];
  const int i0 = blockIdx.x * kGaussThreads + (threadIdx.x & ~31);
  if (i0 >= a.P) return;  // warp-uniform
  const int n = min(32, a.P - i0);
  const int i = i0 + lane;
  const int stride = sh_stride(a.M);
  const GView gv = make_gview(a, lane < n ? i : i0, s_mats);
  if (a.items == nullptr) {
    sh_stage_in(a.shs, a.M, i0, n, sw, stride);
  } else {
    batch_sh_stage_in(a, i0, n, sw, stride);
  }
  float basis[16], cf[3] = {0.f, 0.f, 0.f};
  const bool active = lane < n && a.radii[i] > 0;
  if (active) {
    GOut o;
    exact_gaussian(a, i, gv, sw + lane * stride, basis, cf, o);
    store_gout(a, i, o);
  } else if (lane < n) {
    for (int k = 0; k < 3; ++k) a.dL_dmeans3D[3 * i + k] = 0.f;
    for (int k = 0; k < 6; ++k) a.dL_dcov3D[6 * i + k] = 0.f;
    for (int k = 0; k < 3; ++k) a.dL_dscales[3 * i + k] = 0.f;
    for (int k = 0; k < 4; ++k) a.dL_drotations[4 * i + k] = 0.f;
  }
  sh_store_outer(a.dL_dsh, a.M, i0, n, sw, basis, cf, active);
}

// ---------------------------------------------------------------------------
// Grouped per-Gaussian pass (batched calls): one thread per output row of a
// group (a scene, or a serving request), walking the group's items (views) in
// table order.  Each item's element is the single-view computation above; its
// outputs are summed in registers in item order, starting from zero, with
// explicit-rounding adds -- w2w_group_sum's order over the per-element
// outputs (the per-view arithmetic, inlined here, may fuse a multiply-add
// differently, so the two agree to a few ulps).  The SH rows are staged once per warp for
// all views of a scene (a view of another scene reads its own row from
// memory), and no per-element dL/dSH, dL/dmeans3D, dL/dscales, dL/drotations
// or dL/dcov3D is written.
// ---------------------------------------------------------------------------
template <int kMode>
__global__ void __launch_bounds__(kGaussThreads) gaussians_group_kernel(BackwardArgs a) {
  __shared__ float s_sh[kGaussThreads / 32][32 * kShStride];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  float* sw = s_sh[threadIdx.x >> 5];
  const long long row0 = (long long)blockIdx.x * kGaussThreads + (threadIdx.x & ~31);
  if (row0 >= a.group_rows) return;  // warp-uniform
  const int n = int(min(32LL, a.group_rows - row0));
  const uint32_t row = uint32_t(row0) + uint32_t(lane < n ? lane : 0);
  const uint32_t* gbase = a.group_tables;
  const uint32_t* iptr = gbase + (a.num_groups + 1);
  const uint32_t* ielem = iptr + (a.num_groups + 1);
  int lo = 0, hi = a.num_groups - 1;  // this row's group: the last g with gbase[g] <= row
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(gbase + mid) <= row) lo = mid;
    else hi = mid - 1;
  }
  const int g = lo;
  const uint32_t r = row - __ldg(gbase + g);
  const uint32_t k0 = __ldg(iptr + g), k1 = __ldg(iptr + g + 1);
  const int M = a.M, rg = 3 * M, stride = sh_stride(M);
  const uint32_t e0 = k0 < k1 ? __ldg(ielem + k0) + r : uint32_t(a.P);
  const float* shs0 = e0 < uint32_t(a.P) ? a.items[find_item_elem(a.items, a.num_items, e0)].shs : nullptr;
  // the rows of the warp's first group's scene, contiguous when every lane is in that group
  if (__all_sync(full, g == __shfl_sync(full, g, 0) && shs0 != nullptr)) {
    sh_stage_in(shs0, M, int(__shfl_sync(full, r, 0)), n, sw, stride);
  } else {
    if (lane < n && shs0 != nullptr)
      for (int c = 0; c < 3 * (M < 16 ? M : 16); ++c) sw[lane * stride + c] = __ldg(shs0 + size_t(r) * rg + c);
    __syncwarp();
  }
  float am[3] = {0.f, 0.f, 0.f}, asc[3] = {0.f, 0.f, 0.f}, arot[4] = {0.f, 0.f, 0.f, 0.f}, aop = 0.f;
  float ash[48];
#pragma unroll
  for (int c = 0; c < 48; ++c) ash[c] = 0.f;
  for (uint32_t k = k0; lane < n && k < k1; ++k) {
    const uint32_t i = __ldg(ielem + k) + r;
    if (i >= uint32_t(a.P)) continue;  // a table pointing past the elements: nothing is read there
    const BatchItem& it = a.items[find_item_elem(a.items, a.num_items, i)];
    const GView gv = item_gview(it, int(i));
    if (a.radii[i] > 0) {
      const float* sh_row = it.shs == shs0 ? sw + lane * stride : it.shs + size_t(gv.gi) * rg;
      float basis[16], cf[3];
      GOut o;
      if (kMode == 1) exact_gaussian(a, int(i), gv, sh_row, basis, cf, o);
      else ref_gaussian(a, int(i), gv, sh_row, basis, cf, o);
#pragma unroll
      for (int c = 0; c < 3; ++c) am[c] = add(am[c], o.m3[c]);
#pragma unroll
      for (int c = 0; c < 3; ++c) asc[c] = add(asc[c], o.sc[c]);
#pragma unroll
      for (int c = 0; c < 4; ++c) arot[c] = add(arot[c], o.rot[c]);
#pragma unroll
      for (int b = 0; b < 16; ++b)
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) ash[3 * b + ch] = add(ash[3 * b + ch], mul(basis[b], cf[ch]));
    }
    aop = add(aop, a.dL_dopacity[i]);
  }
  if (lane < n) {
    for (int c = 0; c < 3; ++c) a.g_means3D[3 * size_t(row) + c] = am[c];
    for (int c = 0; c < 3; ++c) a.g_scales[3 * size_t(row) + c] = asc[c];
    for (int c = 0; c < 4; ++c) a.g_rotations[4 * size_t(row) + c] = arot[c];
    a.g_opacity[row] = aop;
  }
  // dL/dSH rows [row0, row0 + n) ([rows, M, 3], contiguous) through shared
  // memory, so the warp's stores are one contiguous run
  __syncwarp();  // every lane is done with the staged input rows
  if (lane < n) {
#pragma unroll
    for (int c = 0; c < 48; ++c)
      if (c < rg) sw[lane * stride + c] = ash[c];
    for (int c = 48; c < rg; ++c) sw[lane * stride + c] = 0.f;  // bands beyond the 16th (none for M <= 16)
  }
  __syncwarp();
  float* dst = a.g_sh + size_t(row0) * rg;
  const int total = n * rg;
  int gr = 0, c = lane;
  while (c >= rg) { c -= rg; ++gr; }
  for (int e = lane; e < total; e += 32) {
    dst[e] = sw[gr * stride + c];
    c += 32;
    while (c >= rg) { c -= rg; ++gr; }
  }
}

}  // namespace

void launch_backward_groups(const BackwardArgs& a, cudaStream_t stream) {
  if (a.group_rows <= 0 || a.num_groups <= 0) return;
  const long long blocks = (a.group_rows + kGaussThreads - 1) / kGaussThreads;
  stage_begin(kStBwdGaussians, stream);
  if (a.grad_mode == 1) gaussians_group_kernel<1><<<unsigned(blocks), kGaussThreads, 0, stream>>>(a);
  else gaussians_group_kernel<0><<<unsigned(blocks), kGaussThreads, 0, stream>>>(a);
  stage_end(kStBwdGaussians, stream, 1);
}

void launch_backward_render(const BackwardArgs& a, cudaStream_t stream) {
  const int tiles = a.items ? a.total_tiles : ((a.W + kTile - 1) / kTile) * ((a.H + kTile - 1) / kTile);
  if (tiles <= 0) return;
  BackwardArgs b = a;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // the heaviest tiles by largest contributor count: knob quarters of the SM count
  b.split = min(tiles / 4, sms * tune_value(kTuneBwdSplit) / 4);
  const int ways = tune_value(kTuneBwdWays);
  stage_begin(kStBwdRender, stream);
  const int grid = tiles + (ways - 1) * b.split;
  const bool da = a.dL_ddepth != nullptr || a.dL_dalpha != nullptr;  // a loss reaches depth or alpha
  if (ways == 3) {
    if (a.grad_mode == 1) render_exact_kernel<3><<<grid, kBlendThreads, 0, stream>>>(b);
    else if (da) render_ref_kernel<3, true><<<grid, kBlendThreads, 0, stream>>>(b);
    else render_ref_kernel<3, false><<<grid, kBlendThreads, 0, stream>>>(b);
  } else {
    if (a.grad_mode == 1) render_exact_kernel<2><<<grid, kBlendThreads, 0, stream>>>(b);
    else if (da) render_ref_kernel<2, true><<<grid, kBlendThreads, 0, stream>>>(b);
    else render_ref_kernel<2, false><<<grid, kBlendThreads, 0, stream>>>(b);
  }
  stage_end(kStBwdRender, stream, 1);
}

void launch_backward_gaussians(const BackwardArgs& a, cudaStream_t stream) {
  if (a.P <= 0) return;
  const int blocks = (a.P + kGaussThreads - 1) / kGaussThreads;
  stage_begin(kStBwdGaussians, stream);
  if (a.grad_mode == 1) gaussians_exact_kernel<<<blocks, kGaussThreads, 0, stream>>>(a);
  else gaussians_ref_kernel<<<blocks, kGaussThreads, 0, stream>>>(a);
  stage_end(kStBwdGaussians, stream, 1);
}

}  // namespace w2w
