// Shared device-side definitions for the sm_100a Gaussian rasterizer.
//
// Floating point: every operation whose rounding affects a bit-exact output
// (projection, ADR culling, key depth bits, blend decisions) is written with
// explicit-rounding intrinsics (__fmul_rn, __fadd_rn, __fmaf_rn, __fdiv_rn,
// __fsqrt_rn, __frcp_rn), which the compiler never contracts.  Where the
// reference's compiler fused a multiply into an add, the same fusion is
// written out here; the per-expression choices were established by comparing
// against the reference extension's own buffers on a B200 and are listed in
// pinned_fp.h (the CPU oracle carries the identical table).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pinned_fp.h"

namespace w2w {

constexpr int kTile = 16;             // tile edge in pixels (reference: 16x16)
constexpr int kBlendThreads = 256;    // one thread per tile pixel
constexpr int kBatch = 256;           // Gaussians staged per shared-memory batch

// Status codes written to the device error word (bitwise OR).
enum : uint32_t {
  kErrNone = 0,
  kErrCapacity = 1u << 0,   // more instances than the binning state holds
  kErrTimeout = 1u << 1,    // a bounded spin wait gave up
  kErrRange = 1u << 2,      // an index fell outside its buffer and was skipped
};

// ---------------------------------------------------------------------------
// explicit-rounding arithmetic
// ---------------------------------------------------------------------------
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }

// Correctly rounded a / b without branches, for operands in div_in_range.
// Markstein's scheme (P. Markstein, IBM J. Res. Dev. 34(1), 1990; Muller et
// al., Handbook of Floating-Point Arithmetic, ch. 5): from the hardware
// reciprocal approximation y0 (rcp.approx, within 1 ulp), one Newton step
// y = y0 + y0 (1 - b y0) gives RN(1/b) (checked against __frcp_rn for every
// significand); q0 = RN(a y); two remainder corrections q <- q + (a - b q) y,
// each remainder exact under fma, make q faithful and then, by Markstein's
// theorem (y = RN(1/b), q faithful), equal to RN(a / b).
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// RN(1/b) for |b| in [2^-20, 2^60].
__device__ __forceinline__ float rcp_markstein(float b) {
  const float y0 = rcp_approx(b);
  return fma(fma(-b, y0, 1.0f), y0, y0);
}
// div_markstein with y = rcp_markstein(b) given (several quotients by one b)
__device__ __forceinline__ float div_markstein_y(float a, float b, float y) {
  const float q0 = mul(a, y);
  const float q1 = fma(fma(-b, q0, a), y, q0);
  return fma(fma(-b, q1, a), y, q1);
}
__device__ __forceinline__ float div_markstein(float a, float b) { return div_markstein_y(a, b, rcp_markstein(b)); }
// Operands for which div_markstein equals div: |b| in [2^-20, 2^60] and
// a = 0 or |a| in [2^-60, 2^100], so the quotient lies in [2^-120, 2^120] and
// no intermediate (reciprocal, product, remainders) leaves the normal range.
__device__ __forceinline__ bool div_in_range(float a, float b) {
  const float fa = fabsf(a), fb = fabsf(b);
  return fb >= 0x1p-20f && fb <= 0x1p60f && fa <= 0x1p100f && (fa >= 0x1p-60f || fa == 0.0f);
}

// a*b + c*d: 0 = both rounded, 1 = fuse a*b, 2 = fuse c*d
template <int V>
__device__ __forceinline__ float s2(float a, float b, float c, float d) {
  if constexpr (V == 1) return fma(a, b, mul(c, d));
  else if constexpr (V == 2) return fma(c, d, mul(a, b));
  else return add(mul(a, b), mul(c, d));
}
// a*b - c*d
template <int V>
__device__ __forceinline__ float d2(float a, float b, float c, float d) {
  if constexpr (V == 1) return fma(a, b, -mul(c, d));
  else if constexpr (V == 2) return fma(-c, d, mul(a, b));
  else return sub(mul(a, b), mul(c, d));
}
// (a*b + c*d) + e*f
template <int V>
__device__ __forceinline__ float s3(float a, float b, float c, float d, float e, float f) {
  if constexpr (V == 1) return fma(e, f, fma(a, b, mul(c, d)));
  else if constexpr (V == 2) return fma(e, f, fma(c, d, mul(a, b)));
  else if constexpr (V == 3) return fma(e, f, add(mul(a, b), mul(c, d)));
  else if constexpr (V == 4) return add(fma(a, b, mul(c, d)), mul(e, f));
  else if constexpr (V == 5) return add(fma(c, d, mul(a, b)), mul(e, f));
  else if constexpr (V == 6) return fma(a, b, fma(c, d, mul(e, f)));
  else return add(add(mul(a, b), mul(c, d)), mul(e, f));
}
// a*b + c
template <int V>
__device__ __forceinline__ float s1(float a, float b, float c) {
  if constexpr (V != 0) return fma(a, b, c);
  else return add(mul(a, b), c);
}

// Row r of (column-major 4x4 m) * (x, y, z, 1): (m0 x + m1 y) + (m2 z + m3).
template <int VA, int VB>
__device__ __forceinline__ float m4row(const float* m, int r, float x, float y, float z) {
  return add(s2<VA>(m[r], x, m[4 + r], y), s1<VB>(m[8 + r], z, m[12 + r]));
}

// ---------------------------------------------------------------------------
// Block culling.  The per-pixel loops run one warp per 8x4 pixel block of a
// 16x16 tile (block b: columns 8*(b & 1) .. +7, rows 4*(b >> 1) .. +3).  For
// every staged list entry the loader computes which of the tile's 8 blocks
// the Gaussian can reach with alpha >= 1/255, and each warp walks only the
// entries whose bit for its block is set.  A skipped entry is one every pixel
// of the block skips anyway, so no decision changes.
//
// The test is exact for the ellipse E = {d : d^T Q d <= t'} against the
// block's continuous pixel-centre rectangle grown by kCullPad: per band of 4
// rows, E's x-extent over the band is [L, R] with
//   R = max over v in band of (-beta v + sqrt(gamma - eps v^2)),
//   L = min over v in band of (-beta v - sqrt(gamma - eps v^2)),
// (beta = B/A, gamma = t'/A, eps = det/A^2 for Q = [[A, B], [B, C]]); R is
// concave in v with its maximum at vr = -B hx / C, L convex with its minimum at
// -vr, so each is one evaluation at the clamped extremum.
//
// Conservativeness.  A pixel reaches alpha >= 1/255 only if q = d^T Q d <=
// t = 2 ln(255 o) + 2e-4 (the blend's own threshold is 1e-4 tighter; exp and
// log rounding is far inside 1e-4).  The per-pixel evaluations round q (or the
// mahalanobis distance / det) with a relative error of a few ulps of
// mag = A dx^2 + 2|B dx dy| + C dy^2 <= k q, k = (sqrt(AC) + |B|)^2 / det.
// The culling threshold t' = t (1 + 4e-4 k) + 1e-4 exceeds that by more than
// 100x for k < 1024; beyond that (or with a non-positive-definite Q) nothing
// is culled.  kCullPad = 1/16 pixel covers the rounding of the pixel offsets
// and of L, R (below 1e-2 pixel for extents under 8192 pixels; larger
// ellipses are not culled).
// ---------------------------------------------------------------------------
constexpr int kBlockW = 8, kBlockH = 4;  // pixel block per warp
constexpr float kCullPad = 0.0625f;

struct CullParams {
  float hy;    // y half-extent of E; +inf: cull nothing, -1: cull everything
  float beta, gamma, eps, vr;
};

// Ellipse parameters from the conic (A, B, C) and opacity.
__device__ __forceinline__ CullParams make_cull_params(float A, float B, float C, float opacity) {
  CullParams p{__int_as_float(0x7f800000), 0.f, 0.f, 0.f, 0.f};
  if (!(opacity > 0.0f)) { p.hy = -1.0f; return p; }
  const float t = 2.0f * logf(255.0f * opacity) + 2e-4f;
  if (t < 0.0f) { p.hy = -1.0f; return p; }  // opacity < 1/255: alpha never reaches 1/255
  if (!(A > 0.0f && C > 0.0f) || !(t < 1e30f)) return p;
  const float det = A * C - B * B;
  if (!(det > 0.0f)) return p;
  const float sac = sqrtf(A * C) + fabsf(B);
  const float k = sac * sac / det;
  if (!(k < 1024.0f)) return p;
  const float tt = t * (1.0f + 4e-4f * k) + 1e-4f;
  const float hx = sqrtf(tt * C / det), hy = sqrtf(tt * A / det);
  if (!(hx < 8192.0f && hy < 8192.0f)) return p;
  p.hy = hy;
  p.beta = B / A;
  p.gamma = tt / A;
  p.eps = det / (A * A);
  p.vr = -B * hx / C;
  return p;
}

__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Renderer.render's activations (Renderer.py:164-167), bit-identical to the
// torch operations the reference runs on a B200 (checked over 2^24 inputs):
// sigmoid = 1 / (1 + exp(-x)) with IEEE division; exp; the quaternion divided
// by max(sqrt((w*w + y*y) + (x*x + z*z)), 1e-12) with every product rounded.
__device__ __forceinline__ float act_sigmoid(float x) { return __fdiv_rn(1.f, __fadd_rn(1.f, expf(-x))); }
__device__ __forceinline__ float4 act_normalize(float w, float x, float y, float z) {
  const float ss = __fadd_rn(__fadd_rn(__fmul_rn(w, w), __fmul_rn(y, y)), __fadd_rn(__fmul_rn(x, x), __fmul_rn(z, z)));
  const float n = fmaxf(__fsqrt_rn(ss), 1e-12f);
  return make_float4(__fdiv_rn(w, n), __fdiv_rn(x, n), __fdiv_rn(y, n), __fdiv_rn(z, n));
}

// Bit b set: the Gaussian may reach alpha >= 1/255 in 8x4 block b of the tile
// whose top-left pixel is (X0, Y0) (kGroups rows of two blocks: the whole
// 16x16 tile for kGroups = 4).  hy/beta/gamma/eps/vr as in CullParams.
template <int kGroups = 4>
__device__ __forceinline__ uint32_t block_mask(float mx, float my, float hy, float beta, float gamma, float eps,
                                               float vr, int X0, int Y0) {
  if (!(hy >= 0.0f && hy < 1e30f)) return hy < 0.0f ? 0u : (1u << (2 * kGroups)) - 1u;
  const float ux = float(X0) - mx, vy = float(Y0) - my;
  const float ulo0 = ux - kCullPad, uhi0 = ux + (7.0f + kCullPad);
  const float ulo1 = ux + (8.0f - kCullPad), uhi1 = ux + (15.0f + kCullPad);
  uint32_t m = 0;
#pragma unroll
  for (int by = 0; by < kGroups; ++by) {
    const float v0 = vy + (float(4 * by) - kCullPad), v1 = vy + (float(4 * by + 3) + kCullPad);
    const float a = fmaxf(v0, -hy), b = fminf(v1, hy);
    const float vR = fminf(fmaxf(vr, a), b), vL = fminf(fmaxf(-vr, a), b);
    const float R = sqrt_approx(fmaxf(0.0f, gamma - eps * vR * vR)) - beta * vR;
    const float L = -sqrt_approx(fmaxf(0.0f, gamma - eps * vL * vL)) - beta * vL;
    const bool band = a <= b;
    const uint32_t c0 = (band && L <= uhi0 && R >= ulo0) ? 1u : 0u;
    const uint32_t c1 = (band && L <= uhi1 && R >= ulo1) ? 2u : 0u;
    m |= (c0 | c1) << (2 * by);
  }
  return m;
}

// Whether the Gaussian may reach alpha >= 1/255 in the 8x4 block whose
// top-left pixel is (bx, by): block_mask's test for one block.
__device__ __forceinline__ bool block_test(float mx, float my, float hy, float beta, float gamma, float eps, float vr,
                                           int bx, int by) {
  if (!(hy >= 0.0f && hy < 1e30f)) return !(hy < 0.0f);
  const float ux = float(bx) - mx, vy = float(by) - my;
  const float v0 = vy - kCullPad, v1 = vy + (3.0f + kCullPad);
  const float a = fmaxf(v0, -hy), b = fminf(v1, hy);
  const float vR = fminf(fmaxf(vr, a), b), vL = fminf(fmaxf(-vr, a), b);
  const float R = sqrt_approx(fmaxf(0.0f, gamma - eps * vR * vR)) - beta * vR;
  const float L = -sqrt_approx(fmaxf(0.0f, gamma - eps * vL * vL)) - beta * vL;
  return a <= b && L <= ux + (7.0f + kCullPad) && R >= ux - kCullPad;
}

// ---------------------------------------------------------------------------
// Per-Gaussian blend record (forward blend and exact backward), 64 bytes.
// The first 48 bytes are what the per-pixel loops read from shared memory;
// the last 20 are the block-culling parameters.
// ---------------------------------------------------------------------------
struct __align__(16) BlendRecord {
  float mx, my;          // screen position (pixels)
  float cxx, cxy, cyy;   // 2-D covariance
  float det;             // the blend's own determinant of the covariance
  float opacity;
  float depth;           // NDC z
  float r, g, b;         // colour (unclamped)
  float hy, beta, gamma, eps, vr;  // CullParams
};
static_assert(sizeof(BlendRecord) == 64, "BlendRecord layout");

// Per-Gaussian record read by the reference-formula backward pass, 64 bytes.
// skip: -ln(255 o) - 1e-4; a pair whose exponent is below it has
// alpha < 1/255 for certain, so its exp is not evaluated.
struct __align__(16) BackwardRecord {
  float mx, my;
  float conic_a, conic_b, conic_c;  // inverse 2-D covariance
  float opacity;
  float depth;
  float r, g, b;
  float skip;
  float hy, beta, gamma, eps, vr;  // CullParams
};
static_assert(sizeof(BackwardRecord) == 64, "BackwardRecord layout");

// ---------------------------------------------------------------------------
// State layouts.  All arrays start on 256-byte boundaries.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Device-written header at the start of the geometry state.
struct GeomHeader {
  uint32_t error;          // kErr* bits
  uint32_t depth_min;      // min/max of depth bits over Gaussians that emit keys
  uint32_t depth_max;
  uint32_t num_rendered;   // sum of tiles touched (the reference's R)
  uint32_t scan_tiles_done;
  uint32_t scan_tile_counter;
  uint32_t pad[10];
};

constexpr int kPreThreads = 256;  // Gaussians per preprocess block (one scan tile)

// ---------------------------------------------------------------------------
// Warp-cooperative staging of SH rows (preprocess and per-Gaussian backward)
// ---------------------------------------------------------------------------
constexpr int kShStride = 49;  // odd row stride: row reads by 32 threads hit 32 banks

__host__ __device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0u; }

// Vector forms for a full warp of degree-3 rows (M == 16): the warp's rows are
// one contiguous span, moved as float4s (coalesced 16-byte accesses; the span
// starts on a 16-byte boundary when the tensor does, since i0 is a multiple of
// 32), each float4's four elements placed by one division per float4.
constexpr int kVecBatch = 4;  // float4 loads in flight per lane

// Scatter float4 number f of a span of rows of `len` floats (row g's element c
// to s[g * stride + off + c]).
__device__ __forceinline__ void scatter4(float* s, int stride, int len, int off, int f, float4 v) {
  int g = (4 * f) / len, c = 4 * f - g * len;
  const float x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    s[g * stride + off + c] = x[w];
    if (++c == len) {
      c = 0;
      ++g;
    }
  }
}

// Stage the span of 32 rows of `len` floats at src (nf = 8 len float4s).
__device__ __forceinline__ void stage_span(const float* src, int len, float* s, int stride, int off) {
  const int lane = threadIdx.x & 31, nf = 8 * len;
  const float4* q = reinterpret_cast<const float4*>(src);
  for (int f0 = 0; f0 < nf; f0 += 32 * kVecBatch) {
    float4 v[kVecBatch];
#pragma unroll
    for (int u = 0; u < kVecBatch; ++u) {
      const int f = f0 + 32 * u + lane;
      v[u] = f < nf ? __ldg(q + f) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < kVecBatch; ++u) {
      const int f = f0 + 32 * u + lane;
      if (f < nf) scatter4(s, stride, len, off, f, v[u]);
    }
  }
}


constexpr int kSortTileMin = 4096;  // smallest onesweep tile of any key type: status words are sized for it
constexpr int kMaxPasses = 8;
constexpr int kMaxDigitBits = 9;             // digit width: ceil(bits / ceil(bits / 9))
constexpr int kMaxBins = 1 << kMaxDigitBits;

// Instance binning from depth-ordered Gaussians (binning.cu)
constexpr int kBinChunk = 4096;     // instance positions per CTA of the count / scatter kernels
constexpr int kBinShare = kBinChunk / 8;  // positions per warp of a chunk
constexpr int kMaxBinTiles = 4096;  // tile counts up to this use the binning path (1024 x 1024 at 16 x 16)
constexpr int kScanTileElems = 4096;  // elements per CTA of the stand-alone scan

struct GeomLayout {
  size_t header, scan_status, depth, clamped, means2D, cov3D, conic, rgb, tiles, offsets, rect, prev_reach,
      record, bwd_record, total;
  // the Gaussians by depth (single-view calls): sorted ids and keys, the
  // sort's ping-pong buffers, its histograms / counters / status words (one
  // span, cleared together), the owned-instance prefix and its scan scratch
  size_t dorder, dkeys, dtmp_keys, dtmp_vals, dprefix, dsort_hist, dsort_counters, dsort_status, dscan;
  // header and scan_status are adjacent so one memset clears both
  __host__ __device__ explicit GeomLayout(long long P) {
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t a = align256(o); o = a + bytes; return a; };
    const size_t p = size_t(P);
    header = take(sizeof(GeomHeader));
    scan_status = take(((p + kPreThreads - 1) / kPreThreads + 1) * 8);
    depth = take(p * 4);
    clamped = take(p * 3);
    means2D = take(p * 8);
    cov3D = take(p * 24);
    conic = take(p * 16);
    rgb = take(p * 12);
    tiles = take(p * 4);
    offsets = take(p * 4);
    rect = take(p * 8);
    prev_reach = take(p * 4);
    record = take(p * sizeof(BlendRecord));
    bwd_record = take(p * sizeof(BackwardRecord));
    dorder = take(p * 4);
    dkeys = take(p * 4);
    dtmp_keys = take(p * 4);
    dtmp_vals = take(p * 4);
    dprefix = take((p + 1) * 4);
    dsort_hist = take(size_t(kMaxPasses) * kMaxBins * 4);
    dsort_counters = take(size_t(kMaxPasses) * 4);
    dsort_status = take(size_t(kMaxPasses) * kMaxBins * ((p + kSortTileMin - 1) / kSortTileMin + 1) * 4);
    dscan = take(256 + ((p + kScanTileElems - 1) / kScanTileElems + 1) * 8);
    total = align256(o);
  }
};

struct ImageLayout {
  size_t n_contrib, ranges, T_final, tile_max, order, order_bwd, queue, total;
  __host__ __device__ ImageLayout(int W, int H)
      : ImageLayout(size_t(W) * size_t(H), size_t((W + kTile - 1) / kTile) * size_t((H + kTile - 1) / kTile)) {}
  // a batch: all items' pixels and tiles back to back
  __host__ __device__ ImageLayout(size_t hw, size_t tiles) {
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t a = align256(o); o = a + bytes; return a; };
    n_contrib = take(hw * 4);
    ranges = take(tiles * 8);
    T_final = take(hw * 4);
    tile_max = take(tiles * 4);
    order = take(tiles * 4);
    order_bwd = take(tiles * 4);
    queue = take(4);  // the persistent blend's tile queue counter
    total = align256(o);
  }
};

// Sort configuration chosen on the host from (R, depth-bit range, tile count).
struct BinHeader {
  uint32_t error;
  uint32_t key64;          // 1: 64-bit packed keys, 0: 32-bit packed keys
  uint32_t depth_bits;     // low depth bits kept in the key
  uint32_t depth_prefix;   // common high depth bits (restored when keys are expanded)
  uint32_t tile_bits;
  uint32_t passes;         // 8-bit digit passes
  uint32_t num_rendered;
  uint32_t masks_valid;    // 1: the blend wrote the block masks (BinLayout::masks) for the backward
  uint32_t n_sort;         // planned render: instances the emission and sort process (R, or 0 to replan)
  uint32_t replan;         // planned render: 1 when R or the depth range did not fit the plan
  uint32_t pad[6];
  uint32_t tile_counter[8];  // per-pass tile acquisition counters (onesweep)
};

constexpr int kSortThreads = 256;

struct BinLayout {
  size_t header, keysA, keysB, valsA, valsB, hist, status, tile_hist, bin_counts, warp_start, masks, total;
  __host__ __device__ BinLayout(long long R, int num_tiles) {
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t a = align256(o); o = a + bytes; return a; };
    const size_t r = size_t(R > 0 ? R : 1);
    const size_t sort_tiles = (r + kSortTileMin - 1) / kSortTileMin;
    header = take(sizeof(BinHeader));
    keysA = take(r * 8);
    keysB = take(r * 8);
    valsA = take(r * 4);
    valsB = take(r * 4);
    // hist, tile_hist, then status: one memset clears them and the used
    // passes' status words
    hist = take(size_t(kMaxPasses) * kMaxBins * 4);
    tile_hist = take(size_t(num_tiles > 0 ? num_tiles : 1) * 4);
    status = take(size_t(kMaxPasses) * sort_tiles * kMaxBins * 4);
    // binning path (tile counts up to kMaxBinTiles): the chunk x tile matrix
    // and every warp share's first depth-order index
    const size_t chunks = num_tiles > 0 && num_tiles <= kMaxBinTiles ? (r + kBinChunk - 1) / kBinChunk : 0;
    bin_counts = take(chunks * size_t(num_tiles > 0 ? num_tiles : 0) * 4);
    warp_start = take(chunks ? ((r + kBinShare - 1) / kBinShare + 1) * 4 : 0);
    // the blend's block masks per list position: the tile's upper blocks, then its lower blocks
    masks = take(2 * r);
    total = align256(o);
  }
};

// ---------------------------------------------------------------------------
// Bounded waits and release/acquire helpers
// ---------------------------------------------------------------------------
constexpr uint32_t kSpinLimit = 1u << 22;   // per wait; each poll is an L2 round trip, so 1-2 s at most

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Relaxed (non-ordering) atomic-visibility accesses, for status words whose
// readers need nothing else the writer wrote.
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

}  // namespace w2w
