// Per-Gaussian forward stage, one fused kernel:
//   EWA projection             (reference projection.cu:7-154)
//   ADR radius + tile count    (ADRculling.cu:33-107)
//   SH colour, degree <= 3     (gaussianForwardPass.cu:11-39, 172-263)
//   key-emission rectangle     (prepareSort.cu:272-282)
//   inclusive scan of tile counts (gaussianRasterizer.cu:77-117), done here as a
//   single-pass decoupled-lookback scan fused with the projection.
//
// The scan carries a second, max-plus component: for every Gaussian the
// largest end slot any earlier Gaussian writes (its start + emitted count).
// In the reference, a Gaussian whose emission rectangle is larger than its
// allocation writes past its slot range into its successors' slots; with this
// prefix maximum each slot gets exactly one deterministic writer (the lowest
// index whose emission covers it), so the key emission is race-free.
#include "common.cuh"
#include "kernels.h"

namespace w2w {

namespace {

// SH constants of the reference forward (gaussianForwardPass.cu:11-39, 199)
constexpr float kC0 = 0.28209479177387814f;
constexpr float kC1 = 0.4886025119029199f;
constexpr float kC2a = 1.0925484305920792f;
constexpr float kC2e = 0.5462742152960396f;
constexpr float kC30 = 0.5900435899266435f;
constexpr float kC31 = 2.890611442640554f;
constexpr float kC32 = 0.4570457994644658f;
constexpr float kC33 = 0.3731763325901154f;
constexpr float kC35 = 1.445305721320277f;

// Scan element: (sum of allocations, max over the span of local start +
// emitted count, whether a view starts inside the span).  The max-plus
// component restarts at a view's first Gaussian: a batched call's views are
// independent key emissions (the spill of one view never reaches the next),
// exactly as separate calls.
struct Pair {
  uint32_t s, x, f;
};
__device__ __forceinline__ Pair combine(Pair lo, Pair hi) {
  return Pair{lo.s + hi.s, hi.f ? lo.s + hi.x : max(lo.x, lo.s + hi.x), lo.f | hi.f};
}

constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagInc = 2ull << 62;
constexpr uint32_t kPairMask = (1u << 30) - 1u;  // counts below 2^30
__device__ __forceinline__ unsigned long long pack(unsigned long long flag, Pair p) {
  return flag | ((unsigned long long)(p.f & 1u) << 60) | ((unsigned long long)(p.s & kPairMask) << 30) |
         (unsigned long long)(p.x & kPairMask);
}
__device__ __forceinline__ Pair unpack(unsigned long long w) {
  return Pair{uint32_t((w >> 30) & kPairMask), uint32_t(w & kPairMask), uint32_t((w >> 60) & 1u)};
}

template <int V>
__device__ __forceinline__ float pixel_coord(float c, float invW, float nd, float S) {
  float t = (V >= 2) ? fma(c, invW, 1.0f) : add(nd, 1.0f);
  t = mul(t, 0.5f);
  return (V == 1 || V == 2) ? fma(t, S, -0.5f) : add(mul(t, S), -0.5f);
}

struct Geometry {
  float cov3[6];
  float depth, mx, my;
  float cxx, cxy, cyy, det;
  float conic[3];
  bool visible;
};

// Projection, restating projection.cu:30-153 with the pinned fusion patterns.
__device__ __forceinline__ void project(const float* __restrict__ V, const float* __restrict__ PM, float focal,
                                        float W, float H, float px, float py, float pz, float sx, float sy,
                                        float sz, float4 q, Geometry& g) {
  using namespace fp;
  const float r = q.x, x = q.y, y = q.z, z = q.w;
  float R[3][3];
  R[0][0] = mul(0.5f, sub(2.0f, mul(4.0f, s2<RQ0>(y, y, z, z))));
  R[0][1] = mul(0.5f, mul(4.0f, d2<RQ1>(x, y, r, z)));
  R[0][2] = mul(0.5f, mul(4.0f, s2<RQ2>(x, z, r, y)));
  R[1][0] = mul(0.5f, mul(4.0f, s2<RQ3>(x, y, r, z)));
  R[1][1] = mul(0.5f, sub(2.0f, mul(4.0f, s2<RQ4>(x, x, z, z))));
  R[1][2] = mul(0.5f, mul(4.0f, d2<RQ5>(y, z, r, x)));
  R[2][0] = mul(0.5f, mul(4.0f, d2<RQ6>(x, z, r, y)));
  R[2][1] = mul(0.5f, mul(4.0f, s2<RQ7>(y, z, r, x)));
  R[2][2] = mul(0.5f, sub(2.0f, mul(4.0f, s2<RQ8>(x, x, y, y))));
  const float s[3] = {sx, sy, sz};
  float A[3][3];  // (R^T S^T S)[c][row] = R[row][c] * s_c * s_c
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int rr = 0; rr < 3; ++rr) A[c][rr] = mul(mul(R[rr][c], s[c]), s[c]);
  g.cov3[0] = s3<SIGMA0>(A[0][0], R[0][0], A[1][0], R[0][1], A[2][0], R[0][2]);
  g.cov3[1] = s3<SIGMA1>(A[0][1], R[0][0], A[1][1], R[0][1], A[2][1], R[0][2]);
  g.cov3[2] = s3<SIGMA2>(A[0][2], R[0][0], A[1][2], R[0][1], A[2][2], R[0][2]);
  g.cov3[3] = s3<SIGMA3>(A[0][1], R[1][0], A[1][1], R[1][1], A[2][1], R[1][2]);
  g.cov3[4] = s3<SIGMA4>(A[0][2], R[1][0], A[1][2], R[1][1], A[2][2], R[1][2]);
  g.cov3[5] = s3<SIGMA5>(A[0][2], R[2][0], A[1][2], R[2][1], A[2][2], R[2][2]);

  float tx = m4row<VIEW_A0, VIEW_B0>(V, 0, px, py, pz);
  float ty = m4row<VIEW_A1, VIEW_B1>(V, 1, px, py, pz);
  float tz = m4row<VIEW_A2, VIEW_B2>(V, 2, px, py, pz);
  const float tw = m4row<VIEW_A3, VIEW_B3>(V, 3, px, py, pz);
  tx = div(tx, tw);
  ty = div(ty, tw);
  tz = div(tz, tw);
  g.visible = false;
  if (tz <= 1.0f) return;  // projection.cu:75

  // inscribed-circle clamp (projection.cu:22, 78-92); the reference's 800 is W
  const float limit = div(W, mul(2.0f, focal));
  float rsx = div(tx, tz), rsy = div(ty, tz);
  const float nx = div(rsx, limit), ny = div(rsy, limit);
  const float sq = s2<RAYR2>(nx, nx, ny, ny);
  if (sq > 1.0f) {
    const float sc = rsqrtf(sq);  // the reference's approximate reciprocal square root
    rsx = mul(rsx, sc);
    rsy = mul(rsy, sc);
  }
  tx = mul(rsx, tz);
  ty = mul(rsy, tz);

  const float zi = __frcp_rn(tz);
  const float zi2 = mul(zi, zi);
  float jx[3], jy[3];
  jx[0] = mul(focal, d2<DPROJ0>(V[0], zi, mul(tx, V[2]), zi2));
  jx[1] = mul(focal, d2<DPROJ1>(V[4], zi, mul(tx, V[6]), zi2));
  jx[2] = mul(focal, d2<DPROJ2>(V[8], zi, mul(tx, V[10]), zi2));
  jy[0] = mul(focal, d2<DPROJ3>(V[1], zi, mul(ty, V[2]), zi2));
  jy[1] = mul(focal, d2<DPROJ4>(V[5], zi, mul(ty, V[6]), zi2));
  jy[2] = mul(focal, d2<DPROJ5>(V[9], zi, mul(ty, V[10]), zi2));
  const float* c = g.cov3;
  const float Sx0 = s3<SIGV0>(c[0], jx[0], c[1], jx[1], c[2], jx[2]);
  const float Sx1 = s3<SIGV1>(c[1], jx[0], c[3], jx[1], c[4], jx[2]);
  const float Sx2 = s3<SIGV2>(c[2], jx[0], c[4], jx[1], c[5], jx[2]);
  const float Sy0 = s3<SIGV3>(c[0], jy[0], c[1], jy[1], c[2], jy[2]);
  const float Sy1 = s3<SIGV4>(c[1], jy[0], c[3], jy[1], c[4], jy[2]);
  const float Sy2 = s3<SIGV5>(c[2], jy[0], c[4], jy[1], c[5], jy[2]);
  const float cxx = s3<DOT30>(jx[0], Sx0, jx[1], Sx1, jx[2], Sx2);
  const float cxy = s3<DOT31>(jx[0], Sy0, jx[1], Sy1, jx[2], Sy2);
  const float cyy = s3<DOT32>(jy[0], Sy0, jy[1], Sy1, jy[2], Sy2);
  const float det = d2<DET>(cxx, cyy, cxy, cxy);
  if (fabsf(det) < 1e-8f) return;  // projection.cu:116
  const float dinv = __frcp_rn(det);
  g.conic[0] = mul(cyy, dinv);
  g.conic[1] = mul(-cxy, dinv);
  g.conic[2] = mul(cxx, dinv);
  g.cxx = cxx;
  g.cxy = cxy;
  g.cyy = cyy;
  g.det = det;

  const float cx = m4row<PROJ_A0, PROJ_B0>(PM, 0, px, py, pz);
  const float cy = m4row<PROJ_A1, PROJ_B1>(PM, 1, px, py, pz);
  const float cz = m4row<PROJ_A2, PROJ_B2>(PM, 2, px, py, pz);
  const float cw = m4row<PROJ_A3, PROJ_B3>(PM, 3, px, py, pz);
  const float invW = __frcp_rn(add(cw, 0.00001f));
  g.mx = pixel_coord<PIX0>(cx, invW, mul(cx, invW), W);
  g.my = pixel_coord<PIX1>(cy, invW, mul(cy, invW), H);
  g.depth = mul(cz, invW);
  g.visible = true;
}

// k*zz - xx - yy with the squares optionally fused into the subtractions
template <int V>
__device__ __forceinline__ float kzz(float k, float x, float y, float xx, float yy, float zz) {
  if constexpr (V == 1) return fma(-y, y, fma(-x, x, mul(k, zz)));
  else if constexpr (V == 2) return fma(-y, y, sub(mul(k, zz), xx));
  else if constexpr (V == 3) return sub(fma(-x, x, mul(k, zz)), yy);
  else return sub(sub(mul(k, zz), xx), yy);
}
// xx - yy
template <int V>
__device__ __forceinline__ float xmy(float x, float y, float xx, float yy) {
  if constexpr (V == 1) return fma(x, x, -yy);
  else if constexpr (V == 2) return fma(-y, y, xx);
  else return sub(xx, yy);
}

// SH colour (gaussianForwardPass.cu:195-263); coefficients needed by a degree
// are used only when stored (degree d needs (d+1)^2 of them).
__device__ __forceinline__ void sh_colour(const float* __restrict__ sh, int M, int deg, float px, float py, float pz,
                                          const float* __restrict__ campos, float rgb[3], uint8_t clamped[3]) {
  using namespace fp;
  const float vx = sub(px, campos[0]), vy = sub(py, campos[1]), vz = sub(pz, campos[2]);
  const float l2 = s3<SH_DOT>(vx, vx, vy, vy, vz, vz);
  const float inv = __frcp_rn(__fsqrt_rn(l2));
  const float x = mul(vx, inv), y = mul(vy, inv), z = mul(vz, inv);
  float o0 = mul(kC0, sh[0]), o1 = mul(kC0, sh[1]), o2 = mul(kC0, sh[2]);
  auto acc = [&](float coef, int idx) {
    o0 = s1<SH_ACC>(coef, sh[3 * idx + 0], o0);
    o1 = s1<SH_ACC>(coef, sh[3 * idx + 1], o1);
    o2 = s1<SH_ACC>(coef, sh[3 * idx + 2], o2);
  };
  if (deg >= 1 && M > 3) {
    acc(mul(-kC1, y), 1);
    acc(mul(kC1, z), 2);
    acc(mul(-kC1, x), 3);
  }
  const float xx = mul(x, x), yy = mul(y, y), zz = mul(z, z);
  if (deg >= 2 && M > 8) {
    const float xy = mul(x, y), yz = mul(y, z), xz = mul(x, z);
    acc(mul(kC2a, xy), 4);
    acc(mul(-kC2a, yz), 5);
    acc(mul(0.3f, kzz<SH2A>(2.0f, x, y, xx, yy, zz)), 6);
    acc(mul(-kC2a, xz), 7);
    acc(mul(kC2e, xmy<SH2B>(x, y, xx, yy)), 8);
  }
  if (deg >= 3 && M > 15) {
    // 3xx - yy, 2zz - 3xx - 3yy and xx - 3yy with the reference's fusions
    const float t9 = SH3A == 1 ? fma(3.0f, xx, -yy) : SH3A == 2 ? fma(-y, y, mul(3.0f, xx)) : sub(mul(3.0f, xx), yy);
    const float t12 = SH3C == 1 ? fma(-3.0f, yy, fma(-3.0f, xx, mul(2.0f, zz)))
                    : SH3C == 2 ? fma(-3.0f, yy, sub(mul(2.0f, zz), mul(3.0f, xx)))
                    : SH3C == 3 ? sub(fma(-3.0f, xx, mul(2.0f, zz)), mul(3.0f, yy))
                                : sub(sub(mul(2.0f, zz), mul(3.0f, xx)), mul(3.0f, yy));
    const float t15 = SH3E == 1 ? fma(-3.0f, yy, xx) : SH3E == 2 ? fma(x, x, -mul(3.0f, yy)) : sub(xx, mul(3.0f, yy));
    acc(mul(mul(-kC30, y), t9), 9);
    acc(mul(mul(mul(kC31, x), y), z), 10);
    acc(mul(mul(-kC32, y), kzz<SH3B>(4.0f, x, y, xx, yy, zz)), 11);
    acc(mul(mul(kC33, z), t12), 12);
    acc(mul(mul(-kC32, x), kzz<SH3B>(4.0f, x, y, xx, yy, zz)), 13);
    acc(mul(mul(kC35, z), xmy<SH3D>(x, y, xx, yy)), 14);
    acc(mul(mul(-kC30, x), t15), 15);
  }
  rgb[0] = add(o0, 0.5f);
  rgb[1] = add(o1, 0.5f);
  rgb[2] = add(o2, 0.5f);
#pragma unroll
  for (int k = 0; k < 3; ++k) clamped[k] = rgb[k] < 0.0f ? 1 : 0;
}

// 4 CTAs per SM (64 registers, a few spilled): measured 2 % faster than 3 at 80.
// kRaw: the raw parameters of Renderer.render, activated here (PreprocessArgs).
// kStage: degree-3 rows (M == 16) of a full warp are staged through shared
// memory as coalesced float4 spans (dynamic shared memory, kStageBytes) instead
// of each thread gathering its own 192-byte row.
constexpr int kStageBytes = kPreThreads * kShStride * 4;

// kMinBlocks: CTAs per SM the register budget is sized for (the tuning knob
// "preprocess_blocks"): 4 caps a thread at 64 registers (some spill to local
// memory), 3 at 80, 2 at 128 (none spill).
template <bool kSh16, bool kRaw, bool kStage, int kMinBlocks>
__global__ void __launch_bounds__(kPreThreads, kMinBlocks)
preprocess_kernel(PreprocessArgs a) {
  __shared__ uint32_t s_tile;
  __shared__ Pair s_warp[kPreThreads / 32];
  __shared__ Pair s_prefix;
  extern __shared__ __align__(16) float s_rows[];
  GeomHeader* hdr = a.header;
  if (threadIdx.x == 0) s_tile = atomicAdd(&hdr->scan_tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const int i = int(tile) * kPreThreads + int(threadIdx.x);
  const int P = a.P;

  // this element's scene and camera: the call's, or its batch item's
  int gi = i, item = -1;
  const float *means3D = a.means3D, *scales = a.scales, *rotations = a.rotations, *opacities = a.opacities,
              *shs = a.shs, *view = a.view, *proj = a.proj, *campos = a.campos;
  int M = a.M, degree = a.degree, Wd = a.W, Hd = a.H, item_P = P;
  float focal = a.focal_x;
  if (a.items != nullptr && i < P) {
    item = find_item_elem(a.items, a.num_items, uint32_t(i));
    const BatchItem& it = a.items[item];
    gi = i - int(it.elem_base);
    means3D = it.means3D; scales = it.scales; rotations = it.rotations; opacities = it.opacities; shs = it.shs;
    view = it.view; proj = it.proj; campos = it.campos;
    M = it.M; degree = it.degree; Wd = it.W; Hd = it.H; item_P = it.P;
    focal = it.focal_x;
  }
  const int gw = (Wd + kTile - 1) / kTile, gh = (Hd + kTile - 1) / kTile;

  // this warp's SH rows, staged when all 32 of its Gaussians exist (and, in a
  // batched call, belong to one scene with 16 coefficients)
  const int i0 = int(tile) * kPreThreads + int(threadIdx.x & ~31u);
  bool staged = kStage && i0 + 32 <= P;  // warp-uniform
  const float* span = kRaw ? nullptr : a.shs + size_t(i0) * 48;  // the warp's first row
  if (staged && a.items != nullptr) {
    const int f = find_item_elem(a.items, a.num_items, uint32_t(i0));
    staged = f == find_item_elem(a.items, a.num_items, uint32_t(i0 + 31)) && a.items[f].M == 16;
    span = a.items[f].shs + size_t(i0 - int(a.items[f].elem_base)) * 48;
  }
  const float* srow = s_rows + int(threadIdx.x >> 5) * 32 * kShStride;
  if (staged) {
    float* w = s_rows + int(threadIdx.x >> 5) * 32 * kShStride;
    if (kRaw) {
      stage_span(a.sh_dc + size_t(i0) * 3, 3, w, kShStride, 0);
      stage_span(a.sh_ac + size_t(i0) * 45, 45, w, kShStride, 3);
    } else {
      stage_span(span, 48, w, kShStride, 0);
    }
    __syncwarp();
  }
  srow += int(threadIdx.x & 31) * kShStride;

  uint32_t alloc = 0, emit = 0;
  uint32_t depth_bits = 0;
  if (i < P) {
    const float px = means3D[3 * gi], py = means3D[3 * gi + 1], pz = means3D[3 * gi + 2];
    float sx, sy, sz, opacity;
    float4 q;
    if constexpr (kRaw) {
      sx = expf(a.svec[3 * gi]);
      sy = expf(a.svec[3 * gi + 1]);
      sz = expf(a.svec[3 * gi + 2]);
      q = act_normalize(a.quat[4 * gi], a.quat[4 * gi + 1], a.quat[4 * gi + 2], a.quat[4 * gi + 3]);
      opacity = act_sigmoid(a.logit[gi]);
    } else {
      sx = scales[3 * gi];
      sy = scales[3 * gi + 1];
      sz = scales[3 * gi + 2];
      q = make_float4(rotations[4 * gi], rotations[4 * gi + 1], rotations[4 * gi + 2], rotations[4 * gi + 3]);
      opacity = opacities[gi];
    }
    Geometry g;
    project(view, proj, focal, float(Wd), float(Hd), px, py, pz, sx, sy, sz, q, g);
    float* cov3 = a.cov3D + 6 * size_t(i);
#pragma unroll
    for (int k = 0; k < 6; ++k) cov3[k] = g.cov3[k];

    // SH colour
    float rgb[3];
    uint8_t clampf[3];
    const float* shp = kRaw ? nullptr : shs + size_t(gi) * M * 3;
    if (staged) {
      sh_colour(srow, 16, degree, px, py, pz, campos, rgb, clampf);
    } else if constexpr (kRaw) {  // the row is sh_dc (3 floats) then sh_ac (3 (M - 1) floats); M <= 16
      float buf[48];
      const float* dc = a.sh_dc + 3 * size_t(gi);
      const float* ac = a.sh_ac + size_t(gi) * 3 * (M - 1);
      // only the coefficients the degree uses: (degree + 1)^2 of the M stored
      const int used = 3 * min(M, (degree + 1) * (degree + 1));
#pragma unroll
      for (int k = 0; k < 3; ++k) buf[k] = __ldg(dc + k);
#pragma unroll
      for (int k = 3; k < 48; ++k) buf[k] = k < used ? __ldg(ac + (k - 3)) : 0.f;
      sh_colour(buf, M, degree, px, py, pz, campos, rgb, clampf);
    } else if constexpr (kSh16) {
      float buf[48];
      const float4* s4 = reinterpret_cast<const float4*>(shp);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        const float4 t = __ldg(s4 + k);
        buf[4 * k] = t.x; buf[4 * k + 1] = t.y; buf[4 * k + 2] = t.z; buf[4 * k + 3] = t.w;
      }
      sh_colour(buf, 16, degree, px, py, pz, campos, rgb, clampf);
    } else {
      sh_colour(shp, M, degree, px, py, pz, campos, rgb, clampf);
    }
    reinterpret_cast<float*>(a.rgb)[3 * i] = rgb[0];
    reinterpret_cast<float*>(a.rgb)[3 * i + 1] = rgb[1];
    reinterpret_cast<float*>(a.rgb)[3 * i + 2] = rgb[2];
    a.clamped[3 * i] = clampf[0];
    a.clamped[3 * i + 1] = clampf[1];
    a.clamped[3 * i + 2] = clampf[2];

    int radius = 0;
    uint32_t rect_lo = 0, rect_hi = 0;
    BlendRecord rec{};
    if (g.visible) {
      // ADR culling (ADRculling.cu:39-107)
      using namespace fp;
      const float ht = mul(add(g.cxx, g.cyy), 0.5f);
      const float dsq = s1<ADR_DELTA>(ht, ht, -g.det);
      const float root = __fsqrt_rn(fmaxf(0.1f, dsq));
      const float ymax = fmaxf(add(ht, root), sub(ht, root));
      const float allp = mul(3.0f, __fsqrt_rn(ymax));
      if (!(opacity <= 0.0039f)) {
        const float ln = logf(mul(opacity, 255.0f));
        const float adapt = __fsqrt_rn(mul(mul(2.0f, ymax), ln));
        const float mr = fminf(adapt, allp);
        radius = int(ceilf(mr));
        int x0 = int(div(sub(g.mx, mr), 16.0f));
        int y0 = int(div(sub(g.my, mr), 16.0f));
        int x1 = int(div(add(add(g.mx, mr), 15.0f), 16.0f));
        int y1 = int(div(add(add(g.my, mr), 15.0f), 16.0f));
        x0 = max(0, x0); y0 = max(0, y0);
        x1 = min(gw, x1); y1 = min(gh, y1);
        x1 = max(x1, x0); y1 = max(y1, y0);
        alloc = uint32_t(x1 - x0) * uint32_t(y1 - y0);
        if (a.compat_spill) {
          // emission rectangle of prepareSort.cu:279-282 (integer radius, floor/ceil)
          const float rf = float(radius);
          const int ex0 = min(gw, max(0, int(floorf(div(sub(g.mx, rf), 16.0f)))));
          const int ex1 = min(gw, max(0, int(ceilf(div(add(g.mx, rf), 16.0f)))));
          const int ey0 = min(gh, max(0, int(floorf(div(sub(g.my, rf), 16.0f)))));
          const int ey1 = min(gh, max(0, int(ceilf(div(add(g.my, rf), 16.0f)))));
          x0 = ex0; x1 = ex1; y0 = ey0; y1 = ey1;
        }
        emit = uint32_t(x1 - x0) * uint32_t(y1 - y0);
        rect_lo = uint32_t(x0) | (uint32_t(y0) << 16);
        rect_hi = uint32_t(x1) | (uint32_t(y1) << 16);
      }
      rec.mx = g.mx; rec.my = g.my;
      rec.cxx = g.cxx; rec.cxy = g.cxy; rec.cyy = g.cyy;
      rec.det = d2<BL_DET>(g.cxx, g.cyy, g.cxy, g.cxy);
      rec.opacity = opacity;
      rec.depth = g.depth;
      rec.r = rgb[0]; rec.g = rgb[1]; rec.b = rgb[2];
      reinterpret_cast<float4*>(a.conic)[i] = make_float4(g.conic[0], g.conic[1], g.conic[2], opacity);
      reinterpret_cast<float2*>(a.means2D)[i] = make_float2(g.mx, g.my);
      a.depth[i] = g.depth;
    } else {
      reinterpret_cast<float4*>(a.conic)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      reinterpret_cast<float2*>(a.means2D)[i] = make_float2(0.f, 0.f);
      a.depth[i] = 0.f;
    }
    if (radius <= 0) { alloc = 0; emit = 0; }
    if (emit > 0) depth_bits = __float_as_uint(g.depth);
    a.radii[i] = radius;
    a.tiles[i] = alloc;
    reinterpret_cast<uint2*>(a.rect)[i] = make_uint2(rect_lo, rect_hi);
    // backward skip threshold (BackwardRecord::skip) and block-culling parameters
    float skip = -__int_as_float(0x7f800000);
    CullParams cp{-1.0f, 0.f, 0.f, 0.f, 0.f};
    if (g.visible) {
      skip = opacity > 0.0f ? -logf(255.0f * opacity) - 1e-4f : __int_as_float(0x7f800000);
      cp = make_cull_params(g.conic[0], g.conic[1], g.conic[2], opacity);
    }
    float4* rp = reinterpret_cast<float4*>(a.record) + 4 * size_t(i);
    rp[0] = make_float4(rec.mx, rec.my, rec.cxx, rec.cxy);
    rp[1] = make_float4(rec.cyy, rec.det, rec.opacity, rec.depth);
    rp[2] = make_float4(rec.r, rec.g, rec.b, cp.hy);
    rp[3] = make_float4(cp.beta, cp.gamma, cp.eps, cp.vr);
    float4* bp = reinterpret_cast<float4*>(a.bwd_record) + 4 * size_t(i);
    if (g.visible) {
      bp[0] = make_float4(g.mx, g.my, g.conic[0], g.conic[1]);
      bp[1] = make_float4(g.conic[2], opacity, g.depth, rgb[0]);
      bp[2] = make_float4(rgb[1], rgb[2], skip, cp.hy);
      bp[3] = make_float4(cp.beta, cp.gamma, cp.eps, cp.vr);
    } else {
      bp[0] = bp[1] = bp[2] = make_float4(0.f, 0.f, 0.f, 0.f);
      bp[3] = make_float4(0.f, 0.f, 0.f, 0.f);
      bp[2].w = -1.0f;
    }
  }

  // depth-bit range of Gaussians that emit keys (sizes the sort)
  {
    const bool has = emit > 0;
    const uint32_t mn = has ? depth_bits : 0xffffffffu;
    const uint32_t mxv = has ? depth_bits : 0u;
    const uint32_t wmn = __reduce_min_sync(0xffffffffu, mn);
    const uint32_t wmx = __reduce_max_sync(0xffffffffu, mxv);
    const bool any = __any_sync(0xffffffffu, has);
    if (any && (threadIdx.x & 31) == 0) {
      atomicMax(&hdr->depth_min, ~wmn);  // stored inverted so a zeroed header means "none"
      atomicMax(&hdr->depth_max, wmx);
    }
  }

  // block-wide inclusive scan of (alloc, emit) with the max-plus component
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Pair v{alloc, emit, uint32_t(i < P && gi == 0)};
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    Pair o;
    o.s = __shfl_up_sync(0xffffffffu, v.s, d);
    o.x = __shfl_up_sync(0xffffffffu, v.x, d);
    o.f = __shfl_up_sync(0xffffffffu, v.f, d);
    if (lane >= d) v = combine(o, v);
  }
  if (lane == 31) s_warp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    Pair w = lane < kPreThreads / 32 ? s_warp[lane] : Pair{0, 0, 0};
#pragma unroll
    for (int d = 1; d < kPreThreads / 32; d <<= 1) {
      Pair o;
      o.s = __shfl_up_sync(0xffffffffu, w.s, d);
      o.x = __shfl_up_sync(0xffffffffu, w.x, d);
      o.f = __shfl_up_sync(0xffffffffu, w.f, d);
      if (lane >= d) w = combine(o, w);
    }
    if (lane < kPreThreads / 32) s_warp[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const Pair block_total = s_warp[kPreThreads / 32 - 1];
  // decoupled lookback by warp 0; each status word carries its flag and pair
  // together and nothing else written by its tile is read, so relaxed
  // accesses suffice.  Each step reads the 32 tiles before t at once and,
  // once every one of them up to the nearest inclusive prefix has published,
  // combines them in index order (an ordered shuffle tree, older tiles on the
  // left); a serial walk would cost one L2 round trip per tile.
  if (warp == 0) {
    unsigned long long* status = a.scan_status;
    const bool publish = (long long)tile != a.unpublished_tile;
    if (tile == 0) {
      if (lane == 0) {
        if (publish) st_relaxed64(status + tile, pack(kFlagInc, block_total));
        s_prefix = Pair{0, 0, 0};
      }
    } else {
      if (lane == 0 && publish) st_relaxed64(status + tile, pack(kFlagAgg, block_total));
      // (0, 0, 0) is an identity on both sides for every pair that occurs
      Pair ex{0, 0, 0};
      long long t = int(tile) - 1;
      uint32_t spins = 0;
      while (true) {
        const long long q = t - lane;
        const unsigned long long w = q >= 0 ? ld_relaxed64(status + q) : kFlagInc;
        const unsigned long long flag = w & (3ull << 62);
        const uint32_t inc = __ballot_sync(0xffffffffu, flag == kFlagInc);
        const uint32_t ready = __ballot_sync(0xffffffffu, flag != 0ull);
        const uint32_t need = inc ? ((inc & (0u - inc)) << 1) - 1u : 0xffffffffu;
        if ((ready & need) != need) {
          if (++spins > a.spin_limit) {
            if (lane == 0) atomicOr(&hdr->error, kErrTimeout);
            break;
          }
          continue;
        }
        Pair p = (need >> lane) & 1u ? unpack(w) : Pair{0, 0, 0};
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          Pair o;
          o.s = __shfl_down_sync(0xffffffffu, p.s, d);
          o.x = __shfl_down_sync(0xffffffffu, p.x, d);
          o.f = __shfl_down_sync(0xffffffffu, p.f, d);
          if (lane + d < 32) p = combine(o, p);
        }
        ex = combine(p, ex);  // lane 0 holds the window; the walk so far is newer
        if (inc) break;
        t -= 32;
      }
      if (lane == 0) {
        s_prefix = ex;
        if (publish) st_relaxed64(status + tile, pack(kFlagInc, combine(ex, block_total)));
      }
    }
  }
  __syncthreads();
  // Exclusive value of this Gaussian.  Every Gaussian emits at least its
  // allocation, so a prefix's max-plus component is never below its sum and
  // (0, 0) is an identity on both sides for all prefixes that occur.
  const Pair prefix = s_prefix;
  Pair ex_lane;
  ex_lane.s = __shfl_up_sync(0xffffffffu, v.s, 1);
  ex_lane.x = __shfl_up_sync(0xffffffffu, v.x, 1);
  ex_lane.f = __shfl_up_sync(0xffffffffu, v.f, 1);
  if (lane == 0) ex_lane = Pair{0, 0, 0};
  const Pair ex_warps = warp > 0 ? s_warp[warp - 1] : Pair{0, 0, 0};
  const Pair excl = combine(prefix, combine(ex_warps, ex_lane));
  if (i < P) {
    a.offsets[i] = excl.s + alloc;
    // a view's first Gaussian has no earlier writer in its view
    a.prev_reach[i] = gi == 0 ? excl.s : excl.x;
    if (item >= 0 && gi == item_P - 1) a.item_end[item] = excl.s + alloc;
  }
  if (tile == uint32_t((P + kPreThreads - 1) / kPreThreads) - 1 && threadIdx.x == 0) {
    const Pair total = tile > 0 ? combine(prefix, block_total) : block_total;
    hdr->num_rendered = total.s;
    if (total.s >= kPairMask || total.x >= kPairMask) atomicOr(&hdr->error, kErrCapacity);
  }
}

}  // namespace

namespace {
template <int kMinBlocks>
void launch_preprocess_as(const PreprocessArgs& a, int blocks, bool raw, bool stage, bool sh16, cudaStream_t stream) {
  // the dynamic shared-memory opt-in of the staging kernels, once per device
  static bool opted[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (stage && (dev < 0 || dev >= 64 || !opted[dev])) {
    cudaFuncSetAttribute(preprocess_kernel<true, false, true, kMinBlocks>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes);
    cudaFuncSetAttribute(preprocess_kernel<false, true, true, kMinBlocks>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes);
    if (dev >= 0 && dev < 64) opted[dev] = true;
  }
  if (raw && stage) preprocess_kernel<false, true, true, kMinBlocks><<<blocks, kPreThreads, kStageBytes, stream>>>(a);
  else if (raw) preprocess_kernel<false, true, false, kMinBlocks><<<blocks, kPreThreads, 0, stream>>>(a);
  else if (stage) preprocess_kernel<true, false, true, kMinBlocks><<<blocks, kPreThreads, kStageBytes, stream>>>(a);
  else if (sh16) preprocess_kernel<true, false, false, kMinBlocks><<<blocks, kPreThreads, 0, stream>>>(a);
  else preprocess_kernel<false, false, false, kMinBlocks><<<blocks, kPreThreads, 0, stream>>>(a);
}
}  // namespace

void launch_preprocess(const PreprocessArgs& a, cudaStream_t stream) {
  const int blocks = (a.P + kPreThreads - 1) / kPreThreads;
  if (blocks == 0) return;
  // degree 3 with 16 stored coefficients reads whole rows: staged spans; a
  // lower degree reads only its first (degree + 1)^2 coefficients per thread
  // (a batched call sets M = 16 and shs non-null when every scene's rows are
  // 16-byte aligned with 16 coefficients; its degrees are per scene)
  const bool raw = a.svec != nullptr;
  const bool batched = a.items != nullptr;
  const bool full_rows = a.M == 16 && (batched ? a.shs != nullptr : a.degree == 3);
  const bool stage = full_rows && (raw ? aligned16(a.sh_dc) && aligned16(a.sh_ac) : aligned16(a.shs));
  const bool sh16 = !raw && full_rows && aligned16(a.shs);
  stage_begin(kStPreprocess, stream);
  switch (tune_value(kTunePreBlocks)) {
    case 2: launch_preprocess_as<2>(a, blocks, raw, stage, sh16, stream); break;
    case 3: launch_preprocess_as<3>(a, blocks, raw, stage, sh16, stream); break;
    default: launch_preprocess_as<4>(a, blocks, raw, stage, sh16, stream); break;
  }
  stage_end(kStPreprocess, stream, 1);
}

}  // namespace w2w
