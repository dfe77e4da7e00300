// Voxel occupancy field of a Gaussian set (reference compute_voxel_field.cu:25-86,
// driven by compute_voxel_field_wrapper.py:79-103), used to extract a mesh.
//
// Voxel (i, j, k) of an R^3 grid sits at p = -1 + 2 (i, j, k) / (R - 1); the
// cube [-1, 1]^3 is cut into B^3 blocks of side s = 2 / B, and a voxel's
// block is floor((p + 1) / s) per axis (the last voxel falls in block B).
// Its value is the sum, over the Gaussians whose mean lies within its block
// grown by relax * s on every side, in Gaussian order, of
// opacity * exp(power), power = -1/2 d^T Sigma^-1 d (positive powers give 0).
//
// The reference loops over every Gaussian for every voxel (R^3 * P tests).
// Here each Gaussian is binned once into the blocks whose grown bounds hold its
// mean (a few per Gaussian), the bins are sorted by block with the stable
// onesweep sort (so each block's list keeps Gaussian order, and with it the
// reference's summation order), and each voxel walks only its block's list;
// the inverse covariance is computed once per Gaussian instead of once per
// voxel-Gaussian pair.
#include "common.cuh"
#include "kernels.h"

namespace w2w {
namespace {

constexpr int kVoxThreads = 256;

__device__ __forceinline__ float vox_coord(int i, int R) {
  return __fadd_rn(-1.0f, __fdiv_rn(__fmul_rn(2.0f, float(i)), float(R - 1)));
}
__device__ __forceinline__ int vox_block(float p, float bs) {
  return __float2int_rz(__fdiv_rn(__fadd_rn(p, 1.0f), bs));
}
__device__ __forceinline__ int vox_block_clamped(float p, float bs, int B) {
  return min(max(vox_block(p, bs), 0), B);
}
// Grown bounds of block b along one axis.
__device__ __forceinline__ float vox_lo(int b, float bs, float relax) {
  return __fsub_rn(__fadd_rn(-1.0f, __fmul_rn(float(b), bs)), __fmul_rn(bs, relax));
}
__device__ __forceinline__ float vox_hi(int b, float bs, float relax) {
  return __fadd_rn(__fadd_rn(-1.0f, __fmul_rn(float(b + 1), bs)), __fmul_rn(bs, relax));
}

// Blocks [lo, hi] along one axis whose grown bounds hold m.
__device__ __forceinline__ void vox_span(float m, const VoxelArgs& a, int& lo, int& hi) {
  const int r = int(ceilf(a.relax)) + 1;
  const int b0 = vox_block(m, a.bs);
  lo = 1;
  hi = 0;
  for (int b = max(b0 - r, 0); b <= min(b0 + r, a.B); ++b) {
    if (!(m < vox_lo(b, a.bs, a.relax) || m > vox_hi(b, a.bs, a.relax))) {
      if (lo > hi) lo = b;
      hi = b;
    }
  }
}

// Per Gaussian: the inverse covariance (cofactors over the regularised
// determinant), its record, and the number of blocks it is binned into.
__global__ void __launch_bounds__(kVoxThreads) voxel_prepare_kernel(VoxelArgs a) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.P) return;
  const float mx = a.means[3 * g], my = a.means[3 * g + 1], mz = a.means[3 * g + 2];
  const float c0 = a.covs[6 * g], c1 = a.covs[6 * g + 1], c2 = a.covs[6 * g + 2];
  const float c3 = a.covs[6 * g + 3], c4 = a.covs[6 * g + 4], c5 = a.covs[6 * g + 5];
  // Sigma = [[c0 c1 c2] [c1 c3 c4] [c2 c4 c5]]
  const float det = c0 * c3 * c5 + 2 * c4 * c2 * c1 - c4 * c4 * c0 - c2 * c2 * c3 - c1 * c1 * c5;
  const float idet = 1.0f / (det + 1e-24f);
  float4* rec = a.rec + 3 * size_t(g);
  rec[0] = make_float4(mx, my, mz, a.opacities[g]);
  rec[1] = make_float4((c3 * c5 - c4 * c4) * idet, (c4 * c2 - c1 * c5) * idet, (c4 * c1 - c2 * c3) * idet,
                       (c0 * c5 - c2 * c2) * idet);
  rec[2] = make_float4((c1 * c2 - c4 * c0) * idet, (c0 * c3 - c1 * c1) * idet, 0.f, 0.f);
  int xl, xh, yl, yh, zl, zh;
  vox_span(mx, a, xl, xh);
  vox_span(my, a, yl, yh);
  vox_span(mz, a, zl, zh);
  a.count[g] = uint32_t(max(xh - xl + 1, 0) * max(yh - yl + 1, 0) * max(zh - zl + 1, 0));
}

// Per Gaussian: its (block, Gaussian) pairs at its scanned offset, blocks in
// x-fastest order.
__global__ void __launch_bounds__(kVoxThreads) voxel_emit_kernel(VoxelArgs a) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.P || a.count[g] == 0) return;
  int xl, xh, yl, yh, zl, zh;
  vox_span(a.means[3 * g], a, xl, xh);
  vox_span(a.means[3 * g + 1], a, yl, yh);
  vox_span(a.means[3 * g + 2], a, zl, zh);
  uint32_t o = a.offsets[g];
  const int nb = a.B + 1;
  for (int z = zl; z <= zh; ++z)
    for (int y = yl; y <= yh; ++y)
      for (int x = xl; x <= xh; ++x) {
        a.keys[o] = uint32_t(x + nb * (y + nb * z));
        a.vals[o] = uint32_t(g);
        ++o;
      }
}

// One thread per voxel, x fastest within a CTA of 8 x 8 x 4 voxels, so a
// warp's voxels share a block and its list entries are broadcast loads.
__global__ void __launch_bounds__(kVoxThreads) voxel_field_kernel(VoxelArgs a, const uint32_t* __restrict__ list,
                                                                    const uint2* __restrict__ ranges) {
  const int i = blockIdx.x * 8 + (threadIdx.x & 7);
  const int j = blockIdx.y * 8 + ((threadIdx.x >> 3) & 7);
  const int k = blockIdx.z * 4 + (threadIdx.x >> 6);
  const int R = a.R;
  if (i >= R || j >= R || k >= R) return;
  const float x = vox_coord(i, R), y = vox_coord(j, R), z = vox_coord(k, R);
  const int nb = a.B + 1;
  // voxel coordinates lie in [-1, 1], so their blocks lie in [0, B]; the
  // clamp only guards the ranges array
  const int blk = vox_block_clamped(x, a.bs, a.B) +
                  nb * (vox_block_clamped(y, a.bs, a.B) + nb * vox_block_clamped(z, a.bs, a.B));
  const uint2 r = ranges[blk];
  float val = 0.0f;
  for (uint32_t e = r.x; e < r.y; ++e) {
    const float4* rec = a.rec + 3 * size_t(__ldg(list + e));
    const float4 q0 = __ldg(rec), q1 = __ldg(rec + 1), q2 = __ldg(rec + 2);
    const float dx = x - q0.x, dy = y - q0.y, dz = z - q0.z;
    float power = -0.5f * (dx * dx * q1.x + dy * dy * q1.w + dz * dz * q2.y) - dx * dy * q1.y - dx * dz * q1.z -
                  dy * dz * q2.x;
    if (power > 0) power = -1e10f;
    val += q0.w * expf(power);
  }
  a.occ[size_t(i) + size_t(R) * (size_t(j) + size_t(R) * size_t(k))] = val;
}

}  // namespace

void launch_voxel_prepare(const VoxelArgs& a, cudaStream_t stream) {
  if (a.P <= 0) return;
  stage_begin(kStOther, stream);
  voxel_prepare_kernel<<<(a.P + kVoxThreads - 1) / kVoxThreads, kVoxThreads, 0, stream>>>(a);
  stage_end(kStOther, stream, 1);
}

void launch_voxel_emit(const VoxelArgs& a, cudaStream_t stream) {
  if (a.P <= 0) return;
  stage_begin(kStOther, stream);
  voxel_emit_kernel<<<(a.P + kVoxThreads - 1) / kVoxThreads, kVoxThreads, 0, stream>>>(a);
  stage_end(kStOther, stream, 1);
}

void launch_voxel_field(const VoxelArgs& a, const uint32_t* list, const uint2* ranges, cudaStream_t stream) {
  const dim3 grid((a.R + 7) / 8, (a.R + 7) / 8, (a.R + 3) / 4);
  stage_begin(kStOther, stream);
  voxel_field_kernel<<<grid, kVoxThreads, 0, stream>>>(a, list, ranges);
  stage_end(kStOther, stream, 1);
}

}  // namespace w2w
