// Shared machinery of the per-tile pixel loops (forward blend, both backward
// pixel passes).
//
// A CTA of 256 threads owns one 16x16 tile; warp w owns the 8x4 pixel block
// w (columns 8*(w & 1) .. +7, rows 4*(w >> 1) .. +3), lane l its pixel
// (l & 7, l >> 3) inside the block.  The tile's list is staged kBatch entries
// at a time, double-buffered: each thread gathers one entry's 64-byte record
// by Gaussian id into registers while the warps walk the previous batch, then
// stores the record's first 48 bytes to shared memory and computes the
// entry's 8-bit block mask (block_mask in common.cuh).  One ballot per block
// bit turns the masks into, per block, eight 32-bit words of "this entry can
// reach my block" flags; each warp expands its own words into a list of entry
// indices (build_list) and walks only those, in list order.
#pragma once

#include "common.cuh"

namespace w2w {

constexpr int kRecVec = 3;  // float4s of a record staged in shared memory

struct TileWalkShared {
  float4 rec[2][kBatch * kRecVec];
  uint32_t id[2][kBatch];
  uint32_t bal[2][8][8];  // [buffer][block][32-entry chunk]
  uint8_t list[8][kBatch];  // per warp: its entries of the current batch, in order
};

// Expand this warp's eight flag words into its entry list (in order); returns
// the count.  Warp-collective.
__device__ __forceinline__ int build_list(TileWalkShared& sm, int buf, int warp, int lane, int start = 0) {
  __syncwarp();  // the previous walk's reads of the list are done
  int count = 0;
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    uint32_t bits = sm.bal[buf][warp][c];
    const int lo = start - 32 * c;  // entries below `start` are dropped
    if (lo > 0) bits = lo >= 32 ? 0u : bits & (0xffffffffu << lo);
    if ((bits >> lane) & 1u) sm.list[warp][count + __popc(bits & lt)] = uint8_t(32 * c + lane);
    count += __popc(bits);
  }
  __syncwarp();
  return count;
}

// Pixel of this thread in tile `tile` of a grid `gw` tiles wide.
struct TilePixel {
  int X0, Y0, px, py, warp, lane;
  __device__ __forceinline__ TilePixel(int tile, int gw) {
    warp = threadIdx.x >> 5;
    lane = threadIdx.x & 31;
    X0 = (tile % gw) * kTile;
    Y0 = (tile / gw) * kTile;
    px = X0 + kBlockW * (warp & 1) + (lane & 7);
    py = Y0 + kBlockH * (warp >> 1) + (lane >> 3);
  }
};

// Tiles are processed heaviest first: CTA b takes tile order[b], where order
// lists the tiles by decreasing list length (tile_order_kernel), so the
// longest lists start in the first wave instead of wherever the raster order
// puts them.
__global__ void tile_order_kernel(const uint2* ranges, int num_tiles, uint32_t* order);

// One entry's record held in registers between its gather and its store.
struct Staged {
  float4 r0, r1, r2, r3;
  uint32_t id;
  bool has;
};

// Gather entry `pos` of the point list (when `has`).  Records are four float4s;
// r2.w and r3 hold the culling parameters (hy; beta, gamma, eps, vr).
__device__ __forceinline__ void stage_load(Staged& st, const float* record, const uint32_t* point_list, size_t pos,
                                           bool has) {
  st.has = has;
  if (has) {
    const float4* rec = reinterpret_cast<const float4*>(record);
    st.id = point_list[pos];
    const float4* r = rec + 4 * size_t(st.id);
    st.r0 = __ldg(r);
    st.r1 = __ldg(r + 1);
    st.r2 = __ldg(r + 2);
    st.r3 = __ldg(r + 3);
  }
}

// Store the staged entry of thread j into buffer `buf` and publish the block
// masks.  Every thread of the CTA must call this (the ballots are full-warp).
__device__ __forceinline__ void stage_store(TileWalkShared& sm, int buf, const Staged& st, int X0, int Y0) {
  const int j = threadIdx.x, lane = j & 31, chunk = j >> 5;
  uint32_t mask = 0;
  if (st.has) {
    float4* s = &sm.rec[buf][kRecVec * j];
    s[0] = st.r0;
    s[1] = st.r1;
    s[2] = st.r2;
    sm.id[buf][j] = st.id;
    mask = block_mask(st.r0.x, st.r0.y, st.r2.w, st.r3.x, st.r3.y, st.r3.z, st.r3.w, X0, Y0);
  }
  uint32_t mine = 0;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const uint32_t w = __ballot_sync(0xffffffffu, (mask >> b) & 1u);
    if (lane == b) mine = w;
  }
  if (lane < 8) sm.bal[buf][lane][chunk] = mine;
}

}  // namespace w2w
