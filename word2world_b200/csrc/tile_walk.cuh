// Shared machinery of the per-tile pixel loops (forward blend, both backward
// pixel passes).
//
// A CTA of 256 threads owns one 16x16 tile; warp w owns the 8x4 pixel block
// w (columns 8*(w & 1) .. +7, rows 4*(w >> 1) .. +3), lane l its pixel
// (l & 7, l >> 3) inside the block.
//
// Independent warps (backward passes): each warp walks the tile's list on its
// own, down from its pixels' largest contributor count, kChunk entries at a
// time: lane j gathers entry j's 64-byte record by
// Gaussian id (the tile's warps gather the same records, so after the first
// they come from L1), tests whether the Gaussian can reach the warp's block
// with alpha >= 1/255 (block_test in common.cuh) and stores the record's first
// 48 bytes to the warp's shared-memory slot; the ballot of the tests is the
// list of entries the warp evaluates, in list order.  The next chunk's records
// are gathered while the current one is walked.  Warps never wait for one
// another: a warp whose block has little to do, or whose pixels have all
// terminated, finishes early instead of idling at a per-batch barrier.
#pragma once

#include "common.cuh"

namespace w2w {

constexpr int kRecVec = 3;  // float4s of a record staged in shared memory
constexpr int kChunk = 32;  // list entries staged per warp step (one per lane)

struct WarpChunk {
  float4 rec[kChunk * kRecVec];
  uint32_t id[kChunk];
};

// Pixel of this thread in tile `tile` of a grid `gw` tiles wide.
struct TilePixel {
  int X0, Y0, px, py, warp, lane, bx, by;  // (bx, by): top-left pixel of the warp's block
  // warp: this thread's 8x4 block of the tile (0..7)
  __device__ __forceinline__ TilePixel(int tile, int gw, int block) {
    warp = block;
    lane = threadIdx.x & 31;
    X0 = (tile % gw) * kTile;
    Y0 = (tile / gw) * kTile;
    bx = X0 + kBlockW * (warp & 1);
    by = Y0 + kBlockH * (warp >> 1);
    px = bx + (lane & 7);
    py = by + (lane >> 3);
  }
  __device__ __forceinline__ TilePixel(int tile, int gw) : TilePixel(tile, gw, int(threadIdx.x >> 5)) {}
};

// Tiles are processed heaviest first: CTA b takes tile order[b], where order
// lists the tiles by decreasing weight (tile_order_kernel: the list length
// from `ranges`, or `counts` when given), so the heaviest start in the first
// wave instead of wherever the raster order puts them.
// `zero`, when given, is cleared over num_tiles entries on the way (the
// blend's per-tile maximum, which its CTAs then combine), and `counter`, when
// given, set to zero (the persistent blend's queue).
__global__ void tile_order_kernel(const uint2* ranges, const uint32_t* counts, int num_tiles, uint32_t* order,
                                  uint32_t* zero, uint32_t* counter);

// One entry's record held in registers between its gather and its store.
struct ChunkLoad {
  float4 r0, r1, r2, r3;
  uint32_t id;
  bool has;
  bool masked;  // `has` already means "may reach the warp's block" (from the blend's block masks)
};

// Block masks the forward blend leaves for the backward passes: per list
// position, 4 bits for the tile's upper four 8x4 blocks (array `top`) and 4
// for its lower four (`bottom`), bit b set when the entry may reach block b
// (block_mask).  `valid` points at the binning header's flag; a state the
// blend did not write (a replayed list) has it clear, and the walk tests
// every entry itself.
struct BlockMasks {
  const uint8_t* top;
  const uint8_t* bottom;
  const uint32_t* valid;
};

// Gather entry `pos` of the point list (when `has`).  Records are four float4s;
// r2.w and r3 hold the culling parameters (hy; beta, gamma, eps, vr).  An id
// of num_records or more (a list left inconsistent by a sort whose bounded
// wait ran out, which its error word reports) is skipped, never read.  With
// `mask` (the warp's mask array, or null) only entries whose bit `bit` is set
// are gathered.
__device__ __forceinline__ void chunk_load(ChunkLoad& st, const float* record, const uint32_t* point_list, size_t pos,
                                           bool has, uint32_t num_records, const uint8_t* mask = nullptr,
                                           int bit = 0) {
  st.has = false;
  st.masked = mask != nullptr;
  if (has && mask != nullptr) has = (mask[pos] >> bit) & 1u;
  if (has) {
    st.id = point_list[pos];
    st.has = st.id < num_records;
  }
  if (st.has) {
    const float4* rec = reinterpret_cast<const float4*>(record);
    const float4* r = rec + 4 * size_t(st.id);
    st.r0 = __ldg(r);
    st.r1 = __ldg(r + 1);
    st.r2 = __ldg(r + 2);
    st.r3 = __ldg(r + 3);
  }
}

// Store lane j's gathered entry in slot j and return the ballot of "may reach
// the block at (bx, by)".  Warp-collective; the caller has synchronised the
// warp after its last read of the previous chunk.
__device__ __forceinline__ uint32_t chunk_store(WarpChunk& c, const ChunkLoad& st, int bx, int by) {
  const int lane = threadIdx.x & 31;
  bool reach = false;
  if (st.has) {
    float4* s = &c.rec[kRecVec * lane];
    s[0] = st.r0;
    s[1] = st.r1;
    s[2] = st.r2;
    c.id[lane] = st.id;
    reach = st.masked || block_test(st.r0.x, st.r0.y, st.r2.w, st.r3.x, st.r3.y, st.r3.z, st.r3.w, bx, by);
  }
  __syncwarp();
  return __ballot_sync(0xffffffffu, reach);
}

// Next set bit of `bits` (cleared), or -1.
__device__ __forceinline__ int pop_entry(uint32_t& bits) {
  if (bits == 0u) return -1;
  const int j = __ffs(bits) - 1;
  bits &= bits - 1u;
  return j;
}

// ---------------------------------------------------------------------------
// Cooperative batches (forward blend): the CTA stages kBatch entries at a time
// (kBatch / blockDim.x per thread), double-buffered, with the block bits of the
// CTA's kW warps computed once per entry (block_mask); each warp expands its
// bits into an entry list (build_list).  The blend walks far past most
// contributors (until every pixel terminates), so sharing each entry's gather
// and test among warps matters more there than letting warps run apart.
// kW = 8: one CTA per tile; kW = 4: two CTAs per tile (its upper and lower
// eight rows), each staging the whole list, so that fewer warps wait at each
// batch's barrier for the slowest of them.
// The next batch is gathered while the current one is walked, in one of two
// ways (the blend's "blend_stage" tuning knob): into registers, stored to
// shared memory after the walk (stage_load / stage_store; kVec = kRecVec), or
// copied straight into shared memory with cp.async (stage_copy / stage_mask;
// kVec = kStageVec), which holds no registers through the walk.
// ---------------------------------------------------------------------------
constexpr int kStageVec = 4;  // float4s per record copied by cp.async (the whole record: the test reads r2.w, r3)

template <int kW, int kVec>
struct TileWalkShared {
  float4 rec[2][kBatch * kVec];
  uint32_t bal[2][kW][kBatch / 32];  // [buffer][warp's block][32-entry chunk]
  uint8_t list[kW][kBatch];          // per warp: its entries of the current batch, in order
};

// Expand this warp's flag words into its entry list (in order); returns the
// count.  Warp-collective.
template <int kW, int kVec>
__device__ __forceinline__ int build_list(TileWalkShared<kW, kVec>& sm, int buf, int warp, int lane, int start = 0) {
  __syncwarp();  // the previous walk's reads of the list are done
  int count = 0;
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int c = 0; c < kBatch / 32; ++c) {
    uint32_t bits = sm.bal[buf][warp][c];
    const int lo = start - 32 * c;  // entries below `start` are dropped
    if (lo > 0) bits = lo >= 32 ? 0u : bits & (0xffffffffu << lo);
    if ((bits >> lane) & 1u) sm.list[warp][count + __popc(bits & lt)] = uint8_t(32 * c + lane);
    count += __popc(bits);
  }
  __syncwarp();
  return count;
}

// Block bits of one entry for the CTA's kW blocks (the tile's blocks
// first_block .. first_block + kW - 1), published as the CTA's ballot words of
// slot j; the masks also go to global memory for the backward passes
// (BlockMasks): bits 0-3 to lo_dst[j], bits 4-7 (eight-warp CTAs) to
// hi_dst[j], where the callers offset the arrays to the batch's first list
// position.  Every thread of a warp must call this for the same chunk (the
// ballots are full-warp).
template <int kW, int kVec>
__device__ __forceinline__ void publish_mask(TileWalkShared<kW, kVec>& sm, int buf, bool has, float mx, float my,
                                             float hy, float4 c, int j, int X0, int Y0, int first_block,
                                             uint8_t* lo_dst, uint8_t* hi_dst) {
  const int lane = j & 31, chunk = j >> 5;
  uint32_t mask = 0;
  if (has) {
    // the CTA's blocks are kW / 2 rows of two, starting at row group first_block / 2
    mask = block_mask<kW / 2>(mx, my, hy, c.x, c.y, c.z, c.w, X0, Y0 + kBlockH * (first_block / 2));
    if (lo_dst != nullptr) lo_dst[j] = uint8_t(mask & 15u);
    if (hi_dst != nullptr) hi_dst[j] = uint8_t(mask >> 4);
  }
  uint32_t mine = 0;
#pragma unroll
  for (int b = 0; b < kW; ++b) {
    const uint32_t w = __ballot_sync(0xffffffffu, (mask >> b) & 1u);
    if (lane == b) mine = w;
  }
  if (lane < kW) sm.bal[buf][lane][chunk] = mine;
}

// One entry's record held in registers between its gather and its store.
struct Staged {
  float4 r0, r1, r2, r3;
  bool has;
};

// Gather entry `pos` of the point list (when `has`) into registers.  Records
// are four float4s; r2.w and r3 hold the culling parameters (hy; beta, gamma,
// eps, vr).  Ids of num_records or more are skipped (see chunk_load).
__device__ __forceinline__ void stage_load(Staged& st, const float* record, const uint32_t* point_list, size_t pos,
                                           bool has, uint32_t num_records) {
  st.has = false;
  uint32_t id = 0;
  if (has) {
    id = point_list[pos];
    st.has = id < num_records;
  }
  if (st.has) {
    const float4* r = reinterpret_cast<const float4*>(record) + 4 * size_t(id);
    st.r0 = __ldg(r);
    st.r1 = __ldg(r + 1);
    st.r2 = __ldg(r + 2);
    st.r3 = __ldg(r + 3);
  }
}

// Store the gathered entry j (slot j of the batch) into buffer `buf` and
// publish its block masks (publish_mask).
template <int kW>
__device__ __forceinline__ void stage_store(TileWalkShared<kW, kRecVec>& sm, int buf, const Staged& st, int j, int X0,
                                            int Y0, int first_block, uint8_t* lo_dst, uint8_t* hi_dst) {
  if (st.has) {
    float4* s = &sm.rec[buf][kRecVec * j];
    s[0] = st.r0;
    s[1] = st.r1;
    s[2] = st.r2;
  }
  publish_mask(sm, buf, st.has, st.r0.x, st.r0.y, st.r2.w, st.r3, j, X0, Y0, first_block, lo_dst, hi_dst);
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// This thread's copies have landed (and are visible to it).
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Start the copy of entry `pos` of the point list (when `has`) into slot
// `dst` (kStageVec float4s); returns whether the slot will hold a record.
// Ids of num_records or more are skipped.  The caller commits the group.
__device__ __forceinline__ bool stage_copy(float4* dst, const float* record, const uint32_t* point_list, size_t pos,
                                           bool has, uint32_t num_records) {
  if (!has) return false;
  const uint32_t id = point_list[pos];
  if (id >= num_records) return false;
  const float4* r = reinterpret_cast<const float4*>(record) + 4 * size_t(id);
#pragma unroll
  for (int u = 0; u < kStageVec; ++u) cp_async16(dst + u, r + u);
  return true;
}

// Publish the block masks of copied entry j (slot j of buffer `buf`, copied
// by this thread, whose copies have landed).
template <int kW>
__device__ __forceinline__ void stage_mask(TileWalkShared<kW, kStageVec>& sm, int buf, bool has, int j, int X0,
                                           int Y0, int first_block, uint8_t* lo_dst, uint8_t* hi_dst) {
  float2 m = make_float2(0.f, 0.f);
  float hy = 0.f;
  float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
  if (has) {
    const float4* s = &sm.rec[buf][kStageVec * j];
    m = *reinterpret_cast<const float2*>(s);
    hy = s[2].w;
    c = s[3];
  }
  publish_mask(sm, buf, has, m.x, m.y, hy, c, j, X0, Y0, first_block, lo_dst, hi_dst);
}

}  // namespace w2w
