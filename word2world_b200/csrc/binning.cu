// Instance binning from depth-ordered Gaussians: the sorted (tile, depth) list
// of a view built with one R-sized write instead of key emission followed by
// a multi-pass radix sort (reference prepareSort.cu:178-435: key emission and
// the stable 64-bit LSD sort; gaussianTiles.cu:6-33: tile ranges).
//
// The reference's order is (tile, depth bits, slot), and a Gaussian's slots
// all precede the slots of every later Gaussian (each Gaussian owns one
// contiguous run of slots, the lowest index winning where emission
// rectangles overlap), so within a tile equal depths keep Gaussian order.
// Hence: sort the P Gaussians stably by their depth bits (a small sort over
// P keys, run after the projection pass), walk the owned instances of the
// Gaussians in that order -- each Gaussian's owned entries in row-major order
// of its emission rectangle, as the reference emits them -- and place every
// instance stably by tile.  Within a tile the instances then appear by
// depth bits, ties in Gaussian order: exactly the reference's sorted list.
//
// The placement is a three-kernel counting sort over the instance sequence
// (position p = place in the depth-ordered walk):
//   count   -- one CTA per chunk of kBinChunk positions: per-tile counts of
//              the chunk (shared-memory atomics), one row of a chunk x tile
//              matrix, and the per-tile totals;
//   offsets -- per tile: its start (exclusive sum of the totals, the tile
//              ranges) plus the exclusive sum down the chunk column, written
//              back over the matrix;
//   scatter -- the chunk again, each warp its contiguous share: per-warp tile
//              counts, their exclusive sums over the chunk's warps, then the
//              walk in order, ranking equal tiles within 32 positions with a
//              match; every instance's Gaussian id and its packed key go to
//              their final place.
// Positions are generated, never stored: each warp expands 32 Gaussians at a
// time (a shuffle binary search finds each lane's owner), so the sequence is
// read as P-sized data twice instead of R-sized keys once per sort pass.
#include <type_traits>

#include "common.cuh"
#include "kernels.h"

namespace w2w {
namespace {

constexpr int kBinThreads = 256;
constexpr int kBinWarps = kBinThreads / 32;
constexpr uint32_t kWarpShare = kBinShare;  // positions per warp of a chunk
static_assert(kBinChunk == kBinShare * kBinWarps && kBinShare % 32 == 0, "whole steps per warp");

// Owned instance range of Gaussian g: slots [p0, p1) of the view's slot array,
// the suffix (from emission index p0 - start) of its row-major emission
// rectangle; 0 when it owns none.  Mirrors the key emission of duplicate.cu.
struct Owned {
  uint32_t count, first_k, x0, y0, w;
};
__device__ __forceinline__ Owned owned_of(const BinArgs& a, uint32_t g) {
  Owned o{0u, 0u, 0u, 0u, 1u};
  const uint32_t start = a.offsets[g] - a.tiles[g];
  const uint2 rc = reinterpret_cast<const uint2*>(a.rect)[g];
  const uint32_t x0 = rc.x & 0xffffu, y0 = rc.x >> 16, x1 = rc.y & 0xffffu, y1 = rc.y >> 16;
  const uint32_t n = (x1 > x0 && y1 > y0) ? (x1 - x0) * (y1 - y0) : 0u;
  const uint32_t p0 = max(start, a.prev_reach[g]);
  const uint32_t p1 = min(start + n, a.R);
  if (p1 > p0) {
    o.count = p1 - p0;
    o.first_k = p0 - start;
    o.x0 = x0;
    o.y0 = y0;
    o.w = x1 - x0;
  }
  return o;
}

// Depth-order owned counts (gathered through the sort's permutation), the
// input of the prefix scan.  A permutation entry of P or more (left by a depth
// sort whose bounded wait ran out, which its error word reports) owns nothing
// and is never used as an index.
__global__ void owned_count_kernel(BinArgs a, uint32_t* __restrict__ count) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= uint32_t(a.P)) return;
  const uint32_t g = a.order[j];
  count[j] = g < uint32_t(a.P) ? owned_of(a, g).count : 0u;
}

// Depth-order index whose position range holds each warp share's first
// position (positions s * kWarpShare for s = 0 .. shares - 1).
__global__ void warp_starts_kernel(BinArgs a, uint32_t shares) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= uint32_t(a.P)) return;
  const uint32_t lo = a.dprefix[j], hi = a.dprefix[j + 1];
  if (hi <= lo) return;
  for (uint32_t s = (lo + kWarpShare - 1) / kWarpShare; s < shares && s * kWarpShare < hi; ++s) a.warp_start[s] = j;
}

// Walk positions [pa, pb) in order, 32 per step: f(valid, p, g, tile, dlow)
// per lane (lanes of a step hold consecutive positions).  j: depth-order index
// holding pa.  Warp-collective.
template <typename F>
__device__ __forceinline__ void walk_positions(const BinArgs& a, uint32_t pa, uint32_t pb, uint32_t j, F&& f) {
  const int lane = threadIdx.x & 31;
  uint32_t pos = pa;
  // every position below R has an owner (each slot is owned by exactly one
  // Gaussian); the bound on j only guards against an inconsistent prefix
  while (pos < pb && j < uint32_t(a.P)) {
    const uint32_t jj = j + uint32_t(lane);
    uint32_t cnt = 0, k0 = 0, xy = 0, w = 1, dlow = 0, g = 0;
    float inv_w = 1.0f;
    if (jj < uint32_t(a.P)) {
      const uint32_t lo = max(a.dprefix[jj], pos), hi = min(a.dprefix[jj + 1], pb);
      g = a.order[jj];
      if (hi > lo && g < uint32_t(a.P)) {  // (an out-of-range entry: see owned_count_kernel)
        const Owned o = owned_of(a, g);
        cnt = hi - lo;
        k0 = o.first_k + (lo - a.dprefix[jj]);
        xy = o.x0 | (o.y0 << 16);
        w = o.w;
        inv_w = __frcp_rn(float(w));
        const uint32_t db = __float_as_uint(a.depth[g]);
        dlow = a.depth_bits >= 32 ? db : (db & ((1u << a.depth_bits) - 1u));
      }
    }
    uint32_t incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t excl = incl - cnt;
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t e = base + uint32_t(lane);
      int o = 0;  // owner lane: lanes whose inclusive count is <= e
#pragma unroll
      for (int b = 16; b > 0; b >>= 1) {
        const uint32_t t = __shfl_sync(0xffffffffu, incl, o + b - 1);
        if (t <= e) o += b;
      }
      o = min(o, 31);
      const uint32_t oex = __shfl_sync(0xffffffffu, excl, o);
      const uint32_t ok0 = __shfl_sync(0xffffffffu, k0, o);
      const uint32_t oxy = __shfl_sync(0xffffffffu, xy, o);
      const uint32_t ow = __shfl_sync(0xffffffffu, w, o);
      const float oinv = __shfl_sync(0xffffffffu, inv_w, o);
      const uint32_t odl = __shfl_sync(0xffffffffu, dlow, o);
      const uint32_t og = __shfl_sync(0xffffffffu, g, o);
      const bool valid = e < total;
      const uint32_t k = ok0 + (e - oex);
      // k / ow without an integer division: k < 2^24 is exact in float, the
      // product's rounding moves the quotient by at most one, and the
      // remainder test corrects it
      uint32_t q = __float2uint_rz(__uint2float_rn(k) * oinv);
      int r = int(k) - int(q * ow);
      if (r < 0) {
        --q;
        r += int(ow);
      } else if (r >= int(ow)) {
        ++q;
        r -= int(ow);
      }
      const uint32_t ty = (oxy >> 16) + q, tx = (oxy & 0xffffu) + uint32_t(r);
      f(valid, pos + e, og, ty * uint32_t(a.gw) + tx, odl);
    }
    pos += total;
    j += 32;
  }
}

__device__ __forceinline__ void chunk_share(const BinArgs& a, int warp, uint32_t& pa, uint32_t& pb, uint32_t& j) {
  const uint32_t c0 = blockIdx.x * uint32_t(kBinChunk);
  pa = c0 + uint32_t(warp) * kWarpShare;
  pb = min(pa + uint32_t(kWarpShare), a.R);
  j = pa < a.R ? a.warp_start[pa / kWarpShare] : 0u;
}

__global__ void __launch_bounds__(kBinThreads) bin_count_kernel(BinArgs a) {
  extern __shared__ uint32_t s_cnt[];  // [T]
  const int T = a.T;
  for (int t = threadIdx.x; t < T; t += kBinThreads) s_cnt[t] = 0u;
  __syncthreads();
  uint32_t pa, pb, j;
  chunk_share(a, int(threadIdx.x >> 5), pa, pb, j);
  walk_positions(a, pa, pb, j, [&](bool valid, uint32_t, uint32_t, uint32_t tile, uint32_t) {
    if (valid && tile < uint32_t(T)) atomicAdd(&s_cnt[tile], 1u);
  });
  __syncthreads();
  uint32_t* row = a.counts + size_t(blockIdx.x) * size_t(T);
  for (int t = threadIdx.x; t < T; t += kBinThreads) {
    const uint32_t v = s_cnt[t];
    row[t] = v;
    if (v) atomicAdd(&a.tile_total[t], v);
  }
}

// One CTA of 32 x 32 threads per 32 tiles: thread (ty, tx) handles tile
// t0 + tx over the ty-th of 32 contiguous segments of the chunks.
__global__ void __launch_bounds__(1024) bin_offsets_kernel(BinArgs a, int chunks) {
  __shared__ uint32_t s_seg[32][33];
  __shared__ uint32_t s_red[32];
  __shared__ uint32_t s_start[32];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int T = a.T;
  const int t0 = blockIdx.x * 32, t = t0 + tx;
  // the block's first position: the totals of every tile before t0
  uint32_t before = 0;
  for (int u = threadIdx.x; u < t0; u += 1024) before += a.tile_total[u];
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) before += __shfl_xor_sync(0xffffffffu, before, d);
  if (tx == 0) s_red[ty] = before;
  const int seg = (chunks + 31) / 32;
  const int r0 = ty * seg, r1 = min(chunks, r0 + seg);
  uint32_t sum = 0;
  if (t < T)
    for (int r = r0; r < r1; ++r) sum += a.counts[size_t(r) * T + t];
  s_seg[ty][tx] = sum;
  __syncthreads();
  if (ty == 0) {
    uint32_t base = 0;
#pragma unroll
    for (int w = 0; w < 32; ++w) base += s_red[w];
    const uint32_t tot = t < T ? a.tile_total[t] : 0u;
    uint32_t incl = tot;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
      if (tx >= d) incl += o;
    }
    const uint32_t start = base + incl - tot;
    s_start[tx] = start;
    // empty tiles get (0, 0), as the reference's zeroed range buffer leaves them
    if (t < T) a.ranges[t] = tot ? make_uint2(start, start + tot) : make_uint2(0u, 0u);
  }
  __syncthreads();
  if (t >= T) return;
  uint32_t run = s_start[tx];
  for (int w = 0; w < ty; ++w) run += s_seg[w][tx];
  for (int r = r0; r < r1; ++r) {
    uint32_t* cell = a.counts + size_t(r) * T + t;
    const uint32_t v = *cell;
    *cell = run;
    run += v;
  }
}

// Shared memory of the scatter kernel: per-warp tile counters [kBinWarps][T],
// the global index of each tile's chunk-local slot 0 [T], then the chunk's
// keys and ids reordered by tile [kBinChunk].
template <typename Key>
struct ScatterSmem {
  size_t wcnt, gofs, keys, vals, total;
  __host__ __device__ explicit ScatterSmem(int T) {
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = (o + 15) & ~size_t(15); o = at + bytes; return at; };
    wcnt = take(size_t(kBinWarps) * size_t(T) * 4);
    gofs = take(size_t(T) * 4);
    keys = take(size_t(kBinChunk) * sizeof(Key));
    vals = take(size_t(kBinChunk) * 4);
    total = (o + 15) & ~size_t(15);
  }
};

// The chunk's instances, placed stably by tile: (1) walk counting per warp
// and tile; (2) each tile's chunk-local slots (tiles in order, warps in order
// within a tile) and the global index of its slot 0; (3) walk again, ranking
// equal tiles within 32 positions, and put each instance's key and id in its
// chunk-local slot; (4) write the chunk out slot by slot, so that each
// tile's run is stored by consecutive threads.
template <bool kKey64>
__global__ void __launch_bounds__(kBinThreads) bin_scatter_kernel(BinArgs a) {
  using Key = typename std::conditional<kKey64, uint64_t, uint32_t>::type;
  extern __shared__ __align__(16) unsigned char s_raw[];
  const int T = a.T;
  const ScatterSmem<Key> L(T);
  uint32_t* s_wcnt = reinterpret_cast<uint32_t*>(s_raw + L.wcnt);
  uint32_t* s_gofs = reinterpret_cast<uint32_t*>(s_raw + L.gofs);
  Key* s_key = reinterpret_cast<Key*>(s_raw + L.keys);
  uint32_t* s_val = reinterpret_cast<uint32_t*>(s_raw + L.vals);
  __shared__ uint32_t s_part[kBinThreads];
  const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
  for (int i = threadIdx.x; i < kBinWarps * T; i += kBinThreads) s_wcnt[i] = 0u;
  __syncthreads();
  uint32_t pa, pb, j;
  chunk_share(a, warp, pa, pb, j);
  uint32_t* mine = s_wcnt + warp * T;
  walk_positions(a, pa, pb, j, [&](bool valid, uint32_t, uint32_t, uint32_t tile, uint32_t) {
    if (valid && tile < uint32_t(T)) atomicAdd(&mine[tile], 1u);
  });
  __syncthreads();
  // (2) each thread a contiguous run of tiles: per-warp exclusive counts
  // within each tile, the run's total, then a block scan of the runs
  const int per = (T + kBinThreads - 1) / kBinThreads;
  const int t0 = int(threadIdx.x) * per, t1 = min(T, t0 + per);
  uint32_t run_total = 0;
  for (int t = t0; t < t1; ++t) {
    uint32_t r = 0;
#pragma unroll
    for (int w = 0; w < kBinWarps; ++w) {
      const uint32_t x = s_wcnt[w * T + t];
      s_wcnt[w * T + t] = r;
      r += x;
    }
    s_gofs[t] = r;  // the tile's count in this chunk, for now
    run_total += r;
  }
  s_part[threadIdx.x] = run_total;
  __syncthreads();
  if (warp == 0) {  // exclusive scan of the 256 run totals, 8 per lane
    uint32_t v[kBinThreads / 32], sum = 0;
#pragma unroll
    for (int i = 0; i < kBinThreads / 32; ++i) {
      v[i] = s_part[lane * (kBinThreads / 32) + i];
      sum += v[i];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    uint32_t ex = incl - sum;
#pragma unroll
    for (int i = 0; i < kBinThreads / 32; ++i) {
      s_part[lane * (kBinThreads / 32) + i] = ex;
      ex += v[i];
    }
  }
  __syncthreads();
  const uint32_t* base = a.counts + size_t(blockIdx.x) * size_t(T);
  uint32_t local = s_part[threadIdx.x];
  for (int t = t0; t < t1; ++t) {
    const uint32_t cnt = s_gofs[t];
#pragma unroll
    for (int w = 0; w < kBinWarps; ++w) s_wcnt[w * T + t] += local;
    s_gofs[t] = base[t] - local;  // global index of chunk-local slot 0 of tile t (mod 2^32)
    local += cnt;
  }
  __syncthreads();
  // (3) rank and place in shared memory
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t db = a.depth_bits;
  walk_positions(a, pa, pb, j, [&](bool valid, uint32_t, uint32_t g, uint32_t tile, uint32_t dlow) {
    const bool ok = valid && tile < uint32_t(T);
    const uint32_t key = ok ? tile : 0xffffffffu;
    const uint32_t peers = __match_any_sync(0xffffffffu, key);
    uint32_t before = 0;
    if (ok) before = mine[tile];
    __syncwarp();
    if (ok) {
      const uint32_t slot = before + __popc(peers & lt);
      if (lane == __ffs(peers) - 1) mine[tile] = before + __popc(peers);
      if (slot < uint32_t(kBinChunk)) {
        if constexpr (kKey64) s_key[slot] = (uint64_t(tile) << db) | dlow;
        else s_key[slot] = (db >= 32 ? 0u : (tile << db)) | dlow;
        s_val[slot] = g;
      }
    }
    __syncwarp();
  });
  __syncthreads();
  // (4) chunk-local slot i of tile t goes to s_gofs[t] + i
  const uint32_t c0 = blockIdx.x * uint32_t(kBinChunk);
  const int n = int(min(uint32_t(kBinChunk), a.R - c0));
  for (int i = threadIdx.x; i < n; i += kBinThreads) {
    const Key key = s_key[i];
    const uint32_t tile = kKey64 ? uint32_t(uint64_t(key) >> db) : (db >= 32 ? 0u : uint32_t(key) >> db);
    const uint32_t out = tile < uint32_t(T) ? s_gofs[tile] + uint32_t(i) : 0xffffffffu;
    if (out < a.R) {
      reinterpret_cast<Key*>(a.keys)[out] = key;
      a.vals[out] = s_val[i];
    } else {
      atomicOr(a.error, kErrRange);
    }
  }
}

__global__ void iota_kernel(uint32_t* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = uint32_t(i);
}

}  // namespace

size_t bin_smem_bytes(int tiles, int key64) {
  return key64 ? ScatterSmem<uint64_t>(tiles).total : ScatterSmem<uint32_t>(tiles).total;
}

void launch_iota(uint32_t* out, int n, cudaStream_t stream) {
  if (n > 0) iota_kernel<<<(n + 255) / 256, 256, 0, stream>>>(out, n);
}

void launch_owned_counts(const BinArgs& a, uint32_t* count, cudaStream_t stream) {
  if (a.P <= 0) return;
  owned_count_kernel<<<(a.P + 255) / 256, 256, 0, stream>>>(a, count);
}

void launch_binning(const BinArgs& a, cudaStream_t stream) {
  if (a.R == 0 || a.P <= 0) return;
  const int chunks = int((a.R + kBinChunk - 1) / kBinChunk);
  const uint32_t shares = (a.R + kWarpShare - 1) / kWarpShare;
  const size_t scatter_smem = bin_smem_bytes(a.T, a.key64);
  // the shared-memory opt-in, for the largest tile count, once per device
  static bool opted[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !opted[dev]) {
    const int most = int(bin_smem_bytes(kMaxBinTiles, 1));
    cudaFuncSetAttribute(bin_scatter_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
    cudaFuncSetAttribute(bin_scatter_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
    if (dev >= 0 && dev < 64) opted[dev] = true;
  }
  stage_begin(kStBinning, stream);
  cudaMemsetAsync(a.tile_total, 0, sizeof(uint32_t) * size_t(a.T), stream);
  warp_starts_kernel<<<(a.P + 255) / 256, 256, 0, stream>>>(a, shares);
  bin_count_kernel<<<chunks, kBinThreads, size_t(a.T) * 4, stream>>>(a);
  bin_offsets_kernel<<<(a.T + 31) / 32, 1024, 0, stream>>>(a, chunks);
  if (a.key64) bin_scatter_kernel<true><<<chunks, kBinThreads, scatter_smem, stream>>>(a);
  else bin_scatter_kernel<false><<<chunks, kBinThreads, scatter_smem, stream>>>(a);
  stage_end(kStBinning, stream, 4);
}

}  // namespace w2w
