// Key emission: one (tile | depth) key and one Gaussian id per covered tile
// (reference prepareSort.cu:239-301).
//
// Gaussian i owns slots [max(start_i, prev_reach_i), min(start_i + emit_i, R)),
// where start_i is its allocation offset and prev_reach_i the largest end slot
// of any earlier Gaussian (both from the preprocess scan).  With the
// reference's emission rectangle (compat mode) a Gaussian may emit more keys
// than it allocated; those keys land in its successors' slots, and each slot
// is written exactly once, by the lowest-index Gaussian whose emission covers
// it.  Entries are written in row-major order of the rectangle
// (prepareSort.cu:191-204).
//
// Batched calls: every view's Gaussians emit into its own slot range, with its
// own tile grid, and tile ids offset by the view's first global tile.
//
// Load balance: each warp expands 32 consecutive Gaussians; every lane emits
// one entry per round, so large and small Gaussians cost the same per entry
// and stores to consecutive slots are coalesced.
#include "common.cuh"
#include "kernels.h"

namespace w2w {
namespace {

constexpr int kDupThreads = 256;

template <bool kKey64>
__global__ void __launch_bounds__(kDupThreads) duplicate_kernel(DuplicateArgs a) {
  const int lane = threadIdx.x & 31;
  const int warp_global = (blockIdx.x * kDupThreads + threadIdx.x) >> 5;
  const int g = warp_global * 32 + lane;
  uint32_t p0 = 0, cnt = 0, start = 0, x0 = 0, y0 = 0, w = 1, dlow = 0, gwv = uint32_t(a.gw), tbase = 0;
  // a planned render's instance count is read from device memory (a.R is then the capacity)
  const uint32_t Rlim = a.n_dev != nullptr ? min(*a.n_dev, a.R) : a.R;
  if (g < a.P) {  // Gaussians that emit nothing have an empty rectangle
    uint32_t end = Rlim;
    if (a.items != nullptr) {  // batched: this view's tile grid, first tile id and end slot
      const int item = find_item_elem(a.items, a.num_items, uint32_t(g));
      gwv = uint32_t(a.items[item].gw);
      tbase = a.items[item].tile_base;
      end = a.item_end[item];
    }
    start = a.offsets[g] - a.tiles[g];
    const uint2 rc = reinterpret_cast<const uint2*>(a.rect)[g];
    x0 = rc.x & 0xffffu;
    y0 = rc.x >> 16;
    const uint32_t x1 = rc.y & 0xffffu, y1 = rc.y >> 16;
    w = x1 > x0 ? x1 - x0 : 1u;
    const uint32_t n = (x1 > x0 && y1 > y0) ? (x1 - x0) * (y1 - y0) : 0u;
    const uint32_t reach = start + n;
    p0 = max(start, a.prev_reach[g]);
    const uint32_t p1 = min(reach, end);
    cnt = p1 > p0 ? p1 - p0 : 0u;
    const uint32_t db = __float_as_uint(a.depth[g]);
    dlow = a.depth_bits >= 32 ? db : (db & ((1u << a.depth_bits) - 1u));
  }
  // warp inclusive scan of the entry counts
  uint32_t incl = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += o;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  const uint32_t excl = incl - cnt;
  for (uint32_t base = 0; base < total; base += 32) {
    const uint32_t e = base + lane;
    // owner lane: number of lanes whose inclusive count is <= e
    int o = 0;
#pragma unroll
    for (int b = 16; b > 0; b >>= 1) {
      const uint32_t t = __shfl_sync(0xffffffffu, incl, o + b - 1);
      if (t <= e) o += b;
    }
    o = min(o, 31);
    const uint32_t op0 = __shfl_sync(0xffffffffu, p0, o);
    const uint32_t oex = __shfl_sync(0xffffffffu, excl, o);
    const uint32_t ost = __shfl_sync(0xffffffffu, start, o);
    const uint32_t ox0 = __shfl_sync(0xffffffffu, x0, o);
    const uint32_t oy0 = __shfl_sync(0xffffffffu, y0, o);
    const uint32_t ow = __shfl_sync(0xffffffffu, w, o);
    const uint32_t odl = __shfl_sync(0xffffffffu, dlow, o);
    const uint32_t ogw = __shfl_sync(0xffffffffu, gwv, o);
    const uint32_t otb = __shfl_sync(0xffffffffu, tbase, o);
    if (e < total) {
      const uint32_t p = op0 + (e - oex);
      const uint32_t k = p - ost;
      const uint32_t ty = oy0 + k / ow, tx = ox0 + k % ow;
      const uint32_t tile = otb + ty * ogw + tx;
      if (p < Rlim) {
        if constexpr (kKey64) {
          reinterpret_cast<uint64_t*>(a.keys)[p] = (uint64_t(tile) << a.depth_bits) | odl;
        } else {
          reinterpret_cast<uint32_t*>(a.keys)[p] = (a.depth_bits >= 32 ? 0u : (tile << a.depth_bits)) | odl;
        }
        a.vals[p] = uint32_t(warp_global * 32 + o);
      }
    }
  }
}

}  // namespace

void launch_duplicate(const DuplicateArgs& a, cudaStream_t stream) {
  if (a.P <= 0 || a.R == 0) return;
  const int blocks = (a.P + kDupThreads - 1) / kDupThreads;
  stage_begin(kStDuplicate, stream);
  if (a.key64) duplicate_kernel<true><<<blocks, kDupThreads, 0, stream>>>(a);
  else duplicate_kernel<false><<<blocks, kDupThreads, 0, stream>>>(a);
  stage_end(kStDuplicate, stream, 1);
}

}  // namespace w2w
