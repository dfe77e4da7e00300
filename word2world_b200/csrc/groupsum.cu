// Per-group sums of per-element gradient rows, for batched calls: a batch's
// items (views) carry their scene's Gaussians as separate element ranges, and
// a scene's (or a request's) gradient is the sum of its items' ranges.
//
// One thread per output value: row r of group g is the sum, over g's items in
// list order, of row r of each item's element range.  The order is fixed, so
// the result is deterministic (a scatter with atomics is not), and every read
// and write is coalesced.
#include "common.cuh"
#include "kernels.h"

namespace w2w {
namespace {

constexpr int kGroupThreads = 256;

__global__ void __launch_bounds__(kGroupThreads)
group_sum_kernel(const float* __restrict__ src, int width, int num_groups, const uint32_t* __restrict__ group_base,
                 const uint32_t* __restrict__ item_ptr, const uint32_t* __restrict__ item_elem,
                 float* __restrict__ dst, long long total) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < total; o += stride) {
    const uint32_t row = uint32_t(o / width);
    const int col = int(o - (long long)row * width);
    // group of this row: the last g with group_base[g] <= row
    int lo = 0, hi = num_groups - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(group_base + mid) <= row) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t r = row - __ldg(group_base + lo);
    float s = 0.0f;
    for (uint32_t k = __ldg(item_ptr + lo); k < __ldg(item_ptr + lo + 1); ++k)
      s += __ldg(src + (size_t(__ldg(item_elem + k)) + r) * size_t(width) + col);
    dst[o] = s;
  }
}

}  // namespace

void launch_group_sum(const float* src, int width, int num_groups, const uint32_t* tables, int num_items,
                      float* dst, long long total_rows, cudaStream_t stream) {
  const long long total = total_rows * width;
  if (total <= 0 || num_groups <= 0) return;
  const uint32_t* group_base = tables;
  const uint32_t* item_ptr = tables + (num_groups + 1);
  const uint32_t* item_elem = item_ptr + (num_groups + 1);
  (void)num_items;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (total + kGroupThreads - 1) / kGroupThreads;
  const int grid = int(want > (long long)sms * 16 ? (long long)sms * 16 : want);
  stage_begin(kStOther, stream);
  group_sum_kernel<<<grid, kGroupThreads, 0, stream>>>(src, width, num_groups, group_base, item_ptr, item_elem, dst,
                                                       total);
  stage_end(kStOther, stream, 1);
}

}  // namespace w2w
