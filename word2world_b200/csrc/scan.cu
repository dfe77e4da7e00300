// Stand-alone single-pass scan of uint32 values with decoupled lookback
// (replaces the recursive Kogge-Stone scan of gaussianRasterizer.cu:77-117,
// which allocates, frees and synchronises the device at every level).  The
// rasterizer itself fuses its scan into the preprocess kernel; this entry
// point serves the isolated-stage workload and callers that scan alone.
#include "common.cuh"
#include "kernels.h"

namespace w2w {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;
static_assert(kScanTile == kScanTileElems, "scratch layouts assume kScanTileElems elements per tile");
constexpr unsigned long long kAgg = 1ull << 62, kInc = 2ull << 62, kFlags = 3ull << 62;

// 64-bit status words: flag in the top two bits, a uint32 partial sum (which
// wraps modulo 2^32, as the reference's uint32 scan does) in the low bits.
__global__ void __launch_bounds__(kScanThreads)
scan_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, long long n, int exclusive,
            unsigned long long* status, uint32_t* counter, uint32_t* err, uint32_t spin_limit,
            long long unpublished_tile) {
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_data[kScanTile];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(counter, 1u);
  __syncthreads();
  const long long tile = s_tile;
  const long long base = tile * kScanTile;
  // coalesced load into shared memory, then each thread scans a contiguous run
  for (int i = tid; i < kScanTile; i += kScanThreads) {
    const long long idx = base + i;
    s_data[i] = idx < n ? in[idx] : 0u;
  }
  __syncthreads();
  uint32_t v[kScanItems];
  uint32_t run = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = s_data[tid * kScanItems + k];
    run += v[k];
  }
  uint32_t x = run;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += o;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
#pragma unroll
    for (int d = 1; d < kScanThreads / 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += o;
    }
    if (lane < kScanThreads / 32) s_warp[lane] = w;
  }
  __syncthreads();
  const uint32_t total = s_warp[kScanThreads / 32 - 1];
  // decoupled lookback by warp 0: each step reads the status words of the 32
  // tiles before t at once and, once every one of them up to the nearest
  // inclusive prefix has published, adds them up (bounded wait).  A status
  // word carries its flag and count together and nothing else written by its
  // tile is read, so relaxed accesses suffice.
  if (warp == 0) {
    const bool publish = tile != unpublished_tile;
    if (tile == 0) {
      if (lane == 0) {
        if (publish) st_relaxed64(status, kInc | total);
        s_prefix = 0;
      }
    } else {
      if (lane == 0 && publish) st_relaxed64(status + tile, kAgg | total);
      uint32_t acc = 0, spins = 0;
      long long t = tile - 1;
      while (true) {
        const long long q = t - lane;
        const unsigned long long w = q >= 0 ? ld_relaxed64(status + q) : kInc;
        const unsigned long long flag = w & kFlags;
        const uint32_t inc = __ballot_sync(0xffffffffu, flag == kInc);
        const uint32_t ready = __ballot_sync(0xffffffffu, flag != 0ull);
        const uint32_t need = inc ? ((inc & (0u - inc)) << 1) - 1u : 0xffffffffu;  // lanes up to the nearest inclusive
        if ((ready & need) != need) {
          if (++spins > spin_limit) {
            if (lane == 0) atomicOr(err, kErrTimeout);
            break;
          }
          continue;
        }
        uint32_t part = (need >> lane) & 1u ? uint32_t(w) : 0u;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) part += __shfl_xor_sync(0xffffffffu, part, d);
        acc += part;
        if (inc) break;
        t -= 32;
      }
      if (lane == 0) {
        s_prefix = acc;
        if (publish) st_relaxed64(status + tile, kInc | uint32_t(acc + total));
      }
    }
  }
  __syncthreads();
  uint32_t pre = s_prefix + (warp > 0 ? s_warp[warp - 1] : 0u) + (x - run);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const uint32_t incl = pre + v[k];
    s_data[tid * kScanItems + k] = exclusive ? pre : incl;
    pre = incl;
  }
  __syncthreads();
  for (int i = tid; i < kScanTile; i += kScanThreads) {
    const long long idx = base + i;
    if (idx < n) out[idx] = s_data[i];
  }
}

// Scratch of the allocation-free entry point, laid out like a caller's
// scratch (see launch_scan) for up to kScanNoAllocMax elements.  Every device
// that loads this library holds it (about 32 KB) until exit.
constexpr long long kScanNoAllocMax = 1LL << 24;
constexpr size_t kNoAllocStatusBytes = size_t((kScanNoAllocMax + kScanTile - 1) / kScanTile) * 8;
static __device__ __align__(256) unsigned char g_scan_scratch[256 + kNoAllocStatusBytes];

}  // namespace

size_t scan_status_words(long long n) { return size_t((n + kScanTile - 1) / kScanTile) + 1; }

size_t scan_scratch_bytes(long long n) { return 256 + scan_status_words(n) * 8; }

long long scan_noalloc_max() { return kScanNoAllocMax; }

// Device address of g_scan_scratch in the current CUDA context.  Host code
// may not use the symbol itself (on the host it is only a stand-in), so the
// address is looked up with the caller's device and context current, at every
// call: the lookup is a host-side table read, and it stays right for any
// context the caller makes current (several driver-API contexts on one
// device, or a context re-created after cudaDeviceReset), where an address
// cached per device would not.  The first lookup in a context also loads the
// library's device code into it.
void* scan_noalloc_scratch(int* status) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_scan_scratch);
  if (e != cudaSuccess || p == nullptr) {
    *status = 2;
    return nullptr;
  }
  *status = 0;
  return p;
}

// scratch: [tile counter u32, error word u32, pad to 256 B][one 64-bit status
// word per tile]; one memset clears all of it.
void launch_scan(const uint32_t* in, uint32_t* out, long long n, int exclusive, void* scratch, cudaStream_t stream) {
  if (n <= 0) return;
  const long long tiles = (n + kScanTile - 1) / kScanTile;
  unsigned char* b = static_cast<unsigned char*>(scratch);
  cudaMemsetAsync(b, 0, 256 + sizeof(unsigned long long) * size_t(tiles), stream);
  uint32_t* counter = reinterpret_cast<uint32_t*>(b);
  unsigned long long* status = reinterpret_cast<unsigned long long*>(b + 256);
  stage_begin(kStScan, stream);
  scan_kernel<<<int(tiles), kScanThreads, 0, stream>>>(in, out, n, exclusive, status, counter, counter + 1,
                                                       spin_limit(), unpublished_tile(kWaitScan));
  stage_end(kStScan, stream, 1);
}

}  // namespace w2w
