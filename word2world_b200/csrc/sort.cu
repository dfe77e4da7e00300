// Stable LSD radix sort of (key, uint32 value) pairs, onesweep style
// (replaces the reference's 32-pass 2-bit sort with a host round trip per pass,
// prepareSort.cu:303-360, and the range kernel gaussianTiles.cu:6-33).
//
// Digits are sort_digit_bits(bits) = ceil(bits / ceil(bits / 9)) wide (up to
// 512 bins), so a 27-bit packed key takes 3 passes instead of 4 with 8-bit
// digits; the last digit is narrower when bits is not a multiple.
//
//   1. histogram kernel: one read of the keys gives the digit histogram of
//      every pass, plus the histogram of key >> tile_shift (the per-tile
//      instance counts);
//   2. offsets kernel: exclusive scans of those histograms; the tile scan is
//      the per-tile [start, end) range table (empty tiles get (0, 0), as the
//      reference's memset leaves them);
//   3. one onesweep kernel per digit: each CTA takes the next tile (6144 32-bit or 5120 64-bit keys)
//      (acquired through an atomic counter, so every earlier tile is already
//      running), ranks its keys stably (warp match.any or per-bit ballots), publishes its
//      per-digit counts and looks back over earlier tiles for their prefix
//      (decoupled lookback), then scatters through shared memory so the
//      global stores are coalesced.  Every wait is bounded: a wait that runs
//      out sets kErrTimeout and the kernel finishes without hanging.
//
// Ranking: match.any costs little when a warp's 32 keys hold few distinct
// digits, as the rasterizer's keys do (emitted Gaussian by Gaussian): 1.5 %
// faster per pass than ballots there; on random keys (the standalone sort) it
// measured 12 % slower than one ballot per digit bit, so SortArgs::match_rank
// chooses.
//
// Stability: keys are ranked in input order within a warp, warps in order
// within a tile, tiles in order globally -- the same order the reference's
// stable 2-bit passes produce, so equal keys keep their input order.
#include "common.cuh"
#include "kernels.h"

namespace w2w {
namespace {

constexpr uint32_t kStatAgg = 1u << 30;
constexpr uint32_t kStatInc = 2u << 30;
constexpr uint32_t kStatMask = (1u << 30) - 1u;
constexpr int kHistThreads = 256;
constexpr int kSmemTileBins = 8192;

// Width of pass p's digit.
__host__ __device__ __forceinline__ int pass_width(int p, int dbits, int bits) {
  const int left = bits - p * dbits;
  return left < dbits ? left : dbits;
}

// Each thread takes runs of kHistRun consecutive keys (vector loads) and
// merges equal consecutive digits before its shared-memory atomic: the
// rasterizer's keys arrive in emission order, where the keys of one Gaussian
// share their depth digits and mostly their tile's digits, so a warp's lanes
// would otherwise collide on one counter.
constexpr int kHistRun = 8;

template <typename K>
__device__ __forceinline__ void load_run(const K* __restrict__ keys, uint32_t i0, uint32_t nn, bool vec,
                                         K (&k)[kHistRun]) {
  if (vec && i0 + kHistRun <= nn) {
    const uint4* q = reinterpret_cast<const uint4*>(keys + i0);
    constexpr int kPer = 16 / sizeof(K);
#pragma unroll
    for (int j = 0; j < kHistRun / kPer; ++j) {
      const uint4 w = __ldg(q + j);
      const K* e = reinterpret_cast<const K*>(&w);
#pragma unroll
      for (int u = 0; u < kPer; ++u) k[j * kPer + u] = e[u];
    }
  } else {
#pragma unroll
    for (int j = 0; j < kHistRun; ++j) k[j] = i0 + j < nn ? keys[i0 + j] : K(0);
  }
}

// Adds the run-merged counts of (k[j] >> shift) & mask, j < cnt, to counters
// (values >= limit are skipped).
template <typename K>
__device__ __forceinline__ void count_run(const K (&k)[kHistRun], int cnt, int shift, uint32_t mask, uint32_t limit,
                                          uint32_t* counters) {
  uint32_t cur = uint32_t(k[0] >> shift) & mask, run = 1;
#pragma unroll
  for (int j = 1; j < kHistRun; ++j) {
    const uint32_t d = uint32_t(k[j] >> shift) & mask;
    const bool flush = j < cnt && d != cur;
    if (flush && cur < limit) atomicAdd(&counters[cur], run);
    run = flush ? 1u : run + (j < cnt ? 1u : 0u);
    cur = flush ? d : cur;
  }
  if (cur < limit) atomicAdd(&counters[cur], run);
}

template <typename K>
__global__ void __launch_bounds__(kHistThreads)
hist_kernel(const K* __restrict__ keys, long long n, int begin_bit, int passes, int dbits, int bits,
            uint32_t* __restrict__ hist, int tile_shift, int num_tiles, uint32_t* __restrict__ tile_hist,
            const uint32_t* __restrict__ n_dev) {
  extern __shared__ uint32_t smem[];
  uint32_t* sh = smem;                      // passes * kMaxBins
  uint32_t* st = smem + passes * kMaxBins;  // num_tiles when they fit
  const bool tiles_in_smem = tile_hist != nullptr && num_tiles <= kSmemTileBins;
  for (int i = threadIdx.x; i < passes * kMaxBins; i += blockDim.x) sh[i] = 0;
  if (tiles_in_smem)
    for (int i = threadIdx.x; i < num_tiles; i += blockDim.x) st[i] = 0;
  __syncthreads();
  // n < 2^30 (checked by every caller); a planned render's count is in device memory
  const uint32_t nn = n_dev != nullptr ? min(*n_dev, uint32_t(n)) : uint32_t(n);
  const bool vec = (reinterpret_cast<uintptr_t>(keys) & 15u) == 0u;
  const uint32_t runs = (nn + kHistRun - 1) / kHistRun;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < runs; c += gridDim.x * blockDim.x) {
    K k[kHistRun];
    const uint32_t i0 = c * kHistRun;
    load_run(keys, i0, nn, vec, k);
    const int cnt = int(min(uint32_t(kHistRun), nn - i0));
    for (int p = 0; p < passes; ++p)
      count_run(k, cnt, begin_bit + dbits * p, (1u << pass_width(p, dbits, bits)) - 1u, 0xffffffffu,
                sh + p * kMaxBins);
    if (tile_hist != nullptr)
      count_run(k, cnt, tile_shift, 0xffffffffu, uint32_t(num_tiles), tiles_in_smem ? st : tile_hist);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kMaxBins; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
  if (tiles_in_smem)
    for (int i = threadIdx.x; i < num_tiles; i += blockDim.x)
      if (st[i]) atomicAdd(&tile_hist[i], st[i]);
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024).
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += o;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < nw ? s_warp[lane] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += o;
    }
    if (lane < nw) s_warp[lane] = w;
  }
  __syncthreads();
  const uint32_t before = warp > 0 ? s_warp[warp - 1] : 0u;
  if (total) *total = s_warp[nw - 1];
  const uint32_t r = before + x - v;
  __syncthreads();
  return r;
}

// Digit histograms -> exclusive digit offsets (in place); tile histogram ->
// [start, end) ranges.  One block of 1024 threads.
__global__ void __launch_bounds__(1024)
offsets_kernel(uint32_t* hist, int passes, const uint32_t* tile_hist, int num_tiles, uint2* ranges) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  for (int p = 0; p < passes; ++p) {
    const uint32_t v = threadIdx.x < kMaxBins ? hist[p * kMaxBins + threadIdx.x] : 0u;
    const uint32_t ex = block_exclusive_scan(v, s_warp, nullptr);
    if (threadIdx.x < kMaxBins) hist[p * kMaxBins + threadIdx.x] = ex;
    __syncthreads();
  }
  if (tile_hist == nullptr || ranges == nullptr) return;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < num_tiles; base += blockDim.x) {
    const int t = base + threadIdx.x;
    const uint32_t c = t < num_tiles ? tile_hist[t] : 0u;
    uint32_t tot;
    const uint32_t ex = block_exclusive_scan(c, s_warp, &tot);
    const uint32_t start = s_carry + ex;
    if (t < num_tiles) ranges[t] = c ? make_uint2(start, start + c) : make_uint2(0u, 0u);
    __syncthreads();
    if (threadIdx.x == 0) s_carry += tot;
    __syncthreads();
  }
}

// Decoupled lookback for the adjacent digits d, d + 1 (d even).  A tile
// publishes both digits' status in one 64-bit store, so their flags always
// agree and one walk serves both.  Each step loads kLook predecessors' status
// words at once (relaxed loads: a status word carries its flag and count
// together and nothing else written by its tile is read) and consumes them
// newest first: aggregates add up until an inclusive prefix ends the walk; a
// tile that has not published yet ends the step, which resumes there.  The
// walk typically spans a few tens of tiles (those that started while it
// runs) and each step costs an L2 round trip (about 0.45 us measured), so a
// step reads several tiles.  Bounded wait.
template <int kLook>
__device__ __forceinline__ uint2 lookback_pair(const uint32_t* status, long long tile, int d, uint32_t* err,
                                               uint32_t spin_limit) {
  const unsigned long long* st = reinterpret_cast<const unsigned long long*>(status + d);
  constexpr unsigned long long kIncPair = (unsigned long long)(kStatInc) << 32 | kStatInc;
  uint32_t a0 = 0, a1 = 0, spins = 0;
  long long t = tile - 1;
  while (true) {
    unsigned long long w[kLook];
#pragma unroll
    for (int i = 0; i < kLook; ++i) w[i] = t - i >= 0 ? ld_relaxed64(st + (t - i) * (kMaxBins / 2)) : kIncPair;
    int used = 0;
    bool stop = false, done = false;
#pragma unroll
    for (int i = 0; i < kLook; ++i) {
      const uint32_t lo = uint32_t(w[i]), hi = uint32_t(w[i] >> 32);
      const uint32_t flag = lo & ~kStatMask;
      if (!stop && flag != 0u) {
        a0 += lo & kStatMask;
        a1 += hi & kStatMask;
        ++used;
        done = flag == kStatInc;
        stop = done;
      } else {
        stop = true;
      }
    }
    if (done) break;
    if (used == 0 && ++spins > spin_limit) {
      atomicOr(err, kErrTimeout);
      break;
    }
    t -= used;
  }
  return make_uint2(a0, a1);
}

// Lookback window: 4 tiles per step measured best on B200 for both key
// widths (20M u64 keys: 2, 4, 16, 32 -> 1.24, 1.18, 1.23, 1.26 ms; the
// rasterizer's 6M u32 keys: 2, 4, 8, 16 -> 0.180, 0.183, 0.218, 0.255 ms);
// wider windows cost more in L2 traffic and registers than the round trips
// they save.
template <typename K>
struct LookbackWindow {
  static constexpr int value = 4;
};

// Tile shape per key type: keys per thread and resident CTAs per SM (the
// register budget).  Every tile holds at least kSortTileMin keys.  Measured on
// a B200, one 9-bit pass: 32-bit keys (the rasterizer's, 5.9M pairs) 24 items
// at 2 CTAs/SM 51.7 us, against 20 / 22 / 26 / 28 / 32 at 2 (57.9, 55.6, 55.8,
// 59.7, 68.0 us) and 16 at 3 (59.8 us); 64-bit keys (20M pairs) 20 items at 2
// CTAs/SM 174.5 us, against 16 / 24 at 2 (186.8, 203.0 us) and 12 / 16 at 3
// (218.7, 211.2 us).
template <typename K>
struct OnesweepShape;
template <>
struct OnesweepShape<uint32_t> {
  static constexpr int kItems = 24, kMinBlocks = 2;
};
template <>
struct OnesweepShape<uint64_t> {
  static constexpr int kItems = 20, kMinBlocks = 2;
};
template <typename K>
__host__ __device__ constexpr int onesweep_tile() { return kSortThreads * OnesweepShape<K>::kItems; }
static_assert(onesweep_tile<uint32_t>() >= kSortTileMin && onesweep_tile<uint64_t>() >= kSortTileMin,
              "scratch is sized for tiles of at least kSortTileMin keys");

template <typename K>
struct OnesweepShared {
  uint32_t wcnt[kSortThreads / 32][kMaxBins];  // per-warp digit counts, then each warp's base within the digit
  uint32_t excl[kMaxBins];                     // digit's first slot in the tile
  uint32_t gofs[kMaxBins];                     // output index of the digit's slot 0 (mod 2^32)
  uint32_t warp_sums[32];
  uint32_t tile;
};

// One tile of a pass.  kFull: every key of the tile exists (all tiles but the
// last), so the per-key bounds checks drop out.  Indices are 32-bit (n < 2^30).
template <typename K, int kWidth, bool kFull, bool kMatch>
__device__ __forceinline__ void onesweep_tile_pass(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                   K* __restrict__ kout, uint32_t* __restrict__ vout, uint32_t n,
                                                   int shift, const uint32_t* __restrict__ digit_base,
                                                   uint32_t* status, uint32_t* err, uint32_t tile,
                                                   uint32_t spin_limit, bool publish, OnesweepShared<K>& sm,
                                                   K* s_keys, uint32_t* s_vals) {
  constexpr int kWarps = kSortThreads / 32;
  constexpr int kItems = OnesweepShape<K>::kItems;
  constexpr int kTile = onesweep_tile<K>();
  constexpr int bins = 1 << kWidth;
  const uint32_t dmask = uint32_t(bins) - 1u;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t base = tile * uint32_t(kTile);
  const uint32_t wbase = base + uint32_t(warp * 32 * kItems + lane);  // item i: wbase + 32 i

  K k[kItems];
  uint32_t v[kItems];
  uint32_t rank[kItems];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t idx = wbase + uint32_t(i * 32);
    if (kFull || idx < n) {
      k[i] = __ldg(kin + idx);
      v[i] = vin != nullptr ? __ldg(vin + idx) : idx;  // no values: the keys' positions
    } else {
      k[i] = K(0);
      v[i] = 0u;
    }
  }
  // early counts: per-warp digit histograms, so the tile's counts are
  // published before the ranking and successors find them sooner
#pragma unroll
  for (int i = 0; i < kItems; ++i)
    if (kFull || wbase + uint32_t(i * 32) < n) atomicAdd(&sm.wcnt[warp][uint32_t(k[i] >> shift) & dmask], 1u);
  __syncthreads();

  // two adjacent digits per thread: exclusive over warps (each warp's base
  // within the digit), tile counts, publish
  const int d0 = 2 * tid;
  uint32_t c0 = 0, c1 = 0;
  if (d0 < bins) {
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      uint2* p = reinterpret_cast<uint2*>(&sm.wcnt[w][d0]);
      const uint2 x = *p;
      *p = make_uint2(c0, c1);
      c0 += x.x;
      c1 += x.y;
    }
    const uint32_t flag = tile == 0 ? kStatInc : kStatAgg;
    if (publish)
      st_relaxed64(reinterpret_cast<unsigned long long*>(status + size_t(tile) * kMaxBins + d0),
                   (uint64_t(flag | c1) << 32) | (flag | c0));
  }
  const uint32_t excl = block_exclusive_scan(c0 + c1, sm.warp_sums, nullptr);  // ends with a barrier
  if (d0 < bins) *reinterpret_cast<uint2*>(sm.excl + d0) = make_uint2(excl, excl + c0);

  // stable rank within the tile's digit: warp base + earlier items of the warp
  // + earlier lanes of this item holding the same digit (the lanes holding
  // it: one match.any, or one ballot per digit bit; see "Ranking" above)
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t d = uint32_t(k[i] >> shift) & dmask;
    const bool valid = kFull || wbase + uint32_t(i * 32) < n;
    uint32_t pm = kFull ? 0xffffffffu : __ballot_sync(0xffffffffu, valid);
    if constexpr (kMatch) {
      pm &= __match_any_sync(0xffffffffu, d);
    } else {
#pragma unroll
      for (int bt = 0; bt < kWidth; ++bt) {
        const uint32_t bal = __ballot_sync(0xffffffffu, (d >> bt) & 1u);
        pm &= ((d >> bt) & 1u) ? bal : ~bal;
      }
    }
    const uint32_t before = valid ? sm.wcnt[warp][d] : 0u;
    rank[i] = before + __popc(pm & lt);
    __syncwarp();
    if (valid && lane == __ffs(pm) - 1) sm.wcnt[warp][d] = before + __popc(pm);
    __syncwarp();
  }

  // exclusive prefix over earlier tiles (decoupled lookback), after the ranking
  // so that predecessors have had that long to publish
  if (d0 < bins) {
    uint32_t a0 = 0, a1 = 0;
    if (tile > 0) {
      const uint2 a = lookback_pair<LookbackWindow<K>::value>(status, tile, d0, err, spin_limit);
      a0 = a.x;
      a1 = a.y;
      if (publish)
        st_relaxed64(reinterpret_cast<unsigned long long*>(status + size_t(tile) * kMaxBins + d0),
                     (uint64_t(kStatInc | (a1 + c1)) << 32) | (kStatInc | (a0 + c0)));
    }
    const uint2 ex = *reinterpret_cast<const uint2*>(sm.excl + d0);
    // sorted slot j of digit d goes to gofs[d] + j
    *reinterpret_cast<uint2*>(sm.gofs + d0) = make_uint2(digit_base[d0] + a0 - ex.x, digit_base[d0 + 1] + a1 - ex.y);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    if (kFull || wbase + uint32_t(i * 32) < n) {
      const uint32_t pos = sm.excl[uint32_t(k[i] >> shift) & dmask] + rank[i];
      s_keys[pos] = k[i];
      s_vals[pos] = v[i];
    }
  }
  __syncthreads();
  const int nvalid = kFull ? kTile : int(min(uint32_t(kTile), n - base));
#pragma unroll 4
  for (int j = tid; j < nvalid; j += kSortThreads) {
    const K key = s_keys[j];
    const uint32_t out = sm.gofs[uint32_t(key >> shift) & dmask] + uint32_t(j);
    if (out < n) {
      kout[out] = key;
      vout[out] = s_vals[j];
    } else {
      atomicOr(err, kErrRange);
    }
  }
}

// kWidth: this pass's digit width (compile-time).  kMatch: rank with
// match.any (keys whose warps hold few distinct digits, such as the
// rasterizer's, emitted Gaussian by Gaussian) or with one ballot per digit
// bit (constant cost whatever the keys: random keys).
template <typename K, int kWidth, bool kMatch>
__global__ void __launch_bounds__(kSortThreads, OnesweepShape<K>::kMinBlocks)
onesweep_kernel(const K* __restrict__ kin, const uint32_t* __restrict__ vin, K* __restrict__ kout,
                uint32_t* __restrict__ vout, long long n, int shift,
                const uint32_t* __restrict__ digit_base, uint32_t* status, uint32_t* counter, uint32_t* err,
                uint32_t spin_limit, long long unpublished_tile, const uint32_t* __restrict__ n_dev) {
  constexpr int kTile = onesweep_tile<K>();
  static_assert(kSortThreads * 2 >= kMaxBins, "at most two digits per thread");
  __shared__ __align__(16) OnesweepShared<K> sm;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  K* s_keys = reinterpret_cast<K*>(s_dyn);
  uint32_t* s_vals = reinterpret_cast<uint32_t*>(s_dyn + sizeof(K) * kTile);
  if (threadIdx.x == 0) sm.tile = atomicAdd(counter, 1u);
  // n < 2^30 (checked by every caller).  A planned render launches tiles for
  // its capacity and reads the count from device memory: a tile past the
  // count has no keys, and no real tile looks back at it, so it leaves
  // before any other work.
  const uint32_t nn = n_dev != nullptr ? min(*n_dev, uint32_t(n)) : uint32_t(n);
  if (n_dev != nullptr) {  // grid-uniform
    __syncthreads();
    if ((unsigned long long)sm.tile * kTile >= nn) return;
  }
  {
    uint4* z = reinterpret_cast<uint4*>(&sm.wcnt[0][0]);
    for (int i = threadIdx.x; i < int(sizeof(sm.wcnt) / 16); i += kSortThreads) z[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  __syncthreads();
  const uint32_t tile = sm.tile;
  if ((unsigned long long)tile * kTile >= nn) return;
  const bool publish = (long long)tile != unpublished_tile;
  if ((unsigned long long)(tile + 1) * kTile <= nn)
    onesweep_tile_pass<K, kWidth, true, kMatch>(kin, vin, kout, vout, nn, shift, digit_base, status, err, tile, spin_limit,
                                        publish, sm, s_keys, s_vals);
  else
    onesweep_tile_pass<K, kWidth, false, kMatch>(kin, vin, kout, vout, nn, shift, digit_base, status, err, tile, spin_limit,
                                         publish, sm, s_keys, s_vals);
}

template <typename K, int kWidth, bool kMatch>
void launch_onesweep_w(int tiles, cudaStream_t stream, const K* kin, const uint32_t* vin, K* kout, uint32_t* vout,
                       long long n, int shift, const uint32_t* digit_base, uint32_t* status, uint32_t* counter,
                       uint32_t* err, uint32_t spin_limit, long long unpublished, const uint32_t* n_dev) {
  const size_t dyn = (sizeof(K) + sizeof(uint32_t)) * size_t(onesweep_tile<K>());
  // the shared-memory opt-in is set once per device (a driver call per launch
  // would widen the gap the device waits between launches)
  static bool opted[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !opted[dev]) {
    cudaFuncSetAttribute(onesweep_kernel<K, kWidth, kMatch>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn));
    if (dev >= 0 && dev < 64) opted[dev] = true;
  }
  onesweep_kernel<K, kWidth, kMatch><<<tiles, kSortThreads, dyn, stream>>>(kin, vin, kout, vout, n, shift, digit_base,
                                                                    status, counter, err, spin_limit, unpublished, n_dev);
}

template <typename K>
void launch_onesweep(int width, int tiles, cudaStream_t stream, const K* kin, const uint32_t* vin, K* kout,
                     uint32_t* vout, long long n, int shift, const uint32_t* digit_base, uint32_t* status,
                     uint32_t* counter, uint32_t* err, uint32_t spin_limit, long long unpublished, bool match,
                     const uint32_t* n_dev) {
  switch (width) {
#define W2W_ONESWEEP_CASE(W)                                                                                      \
  case W:                                                                                                         \
    if (match)                                                                                                    \
      launch_onesweep_w<K, W, true>(tiles, stream, kin, vin, kout, vout, n, shift, digit_base, status, counter,   \
                                    err, spin_limit, unpublished, n_dev);                                         \
    else                                                                                                          \
      launch_onesweep_w<K, W, false>(tiles, stream, kin, vin, kout, vout, n, shift, digit_base, status, counter,  \
                                     err, spin_limit, unpublished, n_dev);                                        \
    break;
    W2W_ONESWEEP_CASE(1) W2W_ONESWEEP_CASE(2) W2W_ONESWEEP_CASE(3) W2W_ONESWEEP_CASE(4) W2W_ONESWEEP_CASE(5)
    W2W_ONESWEEP_CASE(6) W2W_ONESWEEP_CASE(7) W2W_ONESWEEP_CASE(8) W2W_ONESWEEP_CASE(9)
#undef W2W_ONESWEEP_CASE
    default:
      break;
  }
}

template <typename K>
void run_sort(const SortArgs& a, cudaStream_t stream) {
  const int passes = sort_passes(a.bits);
  const int dbits = sort_digit_bits(a.bits);
  const long long n = a.n;
  if (n <= 0) return;
  const long long tiles = (n + onesweep_tile<K>() - 1) / onesweep_tile<K>();
  if (a.clear_span != nullptr) {  // the caller's layout puts everything to clear in one span
    cudaMemsetAsync(a.clear_span, 0, a.clear_bytes, stream);
  } else {
    cudaMemsetAsync(a.hist, 0, sizeof(uint32_t) * kMaxBins * kMaxPasses, stream);
    cudaMemsetAsync(a.counters, 0, sizeof(uint32_t) * kMaxPasses, stream);
    cudaMemsetAsync(a.status, 0, sizeof(uint32_t) * kMaxBins * size_t(tiles) * size_t(passes > 0 ? passes : 1),
                    stream);
    if (a.tile_hist) cudaMemsetAsync(a.tile_hist, 0, sizeof(uint32_t) * size_t(a.num_tiles), stream);
  }
  if (passes > 0 || a.tile_hist) {
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // a few blocks per SM: each block's flush is passes * kMaxBins global atomics (4 per SM measured
    // 0.119 ms of histogram per 4-view step against 0.129 with 2 and 0.135 with 8)
    const long long want = (n + kHistThreads * kHistRun * 4 - 1) / (kHistThreads * kHistRun * 4);
    const int grid = int(max(1LL, min(want, (long long)sms * 4)));
    const bool tiles_in_smem = a.tile_hist != nullptr && a.num_tiles <= kSmemTileBins;
    const size_t smem =
        sizeof(uint32_t) * (size_t(passes) * kMaxBins + (tiles_in_smem ? size_t(a.num_tiles) : 0));
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(hist_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    const int st_hist = a.stage_hist >= 0 ? a.stage_hist : kStSortHist;
    stage_begin(st_hist, stream);
    hist_kernel<K><<<grid, kHistThreads, smem, stream>>>(reinterpret_cast<const K*>(a.keys_in), n, a.begin_bit,
                                                         passes, dbits, a.bits, a.hist, a.tile_shift,
                                                         a.num_tiles, a.tile_hist, a.n_dev);
    offsets_kernel<<<1, 1024, 0, stream>>>(a.hist, passes, a.tile_hist, a.num_tiles, a.ranges);
    stage_end(st_hist, stream, 2);
  }
  const K* kin = reinterpret_cast<const K*>(a.keys_in);
  const uint32_t* vin = a.vals_in;
  for (int p = 0; p < passes; ++p) {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    K* kout = reinterpret_cast<K*>(to_out ? a.keys_out : a.keys_tmp);
    uint32_t* vout = to_out ? a.vals_out : a.vals_tmp;
    const int st_pass = a.stage_pass >= 0 ? a.stage_pass : kStSortPass;
    stage_begin(st_pass, stream);
    launch_onesweep<K>(pass_width(p, dbits, a.bits), int(tiles), stream, kin, vin, kout, vout, n,
                       a.begin_bit + dbits * p, a.hist + kMaxBins * p,
                       a.status + size_t(p) * kMaxBins * size_t(tiles), a.counters + p, a.error,
                       a.spin_limit, p == 0 ? a.unpublished_tile : -1LL, a.match_rank != 0, a.n_dev);
    stage_end(st_pass, stream, 1);
    kin = kout;
    vin = vout;
  }
  if (passes == 0 && a.keys_in != a.keys_out) {
    cudaMemcpyAsync(a.keys_out, a.keys_in, sizeof(K) * size_t(n), cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(a.vals_out, a.vals_in, sizeof(uint32_t) * size_t(n), cudaMemcpyDeviceToDevice, stream);
  }
}

}  // namespace

long long sort_tile_keys(int key64) { return key64 ? onesweep_tile<uint64_t>() : onesweep_tile<uint32_t>(); }

int sort_passes(int bits) { return bits <= 0 ? 0 : (bits + kMaxDigitBits - 1) / kMaxDigitBits; }

int sort_digit_bits(int bits) {
  const int p = sort_passes(bits);
  return p == 0 ? 0 : (bits + p - 1) / p;
}

size_t sort_status_words(long long n) {
  const long long tiles = (n + kSortTileMin - 1) / kSortTileMin;
  return size_t(kMaxPasses) * kMaxBins * size_t(tiles > 0 ? tiles : 1);
}

void launch_sort(const SortArgs& a, cudaStream_t stream) {
  if (a.key64) run_sort<uint64_t>(a, stream);
  else run_sort<uint32_t>(a, stream);
}

}  // namespace w2w
