// Per-tile front-to-back alpha blending (reference pixelGaussiansFull.cu:3-98,
// pixelGaussiansDev.cuh:5-96, gaussEval.h:7-29).
//
// One CTA per 16x16 tile, one thread per pixel, one warp per 8x4 pixel block
// (tile_walk.cuh).  Each warp walks only the list entries that can reach its
// block with alpha >= 1/255, kBlendIlp at a time: all their Gaussian values are
// evaluated before the sequential transmittance/colour updates, so the
// evaluations overlap.  The CTA stops as soon as every pixel of the tile has
// terminated (the reference keeps loading every batch of the tile).
//
// Per pixel the arithmetic is the reference's, in its operation order: the
// Gaussian is evaluated from the 2-D covariance and its determinant
// (mahalanobis / det, negative -> 1000), alpha = min(0.99, o*g), entries with
// alpha < 1/255 are skipped, the pixel terminates before the entry that would
// take transmittance below 1e-4, colour accumulates with fma, and the
// contributor count is the 1-based index of the last blended entry.
#include "common.cuh"
#include "kernels.h"
#include "tile_walk.cuh"
#include "tma.cuh"

#include <algorithm>
#include <mutex>

namespace w2w {
namespace {

constexpr int kBlendIlp = 4;  // list entries evaluated together per warp (the list is read 4 bytes at a time)
static_assert(kBlendIlp == 4, "packed list read");

// The reference's Gaussian value (gaussEval.h:7-29) in two halves: the
// mahalanobis numerator, then exp(-0.5 * num / det) with negative distances
// mapped to 1000.
__device__ __forceinline__ float gauss_num(float px, float py, float mx, float my, float cxx, float cxy, float cyy) {
  using namespace fp;
  const float dx = sub(px, mx), dy = sub(py, my);
  const float tX = d2<BL_TX>(dx, cyy, dy, cxy);
  const float tY = s2<BL_TY>(-dx, cxy, dy, cxx);
  return s2<BL_NUM>(tX, dx, tY, dy);
}
__device__ __forceinline__ float gauss_from_m(float m) {
  if (m < 0.0f) m = 1000.0f;
  return expf(mul(-0.5f, m));
}

struct BlendPixel {
  float C0 = 0.f, C1 = 0.f, C2 = 0.f, Wt = 0.f, D = 0.f, T = 1.0f;
  uint32_t last = 0;
  bool done;

  // Entry with alpha `al` (record words q1, q2), 1-based list position `pos`.
  // Branch-free: the updates are selected, so a warp's lanes never diverge.
  // An entry that does not accumulate adds exactly zero: its weight aT is
  // selected to 0, colours and depth are finite, and C, Wt and D are never
  // -0 (non-negative colours and weights, positive depths), so x + c * 0 = x.
  __device__ __forceinline__ void step(float al, float4 q1, float4 q2, uint32_t pos) {
    const bool blend = !done && al >= 1.0f / 255.0f;
    const float nT = mul(T, sub(1.0f, al));
    const bool term = blend && nT < 0.0001f;
    const bool acc = blend && !term;
    const float aT = acc ? mul(al, T) : 0.0f;
    C0 = fma(q2.x, aT, C0);
    C1 = fma(q2.y, aT, C1);
    C2 = fma(q2.z, aT, C2);
    Wt = add(Wt, aT);
    D = s1<fp::BL_DEPTH>(q1.w, aT, D);
    T = acc ? nT : T;
    last = acc ? pos : last;
    done = done || term;
  }
};

// Warps per CTA, kBlendWarps: 8 (one CTA per tile) or 4 (two CTAs per tile,
// upper and lower eight rows; see tile_walk.cuh), chosen at run time (the
// tuning knob "blend_warps"); kAsync: the next batch is copied into shared
// memory with cp.async instead of gathered into registers (the knob
// "blend_stage"), which leaves the 4-warp CTA few enough registers for five
// CTAs per SM instead of four.  Results are identical in every combination.
template <int kBlendWarps, bool kAsync>
constexpr int blend_min_blocks() {
  return kAsync && kBlendWarps == 4 ? 5 : 16 / kBlendWarps;
}

template <int kBlendWarps, bool kAsync>
__global__ void __launch_bounds__(32 * kBlendWarps, (blend_min_blocks<kBlendWarps, kAsync>()))
    blend_kernel(BlendArgs a) {
  constexpr int kBlendParts = 8 / kBlendWarps;  // CTAs per tile
  constexpr int kBlendCta = 32 * kBlendWarps;
  constexpr int kStagePer = kBatch / kBlendCta;  // entries each thread stages per batch
  constexpr int kVec = kAsync ? kStageVec : kRecVec;  // float4s per staged record
  static_assert(kBatch % kBlendCta == 0, "whole entries per thread");
  __shared__ TileWalkShared<kBlendWarps, kVec> sm;
  const int part = int(blockIdx.x) % kBlendParts;
  const int tile = int(a.order[blockIdx.x / kBlendParts]);
  // this tile's image: the call's, or its batch item's
  int W = a.W, H = a.H, ltile = tile;
  size_t pbase = 0;
  const float* bg = a.bg;
  if (a.items != nullptr) {
    const BatchItem& it = a.items[find_item_tile(a.items, a.num_items, uint32_t(tile))];
    W = it.W;
    H = it.H;
    ltile = tile - int(it.tile_base);
    pbase = size_t(it.pix_base);
    bg = it.bg;
  }
  const int gw = (W + kTile - 1) / kTile;
  const int warp = int(threadIdx.x >> 5), first_block = part * kBlendWarps;
  const TilePixel tp(ltile, gw, first_block + warp);
  const bool inside = tp.px < W && tp.py < H;
  const uint2 range = a.ranges[tile];
  const int n = int(range.y - range.x);
  const float pxf = float(tp.px), pyf = float(tp.py);

  BlendPixel pix;
  pix.done = !inside;
  const int nb = (n + kBatch - 1) / kBatch;
  Staged st[kAsync ? 1 : kStagePer];    // register staging: the batch in flight
  bool staged[kAsync ? kStagePer : 1];  // cp.async staging: slot r * kBlendCta + threadIdx.x holds a record
  auto load = [&](int buf, int base) {
#pragma unroll
    for (int r = 0; r < kStagePer; ++r) {
      const int j = r * kBlendCta + int(threadIdx.x), e = base + j;
      if constexpr (kAsync)
        staged[r] = stage_copy(&sm.rec[buf][kVec * j], a.record, a.point_list, range.x + e, e < n, a.num_records);
      else
        stage_load(st[r], a.record, a.point_list, range.x + e, e < n, a.num_records);
    }
    if constexpr (kAsync) cp_async_commit();
  };
  // block masks for the backward: the upper half's CTA (or the whole tile's)
  // writes the top array, the lower half's the bottom one
  uint8_t* lo_dst = a.mask_top == nullptr ? nullptr : (part == 0 ? a.mask_top : a.mask_bottom) + range.x;
  uint8_t* hi_dst = a.mask_top == nullptr || kBlendParts != 1 ? nullptr : a.mask_bottom + range.x;
  auto store = [&](int buf, int base) {
    if constexpr (kAsync) cp_async_wait_all();
#pragma unroll
    for (int r = 0; r < kStagePer; ++r) {
      const int j = r * kBlendCta + int(threadIdx.x);
      uint8_t* lo = lo_dst ? lo_dst + base : nullptr;
      uint8_t* hi = hi_dst ? hi_dst + base : nullptr;
      if constexpr (kAsync) stage_mask(sm, buf, staged[r], j, tp.X0, tp.Y0, first_block, lo, hi);
      else stage_store(sm, buf, st[r], j, tp.X0, tp.Y0, first_block, lo, hi);
    }
  };
  if (nb > 0) {
    load(0, 0);
    store(0, 0);
  }
  for (int b = 0; b < nb; ++b) {
    const int cur = b & 1;
    // barrier: batch b is staged; every warp has finished batch b-1
    if (__syncthreads_count(pix.done ? 1 : 0) == kBlendCta) break;
    const int next_base = (b + 1) * kBatch;
    if (b + 1 < nb) load(cur ^ 1, next_base);  // in flight while batch b is walked
    if (!__all_sync(0xffffffffu, pix.done)) {
      const float4* s = sm.rec[cur];
      const int cnt = build_list(sm, cur, warp, tp.lane);
      const uint8_t* lst = sm.list[warp];
      const uint32_t base = uint32_t(b * kBatch) + 1u;
      for (int k0 = 0; k0 < cnt; k0 += kBlendIlp) {
        // kBlendIlp entries in flight: their Gaussian values are independent,
        // only the transmittance/colour updates are sequential
        const uint32_t packed = *reinterpret_cast<const uint32_t*>(lst + k0);
        int j[kBlendIlp];
#pragma unroll
        for (int k = 0; k < kBlendIlp; ++k) j[k] = k0 + k < cnt ? int((packed >> (8 * k)) & 255u) : -1;
        float al[kBlendIlp], num[kBlendIlp], m[kBlendIlp];
        float4 q1[kBlendIlp], q2[kBlendIlp];
        bool in_range = true;
#pragma unroll
        for (int k = 0; k < kBlendIlp; ++k) {
          const int jj = j[k] < 0 ? j[0] : j[k];
          const float4 q0 = s[kVec * jj];
          q1[k] = s[kVec * jj + 1];
          q2[k] = s[kVec * jj + 2];
          num[k] = gauss_num(pxf, pyf, q0.x, q0.y, q0.z, q0.w, q1[k].x);
          in_range = in_range && div_in_range(num[k], q1[k].y);
        }
        // the branch-free division when every lane's operands allow it
        if (__all_sync(0xffffffffu, in_range)) {
#pragma unroll
          for (int k = 0; k < kBlendIlp; ++k) m[k] = div_markstein(num[k], q1[k].y);
        } else {
#pragma unroll
          for (int k = 0; k < kBlendIlp; ++k) m[k] = div(num[k], q1[k].y);
        }
#pragma unroll
        for (int k = 0; k < kBlendIlp; ++k)
          al[k] = j[k] < 0 ? 0.0f : fminf(0.99f, mul(q1[k].z, gauss_from_m(m[k])));
#pragma unroll
        for (int k = 0; k < kBlendIlp; ++k) pix.step(al[k], q1[k], q2[k], base + uint32_t(j[k]));
        if (__all_sync(0xffffffffu, pix.done)) break;
      }
    }
    if (b + 1 < nb) store(cur ^ 1, next_base);
  }
  if (inside) {
    const size_t q = size_t(tp.py) * W + tp.px;
    const size_t p = pbase + q, cp = 3 * pbase + q;
    const size_t hw = size_t(W) * H;
    a.n_contrib[p] = pix.last;
    a.out_alpha[p] = pix.Wt;
    a.out_depth[p] = pix.D;
    a.T_final[p] = pix.T;
    a.out_color[cp] = fma(pix.T, bg[0], pix.C0);
    a.out_color[hw + cp] = fma(pix.T, bg[1], pix.C1);
    a.out_color[2 * hw + cp] = fma(pix.T, bg[2], pix.C2);
  }
  // largest contributor count in the tile (the backward starts there); the
  // tile's CTAs combine theirs (tile_max is cleared before the launch)
  __shared__ uint32_t s_max[kBlendWarps];
  const uint32_t wm = __reduce_max_sync(0xffffffffu, pix.last);
  if (tp.lane == 0) s_max[warp] = wm;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t mx = 0;
    for (int w = 0; w < kBlendWarps; ++w) mx = max(mx, s_max[w]);
    if (kBlendParts == 1) a.tile_max[tile] = mx;
    else atomicMax(&a.tile_max[tile], mx);
  }
}

// ---------------------------------------------------------------------------
// Persistent blend over a device tile queue, staged by TMA row gathers.
//
// A CTA runs kW consumer warps (the blocks of one tile half, or of the whole
// tile for kW = 8) and one producer warp, for as long as the queue (tile
// halves in the heaviest-first order; every item of a batched call in one
// queue) has items.  The producer takes the next item with an atomic, reads
// a batch's Gaussian ids from the list, writes the stage's header and the
// bit mask of its valid entries, and gathers the entries' 64-byte records into
// one of kQStages shared-memory stages with TMA (four rows per gather),
// completing on the stage's barrier.  Each consumer warp waits for that
// barrier, tests the staged entries against its own 8x4 block (block_test,
// as the backward's warps do), walks the ones that can reach it as the
// per-tile kernel does, and releases the stage.  A warp whose pixels have all
// terminated tells the producer, which skips the rest of a tile once every
// consumer warp has.  The stages run across tile boundaries, so a CTA never
// drains its pipeline between tiles, and no warp waits at a CTA barrier for
// the slowest warp of a batch: warps drift apart by up to kQStages batches.
// This blend writes no block masks: it clears the binning state's flag, and
// the backward tests each entry itself.
// Every wait is bounded; one that runs out sets kErrTimeout in `error`, and
// the CTA stops after its copies in flight land.  Results are bit-identical
// to blend_kernel's (same entries, same order).
// ---------------------------------------------------------------------------
constexpr int kQStages = 3;
constexpr int kQRec = 4;  // float4s per staged record (the whole record)

struct QueueStage {
  int tile;   // tile id (-1: the queue is empty, stop)
  int part;   // tile half (kW = 4) or 0
  int base;   // list position of the batch's first entry, from the tile's start
  int seq;    // the CTA's item number
  int first;  // 1: the item's first batch
  int pad[3];
};

template <int kW>
struct __align__(128) QueueShared {
  float4 rec[kQStages][kBatch * kQRec];  // 16 KB per stage; gathers land 256 B at a time
  uint32_t valid[kQStages][kBatch / 32];  // bit j of word c: entry 32c + j holds a valid id
  QueueStage hdr[kQStages];
  uint8_t list[kW][kBatch];
  unsigned long long full_bar[kQStages];   // header written and the stage's gathers landed
  unsigned long long empty_bar[kQStages];  // every consumer warp is done with the stage
  uint32_t done[4];                        // per item (seq mod 4): consumer warps whose pixels all terminated
  uint32_t abort;
};

template <int kW>
constexpr size_t queue_smem_bytes() {
  return sizeof(QueueShared<kW>) + 128;  // + alignment slack of the dynamic shared memory base
}

// Bounded wait on `bar`'s phase `parity`: hardware-suspended waits of at
// most kQWaitNs each, limit / 256 + 4 of them (about 0.16 s at the default
// limit).  False when it ran out (or another warp's did), after flagging the
// CTA and the call.  Warp-collective: every lane waits (so each acquires the
// phase itself) and the warp decides together, so its lanes never part ways.
constexpr uint32_t kQWaitNs = 10000;
__device__ __forceinline__ bool queue_wait(unsigned long long* bar, uint32_t parity, volatile uint32_t* abort,
                                           uint32_t limit, uint32_t* error) {
  const uint32_t tries = (limit >> 8) + 4u;
  for (uint32_t i = 0; i < tries; ++i) {
    if (__all_sync(0xffffffffu, tma::bar_try_wait(bar, parity, kQWaitNs))) return true;
    if (__any_sync(0xffffffffu, *abort != 0u)) return false;
  }
  if ((threadIdx.x & 31u) == 0u) {
    *abort = 1u;
    if (error != nullptr) atomicOr(error, kErrTimeout);
  }
  return false;
}

// The producer's position in the queue: its current item (tile part) and
// the next batch of it to stage.  Warp-uniform.
struct QueueCursor {
  int tile = -1, part = 0, n = 0, nb = 1, b = 0;
  uint32_t rx = 0;
  bool end = true;

  // Take the next item (lane 0's atomic, broadcast) as item number `seq`;
  // clears that item's slot of `done` (seen by the consumers through the
  // item's first stage).
  template <int kW>
  __device__ __forceinline__ void fetch(const BlendArgs& a, uint32_t* done, uint32_t seq, int lane) {
    constexpr int kParts = 8 / kW;
    int item = 0;
    if (lane == 0) {
      item = int(atomicAdd(a.queue, 1u));
      done[seq & 3u] = 0u;
    }
    item = __shfl_sync(0xffffffffu, item, 0);
    end = item >= a.total_tiles * kParts;
    b = 0;
    if (end) {
      tile = -1;
      part = 0;
      n = 0;
      nb = 1;
      rx = 0;
      return;
    }
    tile = int(a.order[item / kParts]);
    part = item % kParts;
    const uint2 range = a.ranges[tile];
    rx = range.x;
    n = int(range.y - range.x);
    nb = max(1, (n + kBatch - 1) / kBatch);  // an empty list still has its pixels written
  }
};

// Every consumer warp of item `seq` has terminated (lane 0 reads, the warp agrees).
template <int kW>
__device__ __forceinline__ bool queue_all_done(const uint32_t* done, uint32_t seq, int lane) {
  uint32_t d = 0;
  if (lane == 0) d = *reinterpret_cast<const volatile uint32_t*>(&done[seq & 3u]);
  return __shfl_sync(0xffffffffu, d, 0) == uint32_t(kW);
}

template <int kW>
__global__ void __launch_bounds__(32 * (kW + 1)) blend_queue_kernel(BlendArgs a, const __grid_constant__ CUtensorMap map) {
  extern __shared__ unsigned char q_raw[];
  QueueShared<kW>& s = *reinterpret_cast<QueueShared<kW>*>((reinterpret_cast<uintptr_t>(q_raw) + 127) & ~uintptr_t(127));
  const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
  const uint32_t limit = a.spin_limit;
  volatile uint32_t* abort = &s.abort;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kQStages; ++i) {
      tma::bar_init(&s.full_bar[i], 1);
      tma::bar_init(&s.empty_bar[i], kW);
    }
    s.abort = 0u;
    tma::bar_init_fence();
    // this blend leaves no block masks for the backward passes
    if (blockIdx.x == 0 && a.masks_valid != nullptr) *a.masks_valid = 0u;
  }
  if (threadIdx.x == 32 * kW) tma::prefetch_map(&map);
  __syncthreads();

  if (warp == kW) {
    // ---------------- producer ----------------
    QueueCursor cur;
    uint32_t seq = 0, k = 0;
    cur.fetch<kW>(a, s.done, seq, lane);
    for (;; ++k) {
      if (cur.b > 0 && (cur.b >= cur.nb || queue_all_done<kW>(s.done, seq, lane))) cur.fetch<kW>(a, s.done, ++seq, lane);
      const int st = int(k % kQStages);
      if (!queue_wait(&s.empty_bar[st], ((k / kQStages) & 1u) ^ 1u, abort, limit, a.error)) goto stop;
      const int base = cur.b * kBatch;
      const int cnt = cur.end ? 0 : min(kBatch, cur.n - base);
      const int groups = (cnt + 3) >> 2;
      // lane l gathers groups l and l + 32 (entries 4g .. 4g + 3)
      const uint32_t* ids = a.point_list + cur.rx + base;
      int r[2][4];
      uint32_t vbits = 0;  // bit 4h + q: entry 4 (l + 32h) + q holds a valid id
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int g = lane + 32 * h;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int e = 4 * g + q;
          const uint32_t id = e < cnt ? ids[e] : a.num_records;
          const bool ok = id < a.num_records;
          vbits |= ok ? 1u << (4 * h + q) : 0u;
          r[h][q] = ok ? int(id) : 0;  // a stray id gathers row 0 and stays invalid
        }
      }
      // the stage's valid-entry words and header, by lane 0, before its
      // arrival (which releases them to the consumers)
#pragma unroll
      for (int c = 0; c < kBatch / 32; ++c) {
        const int j = 32 * c + lane, g = j >> 2;
        const uint32_t w = __ballot_sync(0xffffffffu, (__shfl_sync(0xffffffffu, vbits, g & 31) >> (4 * (g >> 5) + (j & 3))) & 1u);
        if (lane == 0) s.valid[st][c] = w;
      }
      if (lane == 0) {
        s.hdr[st] = QueueStage{cur.tile, cur.part, base, int(seq), cur.b == 0 ? 1 : 0, {0, 0, 0}};
        tma::bar_arrive_expect(&s.full_bar[st], uint32_t(groups) * 4u * 64u);  // an empty stage completes at once
      }
      __syncwarp();
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int g = lane + 32 * h;
        if (g < groups) tma::gather4(&s.rec[st][kQRec * 4 * g], &map, &s.full_bar[st], r[h][0], r[h][1], r[h][2], r[h][3]);
      }
      ++cur.b;
      if (cur.end) break;
    }
    return;
  stop:
    // a wait ran out: let the copies of the stages issued last land before the CTA ends
    for (uint32_t kk = k > uint32_t(kQStages) ? k - kQStages : 0u; kk < k; ++kk) {
      const int st = int(kk % kQStages);
      for (uint32_t i = 0; i < (limit >> 8) + 4u && !tma::bar_try_wait(&s.full_bar[st], (kk / kQStages) & 1u, kQWaitNs);
           ++i) {
      }
    }
    return;
  }

  // ---------------- consumers ----------------
  BlendPixel pix;
  pix.done = true;
  bool have = false, reported = true;
  int tile = -1, W = 0, H = 0;
  size_t pbase = 0;
  const float* bg = a.bg;
  TilePixel tp(0, 1, warp);
  float pxf = 0.f, pyf = 0.f;
  auto finish = [&]() {
    if (!have) return;
    if (tp.px < W && tp.py < H) {
      const size_t q = size_t(tp.py) * W + tp.px;
      const size_t p = pbase + q, cp = 3 * pbase + q;
      const size_t hw = size_t(W) * H;
      a.n_contrib[p] = pix.last;
      a.out_alpha[p] = pix.Wt;
      a.out_depth[p] = pix.D;
      a.T_final[p] = pix.T;
      a.out_color[cp] = fma(pix.T, bg[0], pix.C0);
      a.out_color[hw + cp] = fma(pix.T, bg[1], pix.C1);
      a.out_color[2 * hw + cp] = fma(pix.T, bg[2], pix.C2);
    }
    const uint32_t wm = __reduce_max_sync(0xffffffffu, pix.last);
    if (lane == 0 && wm != 0u) atomicMax(&a.tile_max[tile], wm);
  };
  const uint32_t lt = (1u << lane) - 1u;
  for (uint32_t k = 0;; ++k) {
    const int st = int(k % kQStages);
    if (!queue_wait(&s.full_bar[st], (k / kQStages) & 1u, abort, limit, a.error)) return;
    const QueueStage h = s.hdr[st];
    if (h.first != 0 || h.tile < 0) {
      finish();
      if (h.tile < 0) return;
      tile = h.tile;
      int ltile = tile;
      W = a.W;
      H = a.H;
      pbase = 0;
      bg = a.bg;
      if (a.items != nullptr) {
        const BatchItem& it = a.items[find_item_tile(a.items, a.num_items, uint32_t(tile))];
        W = it.W;
        H = it.H;
        ltile = tile - int(it.tile_base);
        pbase = size_t(it.pix_base);
        bg = it.bg;
      }
      tp = TilePixel(ltile, (W + kTile - 1) / kTile, h.part * kW + warp);
      pxf = float(tp.px);
      pyf = float(tp.py);
      pix = BlendPixel();
      pix.done = !(tp.px < W && tp.py < H);
      have = true;
      reported = false;
    }
    if (!__all_sync(0xffffffffu, pix.done)) {
      const float4* sr = s.rec[st];
      // the stage's entries that can reach this warp's block, in order
      int cnt = 0;
#pragma unroll 2
      for (int c = 0; c < kBatch / 32; ++c) {
        const uint32_t vw = s.valid[st][c];
        bool reach = false;
        if ((vw >> lane) & 1u) {
          const int j = 32 * c + lane;
          const float4 r0 = sr[kQRec * j], r2 = sr[kQRec * j + 2], r3 = sr[kQRec * j + 3];
          reach = block_test(r0.x, r0.y, r2.w, r3.x, r3.y, r3.z, r3.w, tp.bx, tp.by);
        }
        const uint32_t bits = __ballot_sync(0xffffffffu, reach);
        if (reach) s.list[warp][cnt + __popc(bits & lt)] = uint8_t(32 * c + lane);
        cnt += __popc(bits);
      }
      __syncwarp();
      const uint8_t* lst = s.list[warp];
      const uint32_t base = uint32_t(h.base) + 1u;
      for (int k0 = 0; k0 < cnt; k0 += kBlendIlp) {
        const uint32_t packed = *reinterpret_cast<const uint32_t*>(lst + k0);
        int j[kBlendIlp];
#pragma unroll
        for (int kk = 0; kk < kBlendIlp; ++kk) j[kk] = k0 + kk < cnt ? int((packed >> (8 * kk)) & 255u) : -1;
        float al[kBlendIlp], num[kBlendIlp], m[kBlendIlp];
        float4 q1[kBlendIlp], q2[kBlendIlp];
        bool in_range = true;
#pragma unroll
        for (int kk = 0; kk < kBlendIlp; ++kk) {
          const int jj = j[kk] < 0 ? j[0] : j[kk];
          const float4 q0 = sr[kQRec * jj];
          q1[kk] = sr[kQRec * jj + 1];
          q2[kk] = sr[kQRec * jj + 2];
          num[kk] = gauss_num(pxf, pyf, q0.x, q0.y, q0.z, q0.w, q1[kk].x);
          in_range = in_range && div_in_range(num[kk], q1[kk].y);
        }
        if (__all_sync(0xffffffffu, in_range)) {
#pragma unroll
          for (int kk = 0; kk < kBlendIlp; ++kk) m[kk] = div_markstein(num[kk], q1[kk].y);
        } else {
#pragma unroll
          for (int kk = 0; kk < kBlendIlp; ++kk) m[kk] = div(num[kk], q1[kk].y);
        }
#pragma unroll
        for (int kk = 0; kk < kBlendIlp; ++kk)
          al[kk] = j[kk] < 0 ? 0.0f : fminf(0.99f, mul(q1[kk].z, gauss_from_m(m[kk])));
#pragma unroll
        for (int kk = 0; kk < kBlendIlp; ++kk) pix.step(al[kk], q1[kk], q2[kk], base + uint32_t(j[kk]));
        if (__all_sync(0xffffffffu, pix.done)) break;
      }
    }
    if (!reported && __all_sync(0xffffffffu, pix.done)) {
      reported = true;
      if (lane == 0) atomicAdd(&s.done[h.seq & 3], 1u);
    }
    __syncwarp();
    if (lane == 0) tma::bar_arrive(&s.empty_bar[st]);
  }
}

}  // namespace

// Bucket sort of the tiles by decreasing list length (quarter-octave buckets;
// order within a bucket is arbitrary).  One CTA.
__global__ void __launch_bounds__(1024) tile_order_kernel(const uint2* ranges, const uint32_t* counts, int num_tiles,
                                                          uint32_t* order, uint32_t* zero, uint32_t* counter) {
  if (counter != nullptr && threadIdx.x == 0) *counter = 0u;
  constexpr int kBuckets = 130;
  __shared__ uint32_t s_cnt[kBuckets];
  __shared__ uint32_t s_pos[kBuckets];
  auto bucket = [](uint32_t n) -> int {
    if (n == 0) return 0;
    const int e = 31 - __clz(n);
    const uint32_t q = e >= 2 ? (n >> (e - 2)) & 3u : (n << (2 - e)) & 3u;
    return 1 + 4 * e + int(q);
  };
  for (int i = threadIdx.x; i < kBuckets; i += blockDim.x) s_cnt[i] = 0;
  if (zero != nullptr)
    for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) zero[t] = 0u;
  __syncthreads();
  auto weight = [&](int t) -> uint32_t {
    if (counts) return counts[t];
    const uint2 r = ranges[t];
    return r.y - r.x;
  };
  for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) atomicAdd(&s_cnt[bucket(weight(t))], 1u);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int b = kBuckets - 1; b >= 0; --b) {
      s_pos[b] = acc;
      acc += s_cnt[b];
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) order[atomicAdd(&s_pos[bucket(weight(t))], 1u)] = uint32_t(t);
}

namespace {

// The driver's tensor-map encoder, looked up once through the runtime (the
// library links only the runtime).
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encoder() {
  static std::once_flag once;
  static EncodeTiled fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

// The records as a 2-D tensor of num_records rows of 16 floats (64 bytes),
// gathered one row per index (box: one row).  False when the map cannot be
// made (no encoder, a base not 16-byte aligned, no rows).
bool record_map(const BlendArgs& a, CUtensorMap* map) {
  if (a.record == nullptr || a.num_records == 0u || (reinterpret_cast<uintptr_t>(a.record) & 15u) != 0u) return false;
  const EncodeTiled enc = encoder();
  if (enc == nullptr) return false;
  const cuuint64_t dims[2] = {16u, cuuint64_t(a.num_records)};
  const cuuint64_t strides[1] = {64u};
  const cuuint32_t box[2] = {16u, 1u};
  const cuuint32_t elem[2] = {1u, 1u};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(a.record), dims, strides, box, elem,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Persistent grid: every CTA the SMs hold at once (at most one per item).
template <int kW>
bool launch_queue(const BlendArgs& a, int tiles, cudaStream_t stream) {
  CUtensorMap map;
  if (a.queue == nullptr || !record_map(a, &map)) return false;
  constexpr int threads = 32 * (kW + 1);
  constexpr size_t smem = queue_smem_bytes<kW>();
  static std::once_flag once;
  static int per_sm = 0;
  std::call_once(once, [] {
    if (cudaFuncSetAttribute(blend_queue_kernel<kW>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) ==
        cudaSuccess)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, blend_queue_kernel<kW>, threads, smem);
  });
  if (per_sm <= 0) return false;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int items = tiles * (8 / kW);
  const int grid = std::min(items, sms * per_sm);
  BlendArgs b = a;
  b.total_tiles = tiles;  // the queue's length (a single-view call leaves it unset)
  blend_queue_kernel<kW><<<grid, threads, smem, stream>>>(b, map);
  return true;
}

}  // namespace

void launch_blend(const BlendArgs& a, cudaStream_t stream) {
  const int tiles = a.items ? a.total_tiles : ((a.W + kTile - 1) / kTile) * ((a.H + kTile - 1) / kTile);
  if (tiles <= 0) return;
  const int warps = tune_value(kTuneBlendWarps);
  const bool async = tune_value(kTuneBlendStage) == 1;
  const bool queue = tune_value(kTuneBlendQueue) == 1 && a.queue != nullptr;
  stage_begin(kStOther, stream);
  // with two CTAs per tile (or the queue) the tile's maxima combine with
  // atomics: clear first; the queue counter starts at zero
  tile_order_kernel<<<1, 1024, 0, stream>>>(a.ranges, nullptr, tiles, a.order,
                                            (warps == 4 || queue) ? a.tile_max : nullptr, queue ? a.queue : nullptr);
  stage_end(kStOther, stream, 1);
  stage_begin(kStBlend, stream);
  const bool queued = queue && (warps == 4 ? launch_queue<4>(a, tiles, stream) : launch_queue<8>(a, tiles, stream));
  if (!queued) {
    if (warps == 4 && async) blend_kernel<4, true><<<tiles * 2, 128, 0, stream>>>(a);
    else if (warps == 4) blend_kernel<4, false><<<tiles * 2, 128, 0, stream>>>(a);
    else if (async) blend_kernel<8, true><<<tiles, 256, 0, stream>>>(a);
    else blend_kernel<8, false><<<tiles, 256, 0, stream>>>(a);
  }
  stage_end(kStBlend, stream, 1);
  // the backward's order: by the largest contributor count the blend just found
  stage_begin(kStOther, stream);
  tile_order_kernel<<<1, 1024, 0, stream>>>(nullptr, a.tile_max, tiles, a.order_bwd, nullptr, nullptr);
  stage_end(kStOther, stream, 1);
}

}  // namespace w2w
