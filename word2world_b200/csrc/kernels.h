// Internal launch interfaces of the rasterizer kernels (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace w2w {

// One view of one scene in a batched call (device copy of the item table).
// Elements (the per-view copies of the scene's Gaussians), tiles and pixels of
// all items are laid out back to back: item v owns elements
// [elem_base, elem_base + P), global tile ids [tile_base, tile_base + tiles)
// and image pixels [pix_base, pix_base + W*H) of every per-pixel buffer.
struct BatchItem {
  const float* means3D;
  const float* scales;
  const float* rotations;
  const float* opacities;
  const float* shs;
  int P, M, degree, W, H, gw, tiles, pad0;
  float focal_x, tan_fovx, tan_fovy, scale_modifier;
  float h_x, h_y, pad1, pad2;  // W / (2 tan_fovx), H / (2 tan_fovy)
  float view[16], proj[16], campos[4], bg[4];
  uint32_t elem_base, tile_base;
  unsigned long long pix_base;
};

// Item owning global element (or tile) index i: the last item whose base is
// <= i (items with no elements share their successor's base and lose ties).
__device__ __forceinline__ int find_item_elem(const BatchItem* items, int n, uint32_t i) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].elem_base <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ int find_item_tile(const BatchItem* items, int n, uint32_t t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].tile_base <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

struct PreprocessArgs {
  int P, W, H, degree, M, compat_spill;
  const BatchItem* items;  // batched call: per-item scene and camera (then P = total elements); else null
  int num_items;
  uint32_t* item_end;      // batched call: end slot of each item's instances (written here)
  float focal_x;
  const float* view;
  const float* proj;
  const float* campos;
  const float* means3D;
  const float* scales;
  const float* rotations;
  const float* opacities;
  const float* shs;
  int* radii;
  GeomHeader* header;
  unsigned long long* scan_status;
  float* depth;
  uint8_t* clamped;
  float* means2D;
  float* cov3D;
  float* conic;
  float* rgb;
  uint32_t* tiles;
  uint32_t* offsets;
  uint32_t* rect;
  uint32_t* prev_reach;
  float* record;      // BlendRecord[P]
  float* bwd_record;  // BackwardRecord[P]
  // raw parameters (Renderer.render's, single-view calls only): when svec is
  // set, scales = exp(svec), rotations = normalize(quat), opacity =
  // sigmoid(logit) and the SH row is sh_dc followed by sh_ac, computed here
  // as the reference's torch preamble computes them
  const float *svec, *quat, *logit, *sh_dc, *sh_ac;
  uint32_t spin_limit = kSpinLimit;  // bounded waits (spin_limit())
  long long unpublished_tile = -1;   // fused scan: tile that skips publishing (tests; -1 = none)
};
void launch_preprocess(const PreprocessArgs& a, cudaStream_t stream);

struct DuplicateArgs {
  int P, gw;
  uint32_t R;
  const BatchItem* items;   // batched call (then per-item tile grids, tile bases and end slots)
  int num_items;
  const uint32_t* item_end;
  int key64;
  uint32_t depth_bits;
  const uint32_t* tiles;
  const uint32_t* offsets;
  const uint32_t* rect;
  const uint32_t* prev_reach;
  const float* depth;
  void* keys;
  uint32_t* vals;
  const uint32_t* n_dev = nullptr;  // planned render: the instance count in device memory (R is then the capacity)
};
void launch_duplicate(const DuplicateArgs& a, cudaStream_t stream);

// LSD radix sort of packed keys (uint32 or uint64) with uint32 values over
// key bits [begin_bit, begin_bit + bits); digits of sort_digit_bits(bits) <= 9
// bits (the last one narrower when bits is not a multiple), one onesweep launch
// per digit.  Pass p writes keys_out when (passes - 1 - p) is even, else keys_tmp,
// so the result lands in keys_out; keys_in must not be keys_out.
// `tile_hist` (may be null) receives a histogram of key >> tile_shift over
// num_tiles bins, and `ranges` (may be null) the per-bin [start, end).
struct SortArgs {
  long long n;
  int key64;
  int begin_bit;   // lowest key bit sorted on
  int bits;        // number of key bits sorted on, from begin_bit
  const void* keys_in;     // first pass reads here (may equal keys_tmp, never keys_out unless passes == 0)
  const uint32_t* vals_in;
  void* keys_out;          // the sorted result always lands here
  uint32_t* vals_out;
  void* keys_tmp;          // ping-pong partner
  uint32_t* vals_tmp;
  uint32_t* hist;        // [kMaxPasses * kMaxBins]
  uint32_t* status;      // [kMaxPasses * sort_tiles * kMaxBins]
  uint32_t* counters;    // [kMaxPasses]
  uint32_t* error;
  uint32_t spin_limit = kSpinLimit;  // bounded waits (spin_limit())
  long long unpublished_tile = -1;   // first pass: tile that skips publishing (tests; -1 = none)
  int match_rank = 0;  // 1: rank digits with match.any (keys whose warps hold few distinct digits)
  const uint32_t* n_dev = nullptr;  // planned render: the key count in device memory (n is then the capacity)
  int stage_hist = -1, stage_pass = -1;  // timing stages (default: the sort's own)
  int tile_shift;
  int num_tiles;
  uint32_t* tile_hist;
  uint2* ranges;
  // optional: one span to zero instead of the four buffers above (hist, the
  // used status words, counters, tile_hist), when the caller's layout makes
  // them contiguous
  void* clear_span;
  size_t clear_bytes;
};
int sort_passes(int bits);
long long sort_tile_keys(int key64);  // keys per onesweep tile for the key width
int sort_digit_bits(int bits);
void launch_sort(const SortArgs& a, cudaStream_t stream);
size_t sort_status_words(long long n);

struct BlendArgs {
  int W, H;
  const BatchItem* items;  // batched call (then per-item images packed at pix_base, 3 * pix_base for colour)
  int num_items, total_tiles;
  const uint2* ranges;
  const uint32_t* point_list;
  const float* record;
  uint32_t num_records;  // records (Gaussians, or batch elements); larger ids in the list are skipped
  uint8_t* mask_top;     // block masks for the backward passes (tile_walk.cuh BlockMasks), or null
  uint8_t* mask_bottom;
  const float* bg;
  float* out_color;
  float* out_depth;
  float* out_alpha;
  uint32_t* n_contrib;
  float* T_final;
  uint32_t* tile_max;
  uint32_t* order;      // tiles by decreasing list length (the blend's processing order)
  uint32_t* order_bwd;  // tiles by decreasing largest contributor count (the backward's)
  uint32_t* queue;      // the persistent blend's queue counter (cleared before its launch), or null
  uint32_t* error;      // error word for the persistent blend's bounded waits, or null
  uint32_t* masks_valid;  // the binning header's block-mask flag (the persistent blend clears it), or null
  uint32_t spin_limit = kSpinLimit;
};
void launch_blend(const BlendArgs& a, cudaStream_t stream);

// Backward.  grad_mode 0 = the reference's formulas, 1 = exact derivative.
struct BackwardArgs {
  int P, W, H, degree, M, grad_mode;
  const BatchItem* items;  // batched call (then P = total elements, per-item cameras and packed images)
  int num_items, total_tiles;
  float focal_x;           // exact mode (the forward's Jacobian focal)
  float h_x, h_y;          // reference mode: W/(2 tan_fovx), H/(2 tan_fovy)
  float tan_fovx, tan_fovy;
  float scale_modifier;
  const float* view;
  const float* proj;
  const float* campos;
  const float* bg;
  const float* means3D;
  const float* scales;
  const float* rotations;
  const float* shs;
  const int* radii;
  const float* cov3D;
  const uint8_t* clamped;
  const float* record;
  const float* bwd_record;
  const uint2* ranges;
  const uint32_t* point_list;
  const uint32_t* n_contrib;
  const uint32_t* tile_max;
  const uint32_t* order_bwd;  // tile order by largest contributor count (written by the blend)
  const uint8_t* mask_top;    // the blend's block masks (tile_walk.cuh BlockMasks); null: test each entry
  const uint8_t* mask_bottom;
  const uint32_t* masks_valid;
  int split;               // heaviest tiles whose walks are split over several CTAs (set at launch)
  const float* T_final;
  const float* out_alpha;
  const float* dL_dcolor;
  const float* dL_ddepth;
  const float* dL_dalpha;
  // accumulated by the per-pixel pass (zeroed by the caller)
  float* dL_dmean2D;   // [P,3]
  float* acc_cov;      // [P,4]: reference mode dL/dconic (x,y,_,w); exact mode dL/dcov2D (xx,xy,yy,_)
  float* dL_dopacity;  // [P]
  float* dL_dcolors;   // [P,3]
  float* acc_depth;    // [P]
  // written by the per-Gaussian pass
  float* dL_dmeans3D;
  float* dL_dcov3D;
  float* dL_dsh;
  float* dL_dscales;
  float* dL_drotations;
  // raw parameters (the fused-preamble path, reference mode, single view):
  // when svec is set the per-Gaussian pass activates svec / quat itself, reads
  // the SH rows from sh_dc and sh_ac, and writes the raw parameters' gradients
  // (dL_dscales then holds d/dsvec, dL_drotations d/dquat, dL_dopacity
  // d/dlogit, and dL_dsh_dc / dL_dsh_ac the SH rows split as the inputs)
  const float *svec, *quat, *logit, *sh_dc, *sh_ac;
  float *dL_dsh_dc, *dL_dsh_ac;
  // densification statistics accumulated by the per-Gaussian pass (or null):
  // for radius > 0, dens_counter += 1 and dens_accum += |dL/dmean2D[:2]|
  float *dens_accum, *dens_counter;
  // grouped per-Gaussian pass (batched calls): per-group sums over the
  // groups' items, tables laid out as w2w_group_sum's ([G + 1] row bases,
  // [G + 1] item pointers, item element bases), outputs [group_rows, ...]
  const uint32_t* group_tables;
  int num_groups;
  long long group_rows;
  float *g_means3D, *g_opacity, *g_scales, *g_rotations, *g_sh;
};
void launch_backward_render(const BackwardArgs& a, cudaStream_t stream);
void launch_backward_gaussians(const BackwardArgs& a, cudaStream_t stream);
void launch_backward_groups(const BackwardArgs& a, cudaStream_t stream);

// Instance binning from depth-ordered Gaussians (binning.cu): a single-view
// call's sorted instance list and tile ranges without key emission or an
// R-sized sort.  `order` is the Gaussians sorted stably by their depth bits,
// `dprefix` the exclusive prefix (P + 1 entries) of their owned instance
// counts in that order.
struct BinArgs {
  int P;
  uint32_t R;
  int gw, T;
  int key64;
  uint32_t depth_bits;
  const uint32_t* order;       // [P]
  const uint32_t* dprefix;     // [P + 1]
  const uint32_t* tiles;       // geometry state: allocation counts, inclusive offsets, emission rectangles,
  const uint32_t* offsets;     // earlier Gaussians' reach and depths
  const uint32_t* rect;
  const uint32_t* prev_reach;
  const float* depth;
  uint32_t* warp_start;        // [ceil(R / kBinShare)] depth-order index at each warp share's start
  uint32_t* counts;            // [ceil(R / kBinChunk)][T]: chunk counts, then each chunk's first slot per tile
  uint32_t* tile_total;        // [T]
  uint2* ranges;               // [T]
  void* keys;                  // sorted packed keys (tile << depth_bits | low depth bits), 32 or 64 bit
  uint32_t* vals;              // sorted Gaussian ids (the point list)
  uint32_t* error;
};
size_t bin_smem_bytes(int tiles, int key64);
void launch_iota(uint32_t* out, int n, cudaStream_t stream);
void launch_owned_counts(const BinArgs& a, uint32_t* count, cudaStream_t stream);
void launch_binning(const BinArgs& a, cudaStream_t stream);

}  // namespace w2w

namespace w2w {
// Launch accounting / stage timing (timing.cu).  Stages bracket the launches
// of one logical step; `kernels` is how many kernels the stage launched.
enum Stage {
  kStPreprocess, kStDuplicate, kStSortHist, kStSortPass, kStBlend, kStBwdRender, kStBwdGaussians, kStScan,
  kStOther, kStDepthSort, kStBinning, kNumStages
};
void stage_begin(int stage, cudaStream_t s);
void stage_end(int stage, cudaStream_t s, int kernels);

// Activation preamble of Renderer.render (activate.cu).
struct ActivateArgs {
  long long P;
  int K;  // rest SH coefficients per Gaussian (sh_ac is [P, K, 3])
  const float *opacity_logit, *svec, *quat, *sh_dc, *sh_ac;
  float *opacity, *scales, *rotations, *shs;
};
struct ActivateBackwardArgs {
  long long P;
  int K;
  const float *g_opacity, *g_scales, *g_rotations, *g_shs;  // gradients of the activated tensors
  const float *opacity, *scales, *quat;                      // activated opacity and scales (or null), raw quaternion
  float *d_opacity_logit, *d_svec, *d_quat, *d_sh_dc, *d_sh_ac;
  const float *opacity_logit, *svec;                         // raw, read when opacity / scales are null
};
void launch_activate(const ActivateArgs& a, cudaStream_t stream);
void launch_activate_backward(const ActivateBackwardArgs& a, cudaStream_t stream);
// Voxel occupancy field (voxel.cu).
struct VoxelArgs {
  int P, R, B;
  float bs, relax;  // block side 2 / B, growth of each block per side in block sides
  const float *means, *covs, *opacities;
  float4* rec;        // [3P] per Gaussian: mean + opacity, inverse covariance
  uint32_t* count;    // [P] blocks each Gaussian is binned into
  const uint32_t* offsets;  // [P] exclusive scan of count
  uint32_t* keys;     // [pairs] block ids
  uint32_t* vals;     // [pairs] Gaussian ids
  float* occ;         // [R^3], x fastest
};
void launch_voxel_prepare(const VoxelArgs& a, cudaStream_t stream);
void launch_voxel_emit(const VoxelArgs& a, cudaStream_t stream);
void launch_voxel_field(const VoxelArgs& a, const uint32_t* list, const uint2* ranges, cudaStream_t stream);
// Per-group sums of element rows (groupsum.cu).  tables: group_base[G + 1]
// (first output row of each group; the last entry is the total),
// item_ptr[G + 1] (CSR into item_elem), item_elem[num_items] (each item's
// first element row).
void launch_group_sum(const float* src, int width, int num_groups, const uint32_t* tables, int num_items,
                      float* dst, long long total_rows, cudaStream_t stream);
// Densification statistics (densify.cu).
void launch_densify_stats(long long P, const float* dL_dmeans2D, const int* radii, float* accum, float* counter,
                          cudaStream_t stream);

size_t scan_status_words(long long n);
// Bounded device waits.  spin_limit(): the iteration limit of every lookback
// wait (kSpinLimit unless a test lowered it).  unpublished_tile(stage): a
// tile of that stage whose CTA skips publishing its status, so that the waits
// behind it run out and report kErrTimeout (tests only; -1 = none).  Both are
// host-side settings read when a kernel is launched.
enum WaitStage { kWaitScan = 0, kWaitSort = 1, kWaitPreprocess = 2, kNumWaitStages = 3 };
uint32_t spin_limit();
long long unpublished_tile(int stage);

// Run-time launch shapes chosen by the autotuner (w2w_tune_set): warps per
// blend CTA (4: two CTAs per tile, 8: one), how many of the heaviest tiles the
// per-pixel backward splits (in quarters of the SM count) and into how many
// segments.  None of them changes a result beyond the order of float atomic
// additions.
// The fourth knob picks how a single-view call builds its sorted list: 0 key
// emission + radix sort (duplicate.cu, sort.cu), 1 binning from the
// depth-ordered Gaussians (binning.cu); both give the same list.
enum TuneKnob {
  kTuneBlendWarps = 0,
  kTuneBwdSplit = 1,
  kTuneBwdWays = 2,
  kTuneBinning = 3,
  kTuneBlendQueue = 4,
  kTunePreBlocks = 5,
  kTunePlanned = 6,
  kTuneBlendStage = 7,
  kNumTuneKnobs = 8
};
int tune_value(int knob);

size_t scan_scratch_bytes(long long n);
void launch_scan(const uint32_t* in, uint32_t* out, long long n, int exclusive, void* scratch, cudaStream_t stream);
long long scan_noalloc_max();
void* scan_noalloc_scratch(int* status);
}  // namespace w2w
