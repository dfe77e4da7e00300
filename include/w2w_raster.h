/*
 * w2w_raster.h -- C ABI of the sm_100a Gaussian rasterizer.
 *
 * Drop-in replacement for the rasterizer path of Word2World's
 * cudaForwardBackwardRenderer extension: the forward is
 * RasterizeGaussiansCUDA / gaussianForwardPass, the backward
 * RasterizeGaussiansBackwardCUDA / backward.  Plain C types only: device
 * pointers, sizes and a CUDA stream.  Every device buffer -- inputs, outputs
 * and the three opaque state buffers -- is allocated by the caller; the
 * library never allocates device memory and never synchronises the device
 * except where stated (w2w_forward_geometry reads one 16-byte header back to
 * the host, as the reference reads R back, prepareSort.cu:382-387).
 *
 * Conventions (identical to the reference):
 *   means3D [P,3], scales [P,3] (activated), rotations [P,4] (w,x,y,z,
 *   normalised), opacities [P] (activated), shs [P,M,3] (RGB innermost);
 *   viewmatrix / projmatrix: 16 floats read column-major (the transposed
 *   matrices the reference trainer passes); campos = minus the camera
 *   position; image outputs are CHW float32; radii int32[P].
 *
 * Status codes: 0 ok, otherwise a W2W_ERR_* value (w2w_status_string()).
 *
 * Device-side failures.  The sort's and the scans' single-pass lookbacks wait
 * on their predecessors with an iteration limit; a wait that runs out, or an
 * instance count beyond the state's capacity, sets bits in a device error
 * word instead of hanging or faulting.  w2w_forward_geometry(_raw) and
 * w2w_batch_forward_geometry read their word back (they synchronise anyway)
 * and return W2W_ERR_TIMEOUT / W2W_ERR_CAPACITY.  The other entry points with
 * such waits (w2w_forward_render, w2w_batch_forward_render, w2w_sort_pairs_u64,
 * w2w_scan_u32, w2w_scan_u32_noalloc) return once their work is enqueued, so
 * by default their status covers the launches only and the word is left for
 * the caller: w2w_state_error(binning_state, 1, stream) after a render,
 * w2w_scratch_error(scratch, stream) after a sort or scan,
 * w2w_scan_noalloc_error(stream) after the allocation-free scan.  With
 * w2w_set_error_check(1) those entry points synchronise their stream before
 * returning and return W2W_ERR_TIMEOUT / W2W_ERR_CAPACITY themselves.
 */
#ifndef W2W_RASTER_H
#define W2W_RASTER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* w2w_stream_t; /* a cudaStream_t; NULL = legacy default stream */

enum {
    W2W_OK = 0,
    W2W_ERR_INVALID = 1,   /* bad argument (null pointer, negative size, mismatched state) */
    W2W_ERR_CUDA = 2,      /* a CUDA launch or runtime call failed */
    W2W_ERR_CAPACITY = 3,  /* instance count exceeds what the state buffer was sized for */
    W2W_ERR_TIMEOUT = 4,   /* a bounded device-side wait gave up (results invalid) */
    W2W_ERR_SCRATCH = 5    /* scratch buffer smaller than required */
};

/* Camera and image settings.  Pointer fields are device pointers. */
typedef struct {
    int P;                   /* number of Gaussians */
    int degree;              /* SH degree evaluated (0..3) */
    int M;                   /* SH coefficients stored per Gaussian */
    int width, height;       /* image size (the reference fixes 800x800) */
    float focal_x;           /* forward Jacobian focal length, pixels (both axes, as the reference) */
    float tan_fovx, tan_fovy;/* backward: focal = width / (2 tan_fovx) (gradientPass.cu:119-120) */
    float scale_modifier;    /* backward scale multiplier (backward.cu:463) */
    int compat_spill;        /* 1: the reference's key-emission rectangle (see w2w_forward_render) */
    const float* viewmatrix; /* [16] */
    const float* projmatrix; /* [16] */
    const float* campos;     /* [3] */
    const float* background; /* [3]; the reference forward hard-codes white */
} w2w_settings;

/* Returned by the geometry phase; sizes the binning state and the sort. */
typedef struct {
    long long num_rendered;   /* R: sum of tiles touched (the reference's num_rendered) */
    uint32_t depth_min_bits;  /* range of the depth bits of Gaussians that emit keys */
    uint32_t depth_max_bits;
    uint32_t error;           /* device error bits (0 = none) */
    uint32_t reserved;        /* bit 0: the geometry phase prepared the depth-ordered binning */
} w2w_geometry_info;

int w2w_version(void);
const char* w2w_status_string(int status);

/* Error-word checking of the entry points that return before their device
 * waits finish (see above): 0 = leave the word for the caller (default),
 * 1 = synchronise the stream and return the word's status.  Process-wide;
 * returns the previous mode.  No counterpart in the reference, which checks
 * nothing (rasterize_points.cu). */
int w2w_set_error_check(int mode);
/* Status of the error word of a sort or scan scratch buffer (the 32-bit word
 * at byte 4 of every stage scratch); synchronises `stream`. */
int w2w_scratch_error(const void* scratch, w2w_stream_t stream);

/* ---- state buffer sizes (bytes; caller allocates device memory) ------------
 * Replace the resize callbacks of rasterize_points.cu:81-87 and the
 * cudaMalloc'd temporaries of gaussianRasterizer.cu:209-212. */
size_t w2w_geometry_state_bytes(int P);
size_t w2w_image_state_bytes(int width, int height);
size_t w2w_binning_state_bytes(long long num_rendered, int width, int height);
size_t w2w_backward_scratch_bytes(int P);

/* Offsets (bytes) of named arrays inside the state buffers, for inspection
 * and parity tests.  Returns (size_t)-1 for an unknown name.
 *   geometry: "depth","clamped","means2D","cov3D","conic_opacity","rgb",
 *             "tiles_touched","offsets","rect","prev_reach","record","header"
 *   image:    "n_contrib","ranges","T_final","tile_max"
 *   binning:  "header","keys_a","keys_b","vals_a","vals_b" */
size_t w2w_geometry_offset(int P, const char* name);
size_t w2w_image_offset(int width, int height, const char* name);
size_t w2w_binning_offset(long long num_rendered, int width, int height, const char* name);

/* ---- forward --------------------------------------------------------------
 * Phase 1 (replaces projection.cu ProjectG, ADRculling.cu tileCulling,
 * gaussianForwardPass.cu calcColour and the scan of gaussianRasterizer.cu:233,
 * i.e. gaussianForwardPass, gaussianRasterizer.cu:118-237): one fused kernel.  Writes radii and
 * the geometry state, then reads the instance count and depth-bit range back
 * into *info (synchronising `stream` once).  When the "binning" tuning knob
 * selects the depth-ordered binning and the image has at most 4096 tiles, it
 * then enqueues the per-Gaussian half of that binning (the Gaussians sorted
 * stably by depth bits, and the prefix of their owned instance counts in that
 * order) into the geometry state and sets bit 0 of info->reserved. */
int w2w_forward_geometry(const w2w_settings* s, const float* means3D, const float* scales,
                         const float* rotations, const float* opacities, const float* shs,
                         int* radii, void* geom_state, w2w_geometry_info* info, w2w_stream_t stream);

/* Phase 2 (replaces prepareAndSort, prepareSort.cu:362-435, gaussianTiles,
 * gaussianTiles.cu:6-33, and pixelGaussiansFull, pixelGaussiansFull.cu:99-122):
 * the sorted instance list and tile ranges, then blending.  binning_state
 * must be w2w_binning_state_bytes(info->num_rendered, W, H) long.  With bit
 * 0 of info->reserved set, every instance is placed once, by tile, walking the
 * Gaussians in the depth order phase 1 prepared (a counting sort whose keys
 * are generated, not stored); otherwise key emission and an onesweep radix
 * sort.  Either way the list is the reference's: sorted by tile, then
 * depth bits, ties in slot order.  The sorted keys are kept in the binning
 * state, packed: only the bits in which keys can differ (tile bits and the
 * low depth bits below the depths' common prefix), in 32 bits when they fit;
 * the order equals that of the reference's 64-bit (tile << 32 | depth bits)
 * keys.  With
 * compat_spill=1 keys are emitted over the reference's emission rectangle;
 * where that writes past a Gaussian's allocation the lowest-index writer owns
 * each slot (the reference leaves this to a race).  Outputs: color [3,H,W],
 * depth [1,H,W], alpha [1,H,W] (sum of alpha*T, as the reference).  The
 * sort's error word is the binning state's (w2w_state_error(binning_state,
 * 1, ...)), returned here in checked mode (w2w_set_error_check). */
int w2w_forward_render(const w2w_settings* s, const void* geom_state, const w2w_geometry_info* info,
                       void* binning_state, void* image_state, float* out_color, float* out_depth,
                       float* out_alpha, w2w_stream_t stream);

/* ---- planned forward (no counterpart in the reference) ----------------------
 * The reference reads R back before it can size and launch its sort
 * (prepareSort.cu:382-387), and so does the pair above; a host that renders
 * many views waits there once per view.  The planned pair launches the whole
 * forward first and reads R afterwards:
 *   1. w2w_forward_geometry(_raw)_async: the projection pass, then a copy of
 *      the geometry header's first 16 bytes into `header_host` (pinned host
 *      memory the caller owns); nothing is synchronised.
 *   2. w2w_forward_render_planned with a capacity C and a number of key depth
 *      bits from earlier views of the same size (w2w_planned_capacity of the
 *      largest R seen; the most depth bits any of them needed), into a binning
 *      state of w2w_binning_state_bytes(C, W, H) bytes.  The kernels read R
 *      from device memory.
 *   3. Once the header copy has landed (an event recorded after step 1),
 *      w2w_geometry_info_from_header decodes it.  If R > C or the view needs
 *      more depth bits than were given (w2w_depth_bits_needed), the planned
 *      launches processed no instance: render again with w2w_forward_render
 *      and a binning state sized for R.  Otherwise the result is the exact
 *      plan's, bit for bit.
 * A planned binning state is laid out for C: functions that take a binning
 * state and a count (w2w_backward, w2w_backward_raw, w2w_binning_offset)
 * take C there, and w2w_binning_layout_count recovers it from R and the
 * state's size.  Capacities are multiples of W2W_PLAN_QUANTUM. */
#define W2W_PLAN_QUANTUM 65536LL
int w2w_forward_geometry_async(const w2w_settings* s, const float* means3D, const float* scales,
                               const float* rotations, const float* opacities, const float* shs, int* radii,
                               void* geom_state, void* header_host, w2w_stream_t stream);
int w2w_forward_geometry_raw_async(const w2w_settings* s, const float* means3D, const float* svec,
                                   const float* quaternion, const float* opacity_logit, const float* sh_dc,
                                   const float* sh_ac, int* radii, void* geom_state, void* header_host,
                                   w2w_stream_t stream);
/* Decodes a header copied by the async geometry calls; returns its error status. */
int w2w_geometry_info_from_header(const void* header_host, w2w_geometry_info* info);
/* Depth bits the view's keys need (the span of its depths' bit patterns). */
int w2w_depth_bits_needed(const w2w_geometry_info* info);
/* Capacity for a planned render sized from an instance count: +25 %, rounded up
 * to a multiple of W2W_PLAN_QUANTUM. */
long long w2w_planned_capacity(long long num_rendered);
int w2w_forward_render_planned(const w2w_settings* s, const void* geom_state, long long capacity, int depth_bits,
                               void* binning_state, void* image_state, float* out_color, float* out_depth,
                               float* out_alpha, w2w_stream_t stream);
/* 1 when a planned render did not fit its plan (the header's flag; synchronises `stream`). */
int w2w_binning_replanned(const void* binning_state, w2w_stream_t stream);
/* The instance count a binning state of `state_bytes` bytes is laid out for:
 * num_rendered itself, or a planned render's capacity; -1 if neither. */
long long w2w_binning_layout_count(long long num_rendered, size_t state_bytes, int width, int height);

/* Device error word of a geometry / binning state (synchronises `stream`). */
int w2w_state_error(const void* state, int which /* 0 geometry, 1 binning */, w2w_stream_t stream);

/* ---- backward -------------------------------------------------------------
 * Replaces RasterizeGaussiansBackwardCUDA (rasterize_points.cu:158-246) and
 * backward (gradientPass.cu:26-207).  grad_mode 0 = the reference's formulas,
 * 1 = the exact derivative of the forward.  All eight outputs are fully
 * written (no pre-zeroing needed); dL_dmeans2D is [P,3] with the third
 * component 0; dL_dcov3D is [P,6]; dL_dsh is [P,M,3].  dL_ddepth and
 * dL_dalpha may be NULL: no loss on depth / alpha (the reference always
 * passes buffers, zero-filled by autograd when unused). */
int w2w_backward(const w2w_settings* s, const float* means3D, const float* scales, const float* rotations,
                 const float* shs, const int* radii, const void* geom_state,
                 long long num_rendered, const void* binning_state, const void* image_state,
                 const float* out_alpha, const float* dL_dcolor, const float* dL_ddepth,
                 const float* dL_dalpha, int grad_mode, void* scratch, size_t scratch_bytes,
                 float* dL_dmeans2D, float* dL_dcolors, float* dL_dopacity, float* dL_dmeans3D,
                 float* dL_dcov3D, float* dL_dsh, float* dL_dscales, float* dL_drotations,
                 w2w_stream_t stream);

/* ---- stages ---------------------------------------------------------------
 * Stable sort of (uint64 key, uint32 value) pairs on key bits
 * [begin_bit, end_bit).  Replaces radix_sort_2bit_coalesced
 * (prepareSort.cu:303-360).  keys_out/vals_out may not alias the inputs. */
size_t w2w_sort_scratch_bytes(long long n);
int w2w_sort_pairs_u64(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out,
                       uint32_t* vals_out, long long n, int begin_bit, int end_bit, void* scratch,
                       size_t scratch_bytes, w2w_stream_t stream);

/* Inclusive / exclusive scan of uint32 values (single-pass decoupled
 * lookback).  Replaces kogge_stone_inclusive_scan_shared_memory
 * (gaussianRasterizer.cu:77-117). */
size_t w2w_scan_scratch_bytes(long long n);
int w2w_scan_u32(const uint32_t* in, uint32_t* out, long long n, int exclusive, void* scratch,
                 size_t scratch_bytes, w2w_stream_t stream);

/* Allocation-free variant of w2w_scan_u32.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc or hand the library a scratch
 * buffer: hosts whose device memory is owned by another allocator (a JVM or
 * Go runtime reaching the library through JNI / cgo, a plugin host with its
 * own pool) and hot loops in which an allocation's implicit device
 * synchronisation is not acceptable.  The lookback scratch lives in a fixed
 * device array inside the library (about 32 KB, held by every GPU that loads
 * the library until the process exits), so the caller passes only the input
 * and output.  At most W2W_SCAN_NOALLOC_MAX elements; larger n returns
 * W2W_ERR_CAPACITY without launching anything.  Every call looks up the
 * array's address in the caller's current CUDA context (a host-side lookup,
 * right for any context, including one re-created after cudaDeviceReset); the
 * first call in a context also loads the library's device code into it, so
 * make that first call before any stream capture on the device.  All calls share the one array and each clears the parts it needs
 * before use; calls that overlap on the GPU (other streams, other threads)
 * race on it, so serialise them.  Never calls cudaMalloc or cudaFree. */
#define W2W_SCAN_NOALLOC_MAX (1LL << 24)
int w2w_scan_u32_noalloc(const uint32_t* in, uint32_t* out, long long n, int exclusive, w2w_stream_t stream);
/* Status of the allocation-free scan's error word (inside the library's
 * fixed array): W2W_ERR_TIMEOUT if a lookback wait of the last call ran out
 * (its output is then invalid).  Synchronises `stream`. */
int w2w_scan_noalloc_error(w2w_stream_t stream);

/* Renderer.render's path on its raw parameters (Renderer.py:164-192): the
 * activation preamble (sigmoid opacity, exp scales, normalised quaternion,
 * concatenated SH; bit-identical to the reference's torch operations) runs
 * inside the projection pass, so the activated tensors never exist.
 * w2w_forward_geometry_raw takes mean [P,3], svec [P,3], quaternion [P,4],
 * opacity logits [P], sh_dc [P,1,3] and sh_ac [P,M-1,3] (1 <= M <= 16) and is
 * otherwise w2w_forward_geometry (w2w_forward_render follows unchanged).
 * w2w_backward_raw is w2w_backward in reference mode whose per-Gaussian pass
 * chains through the activations: it writes d/dsvec, d/dquaternion,
 * d/dlogit and the SH gradient split as sh_dc / sh_ac. */
int w2w_forward_geometry_raw(const w2w_settings* s, const float* means3D, const float* svec, const float* quaternion,
                             const float* opacity_logit, const float* sh_dc, const float* sh_ac, int* radii,
                             void* geom_state, w2w_geometry_info* info, w2w_stream_t stream);
int w2w_backward_raw(const w2w_settings* s, const float* means3D, const float* svec, const float* quaternion,
                     const float* opacity_logit, const float* sh_dc, const float* sh_ac, const int* radii,
                     const void* geom_state, long long num_rendered, const void* binning_state,
                     const void* image_state, const float* out_alpha, const float* dL_dcolor, const float* dL_ddepth,
                     const float* dL_dalpha, void* scratch, size_t scratch_bytes, float* dL_dmeans2D,
                     float* dL_dcolors, float* dL_dopacity_logit, float* dL_dmeans3D, float* dL_dcov3D,
                     float* dL_dsh_dc, float* dL_dsh_ac, float* dL_dsvec, float* dL_dquaternion,
                     w2w_stream_t stream);
/* w2w_backward_raw that also accumulates the training loop's densification
 * statistics (gaussians_handler.py:116-118, which the reference computes
 * after the backward with boolean-mask indexing) in its per-Gaussian pass:
 * for every Gaussian with radius > 0, dens_counter[i] += 1 and dens_accum[i]
 * += |dL/dmean2D[i, 0:2]| (both [P], updated in place with atomics, so views
 * back-propagated on concurrent streams may share them; both null: none). */
int w2w_backward_raw_densify(const w2w_settings* s, const float* means3D, const float* svec,
                             const float* quaternion, const float* opacity_logit, const float* sh_dc,
                             const float* sh_ac, const int* radii, const void* geom_state, long long num_rendered,
                             const void* binning_state, const void* image_state, const float* out_alpha,
                             const float* dL_dcolor, const float* dL_ddepth, const float* dL_dalpha, void* scratch,
                             size_t scratch_bytes, float* dL_dmeans2D, float* dL_dcolors, float* dL_dopacity_logit,
                             float* dL_dmeans3D, float* dL_dcov3D, float* dL_dsh_dc, float* dL_dsh_ac,
                             float* dL_dsvec, float* dL_dquaternion, float* dens_accum, float* dens_counter,
                             w2w_stream_t stream);

/* The activation preamble of Renderer.render (Renderer.py:164-167) in one
 * pass: opacity = sigmoid(logit) [P], scales = exp(svec) [P,3], rotations =
 * normalize(quaternion) [P,4], shs = cat(sh_dc [P,1,3], sh_ac [P,K,3]) [P,K+1,3];
 * bit-identical to the reference's torch operations.  The backward maps the
 * activated tensors' gradients to the raw parameters' (quaternion: the raw
 * one; opacity and scales: the activated ones). */
int w2w_activate_forward(long long P, int K, const float* opacity_logit, const float* svec, const float* quaternion,
                         const float* sh_dc, const float* sh_ac, float* opacity, float* scales, float* rotations,
                         float* shs, w2w_stream_t stream);
int w2w_activate_backward(long long P, int K, const float* g_opacity, const float* g_scales,
                          const float* g_rotations, const float* g_shs, const float* opacity, const float* scales,
                          const float* quaternion, float* d_opacity_logit, float* d_svec, float* d_quaternion,
                          float* d_sh_dc, float* d_sh_ac, w2w_stream_t stream);

/* Voxel occupancy field for mesh extraction (compute_voxel_field.cu:25-124):
 * occ[i + R (j + R k)] = sum over the Gaussians whose mean lies in voxel
 * (i, j, k)'s block (B^3 blocks over [-1, 1]^3, grown by relax_ratio block
 * sides) of opacity * exp(-1/2 d^T Sigma^-1 d), Sigma given by its upper
 * triangle (xx, xy, xz, yy, yz, zz).  Each Gaussian is binned once into the
 * blocks that hold its mean instead of being tested by every voxel.
 * w2w_voxel_field takes device pointers and enqueues on `stream` (its
 * temporaries come from the stream-ordered allocator; it synchronises the
 * stream once, to size them); w2w_compute_voxel_field is the reference's
 * entry point (compute_voxel_field_cuda), with host pointers.  2 <= R <= 2048,
 * 1 <= B <= 1000, 0 <= relax_ratio <= 64; non-finite means are not supported. */
int w2w_voxel_field(const float* means, const float* covs, const float* opacities, int n, int resolution,
                    int num_blocks, float relax_ratio, float* occ, w2w_stream_t stream);
int w2w_compute_voxel_field(float* h_occ, const float* h_means, const float* h_covs, const float* h_opacities,
                            int n, int resolution, int num_blocks, float relax_ratio);

/* Per-group sums of a batched call's per-element gradient rows (width floats
 * per row): output row r of group g = the sum over g's items, in list order,
 * of row (item's first element + r).  `tables` (device) holds group_base[G+1]
 * (the groups' first output rows, then the total), item_ptr[G+1] (CSR offsets
 * into the next array) and item_elem[num_items] (each item's first element
 * row).  No counterpart in the reference, which renders one view per call. */
int w2w_group_sum(const float* src, int width, int num_groups, const uint32_t* tables, int num_items, float* dst,
                  long long total_rows, w2w_stream_t stream);

/* Densification statistics of the training loop (gaussians_handler.py:116-118):
 * for every Gaussian with radii[i] > 0, counter[i] += 1 and accum[i] +=
 * |dL/dmean2D[i, 0:2]| (dL_dmeans2D [P,3], accum and counter [P], updated in
 * place), in one pass and without a host synchronisation. */
int w2w_densification_stats(long long P, const float* dL_dmeans2D, const int* radii, float* accum, float* counter,
                            w2w_stream_t stream);

/* Per-tile [start, end) from sorted keys whose tile id is key >> tile_shift
 * (gaussianTiles.cu:6-33); tiles without entries get (0, 0). */
int w2w_tile_ranges(const uint64_t* sorted_keys, long long n, int tile_shift, uint32_t* ranges,
                    int num_tiles, w2w_stream_t stream);

/* Blend from a given sorted Gaussian list and tile ranges (the reference's
 * pixelGaussiansFull on its own inputs), writing the image state fields
 * ranges (a copy), n_contrib, T_final and tile_max and the three images. */
int w2w_blend(const w2w_settings* s, const void* geom_state, const uint32_t* ranges,
              const uint32_t* point_list, void* image_state, float* out_color, float* out_depth,
              float* out_alpha, w2w_stream_t stream);

/* Copy the sorted keys, expanded to the reference's 64-bit layout
 * (tile << 32 | depth bits), out of a binning state. */
int w2w_binning_keys64(const void* binning_state, long long num_rendered, int width, int height,
                       uint64_t* out, w2w_stream_t stream);
/* The same for a binning state laid out for layout_count >= num_rendered instances. */
int w2w_binning_keys64_layout(const void* binning_state, long long num_rendered, long long layout_count, int width,
                              int height, uint64_t* out, w2w_stream_t stream);

/* ---- batched calls ----------------------------------------------------------
 * Many views of many scenes rendered and back-propagated with one launch per
 * stage.  No counterpart in the reference, whose call renders one view; each
 * item's results equal the single-view entry points' on the same inputs
 * (bit-identical images and per-tile lists; gradients up to float atomic
 * order).  Item v's per-view element copies of its scene's Gaussians, tiles
 * and pixels follow those of items 0..v-1: per-element arrays ([E] = sum of
 * P) hold item v's Gaussians at [sum_{u<v} P_u, + P_v); images are packed,
 * item v's colour as its own [3, H_v, W_v] block at 3 * (sum_{u<v} W_u H_u)
 * and depth / alpha at sum_{u<v} W_u H_u.  All items share one M. */
typedef struct {
    const float* means3D;    /* device pointers into the item's scene, as in w2w_forward_geometry */
    const float* scales;
    const float* rotations;
    const float* opacities;
    const float* shs;
    int P, M, degree, width, height;
    float focal_x, tan_fovx, tan_fovy, scale_modifier;
    float viewmatrix[16];    /* by value (host memory), column-major as in w2w_settings */
    float projmatrix[16];
    float campos[3];
    float background[3];
} w2w_batch_item;

size_t w2w_batch_geometry_state_bytes(const w2w_batch_item* items, int n);
size_t w2w_batch_image_state_bytes(const w2w_batch_item* items, int n);
size_t w2w_batch_binning_state_bytes(long long num_rendered, const w2w_batch_item* items, int n);
size_t w2w_batch_backward_scratch_bytes(const w2w_batch_item* items, int n);
/* Projection, colour, culling and the instance scan of every item (radii [E]).
 * Copies the item table into the geometry state. */
int w2w_batch_forward_geometry(const w2w_batch_item* items, int n, int compat_spill, int* radii,
                               void* geom_state, w2w_geometry_info* info, w2w_stream_t stream);
/* Keys (global tile, depth) of all items, one sort, one blend launch. */
int w2w_batch_forward_render(const w2w_batch_item* items, int n, const void* geom_state,
                             const w2w_geometry_info* info, void* binning_state, void* image_state,
                             float* out_color, float* out_depth, float* out_alpha, w2w_stream_t stream);
/* Per-element gradients ([E, ...]; a scene's gradient is the sum over its
 * items' element ranges).  dL_ddepth and dL_dalpha may be NULL, as in
 * w2w_backward (no loss on depth / alpha). */
int w2w_batch_backward(const w2w_batch_item* items, int n, const void* geom_state, long long num_rendered,
                       const void* binning_state, const void* image_state, const int* radii,
                       const float* out_alpha, const float* dL_dcolor, const float* dL_ddepth,
                       const float* dL_dalpha, int grad_mode, void* scratch, size_t scratch_bytes,
                       float* dL_dmeans2D, float* dL_dcolors, float* dL_dopacity, float* dL_dmeans3D,
                       float* dL_dcov3D, float* dL_dsh, float* dL_dscales, float* dL_drotations,
                       w2w_stream_t stream);
/* The same backward with the per-Gaussian pass summing each group's items
 * (a scene's views, or a serving request's) itself: in place of the five
 * per-element parameter gradients and a w2w_group_sum per tensor, it writes
 * the per-group sums g_means3D [rows,3], g_opacity [rows], g_scales [rows,3],
 * g_rotations [rows,4] and g_sh [rows,M,3] directly, each sum over the
 * group's items in table order (w2w_group_sum's order; equal to its sums up to
 * a few ulps of fused multiply-adds).
 * group_tables is device memory in w2w_group_sum's layout; dL_dmeans2D,
 * dL_dcolors and dL_dopacity stay per element ([E, ...]).  The reference has
 * one call per view and sums views in torch's autograd (GaussianTrainer.py:47-88). */
int w2w_batch_backward_grouped(const w2w_batch_item* items, int n, const void* geom_state,
                               long long num_rendered, const void* binning_state, const void* image_state,
                               const int* radii, const float* out_alpha, const float* dL_dcolor,
                               const float* dL_ddepth, const float* dL_dalpha, int grad_mode, void* scratch,
                               size_t scratch_bytes, const uint32_t* group_tables, int num_groups,
                               long long group_rows, float* dL_dmeans2D, float* dL_dcolors, float* dL_dopacity,
                               float* g_means3D, float* g_opacity, float* g_scales, float* g_rotations,
                               float* g_sh, w2w_stream_t stream);
/* The grouped per-Gaussian pass alone, over the per-element accumulators a
 * previous w2w_batch_backward or w2w_batch_backward_grouped call on the same
 * state left in `scratch` and in dL_dmeans2D, dL_dcolors and dL_dopacity
 * (for instance, per-element gradients first, then the group sums). */
int w2w_batch_gaussians_grouped(const w2w_batch_item* items, int n, const void* geom_state, const int* radii,
                                int grad_mode, void* scratch, size_t scratch_bytes, const float* dL_dmeans2D,
                                const float* dL_dcolors, const float* dL_dopacity, const uint32_t* group_tables,
                                int num_groups, long long group_rows, float* g_means3D, float* g_opacity,
                                float* g_scales, float* g_rotations, float* g_sh, w2w_stream_t stream);

/* ---- observability ---------------------------------------------------------
 * Number of kernels the library has launched in this process. */
unsigned long long w2w_launch_count(void);
/* Per-stage device timing with CUDA events recorded on the launching stream
 * (off by default).  w2w_stage_timing returns the previous setting.
 * w2w_stage_times waits for the recorded events, writes accumulated
 * milliseconds and kernel launches per stage (w2w_stage_count() stages,
 * named by w2w_stage_name) and resets the accumulators. */
int w2w_stage_timing(int enable);
/* The same for the stages whose bit is set in `mask` (bit i: stage i, named by
 * w2w_stage_name); returns the previous mask.  Timing fewer stages keeps the
 * host work between launches, and so the device's idle gaps, smaller. */
unsigned w2w_stage_timing_mask(unsigned mask);
int w2w_stage_count(void);
const char* w2w_stage_name(int stage);
int w2w_stage_times(double* ms, long long* launches, int max_stages);
/* Arithmetic throughput probe (no counterpart in the reference): kind 0 runs
 * FP32 fused multiply-adds, kind 1 SFU base-2 exponentials, on `blocks` CTAs
 * of 256 threads, `iters` steps of 8 independent chains per thread.  *ops
 * receives the instruction count (blocks * 256 * iters * 8); time the launch
 * with events on `stream` to get the GPU's issue rate, the denominator of the
 * per-pixel passes' roofline.  `out` (>= 256 floats, device) is never
 * written in practice; it keeps the chains from being optimised away. */
int w2w_throughput_probe(int kind, long long iters, int blocks, float* out, long long* ops, w2w_stream_t stream);

/* ---- launch-shape tuning -----------------------------------------------------
 * Process-wide knobs read at every launch, set by the autotuner
 * (word2world_b200/autotune.py) from timings of the caller's workload.  No
 * counterpart in the reference, whose launch shapes are fixed
 * (pixelGaussiansFull.cu:99-122).  Knobs (w2w_tune_name): 0 "blend_warps"
 * (4: two 4-warp CTAs per tile, 8: one 8-warp CTA; default 4), 1
 * "backward_split" (the per-pixel backward splits its heaviest tiles, up to
 * this many quarters of the SM count, across CTAs; 0..16, default 2), 2
 * "backward_ways" (segments per split tile, 2 or 3; default 2), 3 "binning"
 * (how a single-view call of at most 4096 tiles builds its sorted list: 0
 * key emission and the radix sort, 1 binning from the depth-ordered
 * Gaussians; default 0; w2w_forward_geometry records the path taken in
 * w2w_geometry_info.reserved, bit 0, and w2w_forward_render follows it), 4
 * "blend_queue" (0: one CTA per tile part, launched heaviest first; 1: a
 * persistent blend, one CTA per resident slot, pulling tile parts from a
 * device queue in the same order, each CTA a producer warp that gathers the
 * batches' records with TMA into a three-stage shared-memory ring and
 * "blend_warps" consumer warps; default 0), 5 "preprocess_blocks" (CTAs per
 * SM the projection pass's register budget is sized for: 4 caps a thread at
 * 64 registers, 3 at 80, 2 at 128; default 4), 6 "planned_forward" (the torch
 * binding's planned forward for repeated image sizes, 1 on, 0 off; default 1;
 * not tuned, the C ABI's entry points take the plan explicitly), 7
 * "blend_stage" (how the per-tile blend gathers a batch's records while it
 * walks the previous one: 0 into registers, 1 into shared memory with
 * cp.async, which fits five 4-warp CTAs per SM instead of four; default 1).
 * Results do not depend on them beyond the order of float atomic additions.
 * w2w_tune_set returns the previous value, or -1 (and changes nothing) for an
 * unknown knob or value. */
int w2w_tune_count(void);
const char* w2w_tune_name(int knob);
int w2w_tune_get(int knob);
int w2w_tune_set(int knob, int value);

/* ---- test hooks --------------------------------------------------------------
 * For tests of the failure path (no counterpart in the reference).
 * w2w_test_set_spin_limit: the iteration limit of every bounded device wait
 * (0 restores the default, 2^22 polls: a second or two); returns the previous
 * limit.  w2w_test_unpublished_tile: the CTA of tile `tile` of a stage (0: the
 * stand-alone scans, 1: the first pass of every sort, 2: the scan fused into
 * w2w_forward_geometry) skips publishing its status, so that the waits behind
 * it run out and the call reports W2W_ERR_TIMEOUT; -1 turns it off.  Returns
 * the previous tile (-2 for an unknown stage).  Nothing faults or hangs: every
 * wait ends at its limit.  Process-wide settings read at launch. */
unsigned w2w_test_set_spin_limit(unsigned limit);
long long w2w_test_unpublished_tile(int stage, long long tile);

#ifdef __cplusplus
}
#endif

#endif /* W2W_RASTER_H */
