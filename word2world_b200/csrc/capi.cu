// C ABI of the rasterizer (declared in include/w2w_raster.h): host
// orchestration of the kernels, state-buffer layouts and argument checks.
// The rasterizer entry points never allocate device memory: every buffer
// comes from the caller (w2w_voxel_field alone takes its temporaries from the
// stream-ordered allocator).  All work is enqueued on the caller's stream.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/w2w_raster.h"
#include "common.cuh"
#include "kernels.h"

using namespace w2w;

namespace {

inline cudaStream_t S(w2w_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

inline int check_launch() {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "w2w: CUDA error: %s\n", cudaGetErrorString(e));
    return W2W_ERR_CUDA;
  }
  return W2W_OK;
}

inline int tiles_x(int W) { return (W + kTile - 1) / kTile; }
inline int tiles_y(int H) { return (H + kTile - 1) / kTile; }
inline int num_tiles(int W, int H) { return tiles_x(W) * tiles_y(H); }

inline int ceil_log2(uint32_t v) {  // bits needed for values in [0, v)
  if (v <= 1) return 0;
  int b = 0;
  uint32_t x = v - 1;
  while (x) { ++b; x >>= 1; }
  return b;
}

bool settings_ok(const w2w_settings* s) {
  return s && s->P >= 0 && s->width > 0 && s->height > 0 && s->M >= 0 && s->degree >= 0 &&
         s->viewmatrix && s->projmatrix && s->campos && s->background && s->width < 65535 * kTile &&
         s->height < 65535 * kTile;
}

template <typename T>
T* at(void* base, size_t off) { return reinterpret_cast<T*>(static_cast<unsigned char*>(base) + off); }
template <typename T>
const T* at(const void* base, size_t off) {
  return reinterpret_cast<const T*>(static_cast<const unsigned char*>(base) + off);
}

// Sort key layout, chosen on the host from the instance count, the tile
// count and the depth-bit range: only the bits in which keys can differ are
// sorted on, packed into 32 bits when they fit.
struct KeyPlan {
  int key64, depth_bits, tile_bits, bits;
  uint32_t prefix;
};
KeyPlan plan_keys_tiles(const w2w_geometry_info& info, int tiles) {
  KeyPlan k{};
  const uint32_t dmin = info.depth_min_bits, dmax = info.depth_max_bits;
  const uint32_t x = dmin ^ dmax;
  int db = 0;
  while (db < 32 && (x >> db) != 0u) ++db;
  k.depth_bits = db;
  k.prefix = db >= 32 ? 0u : (dmin & ~((1u << db) - 1u));
  k.tile_bits = ceil_log2(uint32_t(tiles));
  k.bits = k.tile_bits + k.depth_bits;
  k.key64 = k.bits > 32 ? 1 : 0;
  return k;
}
KeyPlan plan_keys(const w2w_geometry_info& info, int W, int H) {
  KeyPlan k{};
  const uint32_t dmin = info.depth_min_bits, dmax = info.depth_max_bits;
  const uint32_t x = dmin ^ dmax;
  int db = 0;
  while (db < 32 && (x >> db) != 0u) ++db;
  k.depth_bits = db;
  k.prefix = db >= 32 ? 0u : (dmin & ~((1u << db) - 1u));
  k.tile_bits = ceil_log2(uint32_t(num_tiles(W, H)));
  k.bits = k.tile_bits + k.depth_bits;
  k.key64 = k.bits > 32 ? 1 : 0;
  return k;
}

// fold0 / fold1 (may be null): error words of earlier work on the same data
// (the depth sort and prefix scan of the binning path), carried into the
// binning state's word, which the caller reads.
__global__ void write_bin_header(BinHeader* h, KeyPlan k, uint32_t R, uint32_t passes, const uint32_t* fold0,
                                 const uint32_t* fold1) {
  h->error = (fold0 != nullptr ? *fold0 : 0u) | (fold1 != nullptr ? *fold1 : 0u);
  h->masks_valid = 1u;  // the blend that follows writes the block masks
  h->key64 = k.key64;
  h->depth_bits = k.depth_bits;
  h->depth_prefix = k.prefix;
  h->tile_bits = k.tile_bits;
  h->passes = passes;
  h->num_rendered = R;
  for (int i = 0; i < 8; ++i) h->tile_counter[i] = 0;
}

template <typename K>
__global__ void expand_keys(const BinHeader* h, const K* keys, long long n, uint64_t* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t db = h->depth_bits;
  const uint64_t k = uint64_t(keys[i]);
  const uint64_t tile = db >= 64 ? 0 : (k >> db);
  const uint32_t low = db >= 32 ? uint32_t(k) : uint32_t(k & ((1ull << db) - 1ull));
  out[i] = (tile << 32) | uint64_t(h->depth_prefix | low);
}

__global__ void ranges_from_sorted(const uint64_t* keys, long long n, int shift, uint2* ranges, int ntiles) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t t = keys[i] >> shift;
  if (t >= uint64_t(ntiles)) return;
  if (i == 0 || (keys[i - 1] >> shift) != t) ranges[t].x = uint32_t(i);
  if (i == n - 1 || (keys[i + 1] >> shift) != t) ranges[t].y = uint32_t(i + 1);
}

size_t sort_scratch_layout(long long n, size_t* keys_tmp, size_t* vals_tmp, size_t* hist, size_t* status,
                           size_t* counters, size_t* err) {
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t a = align256(o); o = a + bytes; return a; };
  const size_t nn = size_t(n > 0 ? n : 1);
  // the error word sits at byte 4 of every stage scratch (sort and scan), where
  // w2w_scratch_error reads it
  *err = take(256) + 4;
  *keys_tmp = take(nn * 8);
  *vals_tmp = take(nn * 4);
  *hist = take(size_t(kMaxPasses) * kMaxBins * 4);
  *status = take(sort_status_words(n) * 4);
  *counters = take(kMaxPasses * 4);
  return align256(o);
}

// Whether entry points with bounded device waits read their error word back
// before returning (w2w_set_error_check).
std::atomic<int> g_error_check{0};

int status_of(uint32_t err) {
  if (err & kErrTimeout) return W2W_ERR_TIMEOUT;
  if (err & (kErrCapacity | kErrRange)) return W2W_ERR_CAPACITY;
  return W2W_OK;
}

// Synchronises `st` and maps the device error word at `word` to a status.
int read_error_word(const void* word, cudaStream_t st) {
  uint32_t e = 0;
  if (cudaMemcpyAsync(&e, word, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return W2W_ERR_CUDA;
  return status_of(e);
}

// After a launch sequence: the launch status, then (in checked mode) the
// error word's.
int finish(const void* err_word, cudaStream_t st) {
  const int rc = check_launch();
  if (rc != W2W_OK || err_word == nullptr || g_error_check.load(std::memory_order_relaxed) == 0) return rc;
  return read_error_word(err_word, st);
}

}  // namespace

extern "C" {

int w2w_version(void) { return 1; }

int w2w_set_error_check(int mode) { return g_error_check.exchange(mode ? 1 : 0); }

int w2w_scratch_error(const void* scratch, w2w_stream_t stream) {
  if (!scratch) return W2W_ERR_INVALID;
  return read_error_word(static_cast<const unsigned char*>(scratch) + 4, S(stream));
}

int w2w_scan_noalloc_error(w2w_stream_t stream) {
  int rc = 0;
  void* scratch = scan_noalloc_scratch(&rc);
  if (rc != 0 || scratch == nullptr) return W2W_ERR_CUDA;
  return read_error_word(static_cast<const unsigned char*>(scratch) + 4, S(stream));
}

const char* w2w_status_string(int status) {
  switch (status) {
    case W2W_OK: return "ok";
    case W2W_ERR_INVALID: return "invalid argument";
    case W2W_ERR_CUDA: return "CUDA error";
    case W2W_ERR_CAPACITY: return "capacity exceeded";
    case W2W_ERR_TIMEOUT: return "device wait timed out";
    case W2W_ERR_SCRATCH: return "scratch buffer too small";
    default: return "unknown status";
  }
}

size_t w2w_geometry_state_bytes(int P) { return P < 0 ? 0 : GeomLayout(P).total; }
size_t w2w_image_state_bytes(int W, int H) { return (W <= 0 || H <= 0) ? 0 : ImageLayout(W, H).total; }
size_t w2w_binning_state_bytes(long long R, int W, int H) {
  if (R < 0 || W <= 0 || H <= 0) return 0;
  return BinLayout(R, num_tiles(W, H)).total;
}
size_t w2w_backward_scratch_bytes(int P) {
  return P < 0 ? 0 : align256(size_t(P) * 16) + align256(size_t(P) * 4);
}

size_t w2w_geometry_offset(int P, const char* name) {
  const GeomLayout L(P);
  if (!name) return size_t(-1);
  if (!strcmp(name, "header")) return L.header;
  if (!strcmp(name, "depth")) return L.depth;
  if (!strcmp(name, "clamped")) return L.clamped;
  if (!strcmp(name, "means2D")) return L.means2D;
  if (!strcmp(name, "cov3D")) return L.cov3D;
  if (!strcmp(name, "conic_opacity")) return L.conic;
  if (!strcmp(name, "rgb")) return L.rgb;
  if (!strcmp(name, "tiles_touched")) return L.tiles;
  if (!strcmp(name, "offsets")) return L.offsets;
  if (!strcmp(name, "rect")) return L.rect;
  if (!strcmp(name, "prev_reach")) return L.prev_reach;
  if (!strcmp(name, "record")) return L.record;
  if (!strcmp(name, "bwd_record")) return L.bwd_record;
  return size_t(-1);
}

size_t w2w_image_offset(int W, int H, const char* name) {
  const ImageLayout L(W, H);
  if (!name) return size_t(-1);
  if (!strcmp(name, "n_contrib")) return L.n_contrib;
  if (!strcmp(name, "ranges")) return L.ranges;
  if (!strcmp(name, "T_final")) return L.T_final;
  if (!strcmp(name, "tile_max")) return L.tile_max;
  if (!strcmp(name, "order")) return L.order;
  if (!strcmp(name, "order_bwd")) return L.order_bwd;
  return size_t(-1);
}

size_t w2w_binning_offset(long long R, int W, int H, const char* name) {
  const BinLayout L(R, num_tiles(W, H));
  if (!name) return size_t(-1);
  if (!strcmp(name, "header")) return L.header;
  if (!strcmp(name, "keys_a")) return L.keysA;
  if (!strcmp(name, "keys_b")) return L.keysB;
  if (!strcmp(name, "vals_a")) return L.valsA;
  if (!strcmp(name, "vals_b")) return L.valsB;
  return size_t(-1);
}

// Single-view calls with at most kMaxBinTiles tiles bin their instances from
// the depth-ordered Gaussians (binning.cu) when the tuning knob selects it;
// others emit keys and sort them.  The geometry phase records its choice in
// the info it returns, so the render follows it whatever the knob says then.
inline bool use_binning(int P, int W, int H) {
  return P > 0 && num_tiles(W, H) <= kMaxBinTiles && tune_value(kTuneBinning) == 1;
}
constexpr uint32_t kInfoDepthOrder = 1u;  // w2w_geometry_info::reserved: the depth order is prepared

// The binning path's per-Gaussian half, after the projection pass: the
// Gaussians sorted stably by the depth bits their keys keep, and the prefix of
// their owned instance counts in that order.  Errors land in the geometry
// header's word and the prefix scan's scratch word (read back by the render).
static void launch_depth_order(const w2w_settings* s, void* geom_state, const w2w_geometry_info& info,
                               cudaStream_t st) {
  const int P = s->P;
  const GeomLayout L(P);
  const KeyPlan kp = plan_keys(info, s->width, s->height);
  uint32_t* order = at<uint32_t>(geom_state, L.dorder);
  if (kp.depth_bits == 0) {
    launch_iota(order, P, st);  // one depth: Gaussian order
  } else {
    SortArgs so{};
    so.n = P; so.key64 = 0; so.begin_bit = 0; so.bits = kp.depth_bits;
    so.keys_in = at<uint32_t>(geom_state, L.depth);  // the depths' float bits
    so.vals_in = nullptr;                            // values: the Gaussian ids
    so.keys_out = at<uint32_t>(geom_state, L.dkeys); so.vals_out = order;
    so.keys_tmp = at<uint32_t>(geom_state, L.dtmp_keys); so.vals_tmp = at<uint32_t>(geom_state, L.dtmp_vals);
    so.hist = at<uint32_t>(geom_state, L.dsort_hist);
    so.counters = at<uint32_t>(geom_state, L.dsort_counters);
    so.status = at<uint32_t>(geom_state, L.dsort_status);
    so.error = &at<GeomHeader>(geom_state, L.header)->error;
    so.tile_shift = 0; so.num_tiles = 0; so.tile_hist = nullptr; so.ranges = nullptr;
    const int passes = sort_passes(kp.depth_bits);
    so.clear_span = at<void>(geom_state, L.dsort_hist);
    so.clear_bytes = L.dsort_status - L.dsort_hist +
                     size_t(passes) * kMaxBins * 4 * size_t((P + sort_tile_keys(0) - 1) / sort_tile_keys(0));
    so.spin_limit = spin_limit();
    so.unpublished_tile = unpublished_tile(kWaitSort);
    so.stage_hist = so.stage_pass = kStDepthSort;
    launch_sort(so, st);
  }
  BinArgs b{};
  b.P = P; b.R = uint32_t(info.num_rendered);
  b.order = order;
  b.tiles = at<uint32_t>(geom_state, L.tiles);
  b.offsets = at<uint32_t>(geom_state, L.offsets);
  b.rect = at<uint32_t>(geom_state, L.rect);
  b.prev_reach = at<uint32_t>(geom_state, L.prev_reach);
  uint32_t* count = at<uint32_t>(geom_state, L.dtmp_vals);  // free once the sort is done
  uint32_t* dprefix = at<uint32_t>(geom_state, L.dprefix);
  stage_begin(kStDepthSort, st);
  launch_owned_counts(b, count, st);
  cudaMemsetAsync(dprefix, 0, 4, st);
  stage_end(kStDepthSort, st, 1);
  launch_scan(count, dprefix + 1, P, 0, at<void>(geom_state, L.dscan), st);
}

// raw != null: Renderer.render's raw parameters, activated by preprocess
struct RawParams {
  const float *svec, *quat, *logit, *sh_dc, *sh_ac;
};

// The projection pass alone (P > 0): header cleared, preprocess launched.
static int geometry_launch(const w2w_settings* s, const float* means3D, const float* scales, const float* rotations,
                           const float* opacities, const float* shs, const RawParams* raw, int* radii,
                           void* geom_state, w2w_stream_t stream) {
  const GeomLayout L(s->P);
  cudaStream_t st = S(stream);
  cudaMemsetAsync(geom_state, 0, L.depth, st);  // header + scan status
  PreprocessArgs a{};
  a.P = s->P; a.W = s->width; a.H = s->height; a.degree = s->degree; a.M = s->M;
  a.compat_spill = s->compat_spill;
  a.focal_x = s->focal_x;
  a.view = s->viewmatrix; a.proj = s->projmatrix; a.campos = s->campos;
  a.means3D = means3D; a.scales = scales; a.rotations = rotations; a.opacities = opacities; a.shs = shs;
  a.radii = radii;
  a.header = at<GeomHeader>(geom_state, L.header);
  a.scan_status = at<unsigned long long>(geom_state, L.scan_status);
  a.depth = at<float>(geom_state, L.depth);
  a.clamped = at<uint8_t>(geom_state, L.clamped);
  a.means2D = at<float>(geom_state, L.means2D);
  a.cov3D = at<float>(geom_state, L.cov3D);
  a.conic = at<float>(geom_state, L.conic);
  a.rgb = at<float>(geom_state, L.rgb);
  a.tiles = at<uint32_t>(geom_state, L.tiles);
  a.offsets = at<uint32_t>(geom_state, L.offsets);
  a.rect = at<uint32_t>(geom_state, L.rect);
  a.prev_reach = at<uint32_t>(geom_state, L.prev_reach);
  a.record = at<float>(geom_state, L.record);
  a.bwd_record = at<float>(geom_state, L.bwd_record);
  a.spin_limit = spin_limit();
  a.unpublished_tile = unpublished_tile(kWaitPreprocess);
  if (raw != nullptr) {
    a.svec = raw->svec; a.quat = raw->quat; a.logit = raw->logit; a.sh_dc = raw->sh_dc; a.sh_ac = raw->sh_ac;
  }
  launch_preprocess(a, st);
  return check_launch();
}

static int forward_geometry(const w2w_settings* s, const float* means3D, const float* scales, const float* rotations,
                            const float* opacities, const float* shs, const RawParams* raw, int* radii,
                            void* geom_state, w2w_geometry_info* info, w2w_stream_t stream) {
  std::memset(info, 0, sizeof(*info));
  if (s->P == 0) return W2W_OK;
  const int rc = geometry_launch(s, means3D, scales, rotations, opacities, shs, raw, radii, geom_state, stream);
  if (rc) return rc;
  cudaStream_t st = S(stream);
  GeomHeader h;
  if (cudaMemcpyAsync(&h, at<GeomHeader>(geom_state, GeomLayout(s->P).header), sizeof(h), cudaMemcpyDeviceToHost,
                      st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return W2W_ERR_CUDA;
  info->num_rendered = h.num_rendered;
  info->depth_min_bits = ~h.depth_min;
  info->depth_max_bits = h.depth_max;
  info->error = h.error;
  if (h.error & kErrTimeout) return W2W_ERR_TIMEOUT;
  if (h.error & kErrCapacity) return W2W_ERR_CAPACITY;
  if (h.num_rendered > 0 && use_binning(s->P, s->width, s->height)) {
    launch_depth_order(s, geom_state, *info, st);
    info->reserved |= kInfoDepthOrder;  // tells w2w_forward_render which path to take
    return check_launch();
  }
  return W2W_OK;
}

int w2w_forward_geometry(const w2w_settings* s, const float* means3D, const float* scales, const float* rotations,
                         const float* opacities, const float* shs, int* radii, void* geom_state,
                         w2w_geometry_info* info, w2w_stream_t stream) {
  if (!settings_ok(s) || !info || (s->P > 0 && (!means3D || !scales || !rotations || !opacities || !radii ||
                                                !geom_state || (s->M > 0 && !shs))))
    return W2W_ERR_INVALID;
  return forward_geometry(s, means3D, scales, rotations, opacities, shs, nullptr, radii, geom_state, info, stream);
}

int w2w_forward_geometry_raw(const w2w_settings* s, const float* means3D, const float* svec, const float* quaternion,
                             const float* opacity_logit, const float* sh_dc, const float* sh_ac, int* radii,
                             void* geom_state, w2w_geometry_info* info, w2w_stream_t stream) {
  if (!settings_ok(s) || !info || s->M < 1 || s->M > 16 ||
      (s->P > 0 && (!means3D || !svec || !quaternion || !opacity_logit || !sh_dc || (s->M > 1 && !sh_ac) ||
                    !radii || !geom_state)))
    return W2W_ERR_INVALID;
  const RawParams raw{svec, quaternion, opacity_logit, sh_dc, sh_ac};
  return forward_geometry(s, means3D, nullptr, nullptr, nullptr, nullptr, &raw, radii, geom_state, info, stream);
}

int w2w_forward_render(const w2w_settings* s, const void* geom_state, const w2w_geometry_info* info,
                       void* binning_state, void* image_state, float* out_color, float* out_depth,
                       float* out_alpha, w2w_stream_t stream) {
  if (!settings_ok(s) || !info || !image_state || !out_color || !out_depth || !out_alpha) return W2W_ERR_INVALID;
  const long long R = info->num_rendered;
  if (R < 0 || R >= (1LL << 30)) return W2W_ERR_CAPACITY;
  if (R > 0 && (!geom_state || !binning_state)) return W2W_ERR_INVALID;
  cudaStream_t st = S(stream);
  const int W = s->width, H = s->height, T = num_tiles(W, H);
  const ImageLayout IL(W, H);
  uint2* ranges = at<uint2>(image_state, IL.ranges);
  const uint32_t* point_list = nullptr;
  const void* err_word = nullptr;  // the binning header's error word
  if (R == 0) {
    cudaMemsetAsync(ranges, 0, sizeof(uint2) * size_t(T), st);
  } else if ((info->reserved & kInfoDepthOrder) != 0u) {
    const GeomLayout GL(s->P);
    const BinLayout BL(R, T);
    const KeyPlan kp = plan_keys(*info, W, H);
    BinHeader* bh = at<BinHeader>(binning_state, BL.header);
    err_word = &bh->error;
    stage_begin(kStOther, st);
    write_bin_header<<<1, 1, 0, st>>>(bh, kp, uint32_t(R), 0u, &at<GeomHeader>(geom_state, GL.header)->error,
                                      at<uint32_t>(geom_state, GL.dscan + 4));
    stage_end(kStOther, st, 1);
    BinArgs b{};
    b.P = s->P; b.R = uint32_t(R); b.gw = tiles_x(W); b.T = T;
    b.key64 = kp.key64; b.depth_bits = uint32_t(kp.depth_bits);
    b.order = at<uint32_t>(geom_state, GL.dorder);
    b.dprefix = at<uint32_t>(geom_state, GL.dprefix);
    b.tiles = at<uint32_t>(geom_state, GL.tiles);
    b.offsets = at<uint32_t>(geom_state, GL.offsets);
    b.rect = at<uint32_t>(geom_state, GL.rect);
    b.prev_reach = at<uint32_t>(geom_state, GL.prev_reach);
    b.depth = at<float>(geom_state, GL.depth);
    b.warp_start = at<uint32_t>(binning_state, BL.warp_start);
    b.counts = at<uint32_t>(binning_state, BL.bin_counts);
    b.tile_total = at<uint32_t>(binning_state, BL.tile_hist);
    b.ranges = ranges;
    b.keys = at<void>(binning_state, BL.keysA);
    b.vals = at<uint32_t>(binning_state, BL.valsA);
    b.error = &bh->error;
    launch_binning(b, st);
    point_list = b.vals;
  } else {
    const GeomLayout GL(s->P);
    const BinLayout BL(R, T);
    const KeyPlan kp = plan_keys(*info, W, H);
    const int passes = sort_passes(kp.bits);
    BinHeader* bh = at<BinHeader>(binning_state, BL.header);
    err_word = &bh->error;
    stage_begin(kStOther, st);
    write_bin_header<<<1, 1, 0, st>>>(bh, kp, uint32_t(R), uint32_t(passes), nullptr, nullptr);
    stage_end(kStOther, st, 1);
    // the sort result lands in (keysA, valsA); key emission targets the
    // buffer that makes the ping-pong end there
    const bool odd = (passes % 2) == 1;
    void* keysA = at<void>(binning_state, BL.keysA);
    void* keysB = at<void>(binning_state, BL.keysB);
    uint32_t* valsA = at<uint32_t>(binning_state, BL.valsA);
    uint32_t* valsB = at<uint32_t>(binning_state, BL.valsB);
    DuplicateArgs d{};
    d.P = s->P; d.gw = tiles_x(W); d.R = uint32_t(R); d.key64 = kp.key64; d.depth_bits = uint32_t(kp.depth_bits);
    d.tiles = at<uint32_t>(geom_state, GL.tiles);
    d.offsets = at<uint32_t>(geom_state, GL.offsets);
    d.rect = at<uint32_t>(geom_state, GL.rect);
    d.prev_reach = at<uint32_t>(geom_state, GL.prev_reach);
    d.depth = at<float>(geom_state, GL.depth);
    d.keys = odd ? keysB : keysA;
    d.vals = odd ? valsB : valsA;
    launch_duplicate(d, st);
    SortArgs so{};
    so.n = R; so.key64 = kp.key64; so.begin_bit = 0; so.bits = kp.bits;
    so.keys_in = d.keys; so.vals_in = d.vals;
    so.match_rank = 1;  // emitted Gaussian by Gaussian: few distinct digits per warp
    so.keys_out = keysA; so.vals_out = valsA;
    so.keys_tmp = keysB; so.vals_tmp = valsB;
    so.hist = at<uint32_t>(binning_state, BL.hist);
    so.status = at<uint32_t>(binning_state, BL.status);
    so.counters = bh->tile_counter;
    so.error = &bh->error;
    so.tile_shift = kp.depth_bits;
    so.num_tiles = T;
    so.tile_hist = at<uint32_t>(binning_state, BL.tile_hist);
    so.ranges = ranges;
    // hist, tile_hist and the used status words are contiguous; the tile
    // counters were cleared by write_bin_header
    so.clear_span = at<void>(binning_state, BL.hist);
    so.clear_bytes = BL.status - BL.hist + size_t(passes > 0 ? passes : 1) * kMaxBins * 4 *
                     size_t((R + sort_tile_keys(kp.key64) - 1) / sort_tile_keys(kp.key64));
    so.spin_limit = spin_limit();
    so.unpublished_tile = unpublished_tile(kWaitSort);
    launch_sort(so, st);
    point_list = valsA;
  }
  BlendArgs b{};
  b.W = W; b.H = H;
  b.ranges = ranges;
  b.point_list = point_list;
  b.record = R > 0 ? at<float>(geom_state, GeomLayout(s->P).record) : nullptr;
  b.num_records = uint32_t(s->P);
  if (R > 0) {
    const BinLayout BL(R, T);
    b.mask_top = at<uint8_t>(binning_state, BL.masks);
    b.mask_bottom = b.mask_top + R;
    b.masks_valid = &at<BinHeader>(binning_state, BL.header)->masks_valid;
  }
  b.bg = s->background;
  b.out_color = out_color; b.out_depth = out_depth; b.out_alpha = out_alpha;
  b.n_contrib = at<uint32_t>(image_state, IL.n_contrib);
  b.T_final = at<float>(image_state, IL.T_final);
  b.tile_max = at<uint32_t>(image_state, IL.tile_max);
  b.order = at<uint32_t>(image_state, IL.order);
  b.order_bwd = at<uint32_t>(image_state, IL.order_bwd);
  b.queue = at<uint32_t>(image_state, IL.queue);
  b.error = const_cast<uint32_t*>(static_cast<const uint32_t*>(err_word));
  b.spin_limit = spin_limit();
  launch_blend(b, st);
  return finish(err_word, st);
}

// ---- planned forward --------------------------------------------------------
// A render whose sort and blend are launched before the host knows the view's
// instance count R: the binning state is laid out for a capacity C and the
// keys carry a guessed number of depth bits; a one-thread kernel checks both
// against the projection pass's header on the device and either lets the
// emission, histogram, sort passes and blend process R instances (read from
// device memory), or sets `replan` and makes them process none, after which
// the caller renders again with the exact plan.  A guess with more depth bits
// than the view needs sorts the same way: the extra bits are the common high
// bits of every depth (the range of the depths' bit patterns), constant across
// the keys, so the sorted list, the ranges and everything after them are
// bit-identical to the exact plan's.

static int geometry_async(const w2w_settings* s, const float* means3D, const float* scales, const float* rotations,
                          const float* opacities, const float* shs, const RawParams* raw, int* radii,
                          void* geom_state, void* header_host, w2w_stream_t stream) {
  if (!header_host) return W2W_ERR_INVALID;
  if (s->P == 0) {
    std::memset(header_host, 0, 16);
    return W2W_OK;
  }
  const int rc = geometry_launch(s, means3D, scales, rotations, opacities, shs, raw, radii, geom_state, stream);
  if (rc) return rc;
  // the header's first four words: error, depth min (inverted), depth max, R
  if (cudaMemcpyAsync(header_host, at<GeomHeader>(geom_state, GeomLayout(s->P).header), 16, cudaMemcpyDeviceToHost,
                      S(stream)) != cudaSuccess)
    return W2W_ERR_CUDA;
  return W2W_OK;
}

int w2w_forward_geometry_async(const w2w_settings* s, const float* means3D, const float* scales,
                               const float* rotations, const float* opacities, const float* shs, int* radii,
                               void* geom_state, void* header_host, w2w_stream_t stream) {
  if (!settings_ok(s) || (s->P > 0 && (!means3D || !scales || !rotations || !opacities || !radii || !geom_state ||
                                       (s->M > 0 && !shs))))
    return W2W_ERR_INVALID;
  return geometry_async(s, means3D, scales, rotations, opacities, shs, nullptr, radii, geom_state, header_host,
                        stream);
}

int w2w_forward_geometry_raw_async(const w2w_settings* s, const float* means3D, const float* svec,
                                   const float* quaternion, const float* opacity_logit, const float* sh_dc,
                                   const float* sh_ac, int* radii, void* geom_state, void* header_host,
                                   w2w_stream_t stream) {
  if (!settings_ok(s) || s->M < 1 || s->M > 16 ||
      (s->P > 0 && (!means3D || !svec || !quaternion || !opacity_logit || !sh_dc || (s->M > 1 && !sh_ac) ||
                    !radii || !geom_state)))
    return W2W_ERR_INVALID;
  const RawParams raw{svec, quaternion, opacity_logit, sh_dc, sh_ac};
  return geometry_async(s, means3D, nullptr, nullptr, nullptr, nullptr, &raw, radii, geom_state, header_host, stream);
}

int w2w_geometry_info_from_header(const void* header_host, w2w_geometry_info* info) {
  if (!header_host || !info) return W2W_ERR_INVALID;
  uint32_t w[4];
  std::memcpy(w, header_host, sizeof(w));
  std::memset(info, 0, sizeof(*info));
  info->error = w[0];
  info->depth_min_bits = ~w[1];
  info->depth_max_bits = w[2];
  info->num_rendered = w[3];
  if (w[0] & kErrTimeout) return W2W_ERR_TIMEOUT;
  if (w[0] & kErrCapacity) return W2W_ERR_CAPACITY;
  return W2W_OK;
}

int w2w_depth_bits_needed(const w2w_geometry_info* info) {
  if (!info) return -1;
  const uint32_t x = info->depth_min_bits ^ info->depth_max_bits;
  int db = 0;
  while (db < 32 && (x >> db) != 0u) ++db;
  return db;
}

long long w2w_planned_capacity(long long num_rendered) {
  if (num_rendered < 0) return -1;
  const long long want = num_rendered + num_rendered / 4;  // 25 % headroom over the count it was sized from
  long long c = (want + W2W_PLAN_QUANTUM - 1) / W2W_PLAN_QUANTUM * W2W_PLAN_QUANTUM;
  if (c < W2W_PLAN_QUANTUM) c = W2W_PLAN_QUANTUM;
  return c < (1LL << 30) ? c : -1;
}

long long w2w_binning_layout_count(long long num_rendered, size_t state_bytes, int W, int H) {
  if (num_rendered < 0 || W <= 0 || H <= 0) return -1;
  const int T = num_tiles(W, H);
  if (BinLayout(num_rendered, T).total == state_bytes) return num_rendered;
  // a planned render's state: the capacity, a multiple of W2W_PLAN_QUANTUM at
  // least num_rendered (the layout grows by more than 16 bytes per instance,
  // so at most state_bytes / 16 of them)
  long long lo = (num_rendered + W2W_PLAN_QUANTUM - 1) / W2W_PLAN_QUANTUM;
  long long hi = (long long)(state_bytes / 16) / W2W_PLAN_QUANTUM + 1;
  if (lo < 1) lo = 1;
  while (lo < hi) {
    const long long mid = (lo + hi) / 2;
    if (BinLayout(mid * W2W_PLAN_QUANTUM, T).total < state_bytes) lo = mid + 1;
    else hi = mid;
  }
  return BinLayout(lo * W2W_PLAN_QUANTUM, T).total == state_bytes ? lo * W2W_PLAN_QUANTUM : -1;
}

}  // extern "C"

// The planned render's header: the caller's key plan, checked against the
// view's own count and depth range (the projection pass's header).
__global__ void plan_bin_header(BinHeader* h, const GeomHeader* g, uint32_t capacity, KeyPlan k, uint32_t passes) {
  const uint32_t R = g->num_rendered;
  const uint32_t dmin = ~g->depth_min, dmax = g->depth_max;
  const uint32_t x = dmin ^ dmax;
  int need = 0;
  while (need < 32 && (x >> need) != 0u) ++need;
  const bool ok = R <= capacity && need <= k.depth_bits && (g->error & (kErrTimeout | kErrCapacity)) == 0u;
  h->error = 0u;
  h->masks_valid = 1u;
  h->key64 = k.key64;
  h->depth_bits = k.depth_bits;
  h->depth_prefix = k.depth_bits >= 32 ? 0u : (dmin & ~((1u << k.depth_bits) - 1u));
  h->tile_bits = k.tile_bits;
  h->passes = passes;
  h->num_rendered = R;
  h->n_sort = ok ? R : 0u;
  h->replan = ok ? 0u : 1u;
  for (int i = 0; i < 8; ++i) h->tile_counter[i] = 0;
}

extern "C" {

int w2w_forward_render_planned(const w2w_settings* s, const void* geom_state, long long capacity, int depth_bits,
                               void* binning_state, void* image_state, float* out_color, float* out_depth,
                               float* out_alpha, w2w_stream_t stream) {
  if (!settings_ok(s) || s->P <= 0 || !geom_state || !binning_state || !image_state || !out_color || !out_depth ||
      !out_alpha || capacity < 1 || capacity >= (1LL << 30) || depth_bits < 0 || depth_bits > 32)
    return W2W_ERR_INVALID;
  cudaStream_t st = S(stream);
  const int W = s->width, H = s->height, T = num_tiles(W, H);
  const ImageLayout IL(W, H);
  const GeomLayout GL(s->P);
  const BinLayout BL(capacity, T);
  KeyPlan kp{};
  kp.depth_bits = depth_bits;
  kp.tile_bits = ceil_log2(uint32_t(T));
  kp.bits = kp.tile_bits + kp.depth_bits;
  kp.key64 = kp.bits > 32 ? 1 : 0;
  const int passes = sort_passes(kp.bits);
  BinHeader* bh = at<BinHeader>(binning_state, BL.header);
  stage_begin(kStOther, st);
  plan_bin_header<<<1, 1, 0, st>>>(bh, at<GeomHeader>(geom_state, GL.header), uint32_t(capacity), kp,
                                   uint32_t(passes));
  stage_end(kStOther, st, 1);
  // the sort result lands in (keysA, valsA); key emission targets the buffer
  // that makes the ping-pong end there
  const bool odd = (passes % 2) == 1;
  void* keysA = at<void>(binning_state, BL.keysA);
  void* keysB = at<void>(binning_state, BL.keysB);
  uint32_t* valsA = at<uint32_t>(binning_state, BL.valsA);
  uint32_t* valsB = at<uint32_t>(binning_state, BL.valsB);
  DuplicateArgs d{};
  d.P = s->P; d.gw = tiles_x(W); d.R = uint32_t(capacity); d.key64 = kp.key64;
  d.depth_bits = uint32_t(kp.depth_bits);
  d.tiles = at<uint32_t>(geom_state, GL.tiles);
  d.offsets = at<uint32_t>(geom_state, GL.offsets);
  d.rect = at<uint32_t>(geom_state, GL.rect);
  d.prev_reach = at<uint32_t>(geom_state, GL.prev_reach);
  d.depth = at<float>(geom_state, GL.depth);
  d.keys = odd ? keysB : keysA;
  d.vals = odd ? valsB : valsA;
  d.n_dev = &bh->n_sort;
  launch_duplicate(d, st);
  SortArgs so{};
  so.n = capacity; so.key64 = kp.key64; so.begin_bit = 0; so.bits = kp.bits;
  so.keys_in = d.keys; so.vals_in = d.vals;
  so.match_rank = 1;  // emitted Gaussian by Gaussian: few distinct digits per warp
  so.n_dev = &bh->n_sort;
  so.keys_out = keysA; so.vals_out = valsA;
  so.keys_tmp = keysB; so.vals_tmp = valsB;
  so.hist = at<uint32_t>(binning_state, BL.hist);
  so.status = at<uint32_t>(binning_state, BL.status);
  so.counters = bh->tile_counter;
  so.error = &bh->error;
  so.tile_shift = kp.depth_bits;
  so.num_tiles = T;
  so.tile_hist = at<uint32_t>(binning_state, BL.tile_hist);
  so.ranges = at<uint2>(image_state, IL.ranges);
  so.clear_span = at<void>(binning_state, BL.hist);
  so.clear_bytes = BL.status - BL.hist + size_t(passes > 0 ? passes : 1) * kMaxBins * 4 *
                   size_t((capacity + sort_tile_keys(kp.key64) - 1) / sort_tile_keys(kp.key64));
  so.spin_limit = spin_limit();
  so.unpublished_tile = unpublished_tile(kWaitSort);
  launch_sort(so, st);
  BlendArgs b{};
  b.W = W; b.H = H;
  b.ranges = at<uint2>(image_state, IL.ranges);
  b.point_list = valsA;
  b.record = at<float>(geom_state, GL.record);
  b.num_records = uint32_t(s->P);
  b.mask_top = at<uint8_t>(binning_state, BL.masks);
  b.mask_bottom = b.mask_top + capacity;
  b.masks_valid = &bh->masks_valid;
  b.bg = s->background;
  b.out_color = out_color; b.out_depth = out_depth; b.out_alpha = out_alpha;
  b.n_contrib = at<uint32_t>(image_state, IL.n_contrib);
  b.T_final = at<float>(image_state, IL.T_final);
  b.tile_max = at<uint32_t>(image_state, IL.tile_max);
  b.order = at<uint32_t>(image_state, IL.order);
  b.order_bwd = at<uint32_t>(image_state, IL.order_bwd);
  b.queue = at<uint32_t>(image_state, IL.queue);
  b.error = &bh->error;
  b.spin_limit = spin_limit();
  launch_blend(b, st);
  return finish(&bh->error, st);
}

int w2w_binning_replanned(const void* binning_state, w2w_stream_t stream) {
  if (!binning_state) return -1;
  uint32_t v = 0;
  cudaStream_t st = S(stream);
  if (cudaMemcpyAsync(&v, &static_cast<const BinHeader*>(binning_state)->replan, 4, cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return -1;
  return int(v);
}

int w2w_state_error(const void* state, int which, w2w_stream_t stream) {
  if (!state) return -1;
  uint32_t e = 0;
  cudaStream_t st = S(stream);
  if (cudaMemcpyAsync(&e, state, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return -1;
  (void)which;  // both headers start with their error word
  return int(e);
}

struct RawGrads {
  const float *svec, *quat, *logit, *sh_dc, *sh_ac;
  float *d_sh_dc, *d_sh_ac;
  float *dens_accum, *dens_counter;  // densification statistics, or null
};

static int backward_impl(const w2w_settings* s, const float* means3D, const float* scales, const float* rotations,
                         const float* shs, const RawGrads* raw, const int* radii, const void* geom_state,
                         long long R, const void* binning_state, const void* image_state, const float* out_alpha,
                         const float* dL_dcolor, const float* dL_ddepth, const float* dL_dalpha, int grad_mode,
                         void* scratch, size_t scratch_bytes, float* dL_dmeans2D, float* dL_dcolors,
                         float* dL_dopacity, float* dL_dmeans3D, float* dL_dcov3D, float* dL_dsh, float* dL_dscales,
                         float* dL_drotations, w2w_stream_t stream) {
  const int P = s->P;
  if (!scratch || scratch_bytes < w2w_backward_scratch_bytes(P)) return W2W_ERR_SCRATCH;
  cudaStream_t st = S(stream);
  const int W = s->width, H = s->height;
  const GeomLayout GL(P);
  const ImageLayout IL(W, H);
  float* acc_cov = static_cast<float*>(scratch);
  float* acc_depth = at<float>(scratch, align256(size_t(P) * 16));
  cudaMemsetAsync(scratch, 0, w2w_backward_scratch_bytes(P), st);
  cudaMemsetAsync(dL_dmeans2D, 0, sizeof(float) * 3 * size_t(P), st);
  cudaMemsetAsync(dL_dcolors, 0, sizeof(float) * 3 * size_t(P), st);
  cudaMemsetAsync(dL_dopacity, 0, sizeof(float) * size_t(P), st);
  BackwardArgs a{};
  a.P = P; a.W = W; a.H = H; a.degree = s->degree; a.M = s->M; a.grad_mode = grad_mode;
  a.h_x = float(W) / (2.0f * s->tan_fovx);
  a.h_y = float(H) / (2.0f * s->tan_fovy);
  a.focal_x = a.h_x;  // exact mode: the forward's focal under the W / (2 tan) convention
  a.tan_fovx = s->tan_fovx; a.tan_fovy = s->tan_fovy;
  a.scale_modifier = s->scale_modifier;
  a.view = s->viewmatrix; a.proj = s->projmatrix; a.campos = s->campos; a.bg = s->background;
  a.means3D = means3D; a.scales = scales; a.rotations = rotations; a.shs = shs;
  a.radii = radii;
  a.cov3D = at<float>(geom_state, GL.cov3D);
  a.clamped = at<uint8_t>(geom_state, GL.clamped);
  a.record = at<float>(geom_state, GL.record);
  a.bwd_record = at<float>(geom_state, GL.bwd_record);
  a.ranges = at<uint2>(image_state, IL.ranges);
  a.point_list = R > 0 ? at<uint32_t>(binning_state, BinLayout(R, num_tiles(W, H)).valsA) : nullptr;
  if (R > 0) {
    const BinLayout BL(R, num_tiles(W, H));
    a.mask_top = at<uint8_t>(binning_state, BL.masks);
    a.mask_bottom = a.mask_top + R;
    a.masks_valid = &at<BinHeader>(binning_state, BL.header)->masks_valid;
  }
  a.n_contrib = at<uint32_t>(image_state, IL.n_contrib);
  a.tile_max = at<uint32_t>(image_state, IL.tile_max);
  a.order_bwd = at<uint32_t>(image_state, IL.order_bwd);
  a.T_final = at<float>(image_state, IL.T_final);
  a.out_alpha = out_alpha;
  a.dL_dcolor = dL_dcolor; a.dL_ddepth = dL_ddepth; a.dL_dalpha = dL_dalpha;
  a.dL_dmean2D = dL_dmeans2D; a.acc_cov = acc_cov; a.dL_dopacity = dL_dopacity; a.dL_dcolors = dL_dcolors;
  a.acc_depth = acc_depth;
  a.dL_dmeans3D = dL_dmeans3D; a.dL_dcov3D = dL_dcov3D; a.dL_dsh = dL_dsh; a.dL_dscales = dL_dscales;
  a.dL_drotations = dL_drotations;
  if (raw != nullptr) {
    a.svec = raw->svec; a.quat = raw->quat; a.logit = raw->logit; a.sh_dc = raw->sh_dc; a.sh_ac = raw->sh_ac;
    a.dL_dsh_dc = raw->d_sh_dc; a.dL_dsh_ac = raw->d_sh_ac;
    a.dens_accum = raw->dens_accum; a.dens_counter = raw->dens_counter;
  }
  if (R > 0) launch_backward_render(a, st);
  launch_backward_gaussians(a, st);
  return check_launch();
}

int w2w_backward(const w2w_settings* s, const float* means3D, const float* scales, const float* rotations,
                 const float* shs, const int* radii, const void* geom_state,
                 long long R, const void* binning_state, const void* image_state, const float* out_alpha,
                 const float* dL_dcolor, const float* dL_ddepth, const float* dL_dalpha, int grad_mode,
                 void* scratch, size_t scratch_bytes, float* dL_dmeans2D, float* dL_dcolors, float* dL_dopacity,
                 float* dL_dmeans3D, float* dL_dcov3D, float* dL_dsh, float* dL_dscales, float* dL_drotations,
                 w2w_stream_t stream) {
  if (!settings_ok(s) || (grad_mode != 0 && grad_mode != 1)) return W2W_ERR_INVALID;
  const int P = s->P;
  if (P == 0) return W2W_OK;
  if (!means3D || !scales || !rotations || !radii || !geom_state || !image_state || !out_alpha ||
      !dL_dcolor || !dL_dmeans2D || !dL_dcolors || !dL_dopacity || !dL_dmeans3D ||
      !dL_dcov3D || !dL_dscales || !dL_drotations || (s->M > 0 && (!shs || !dL_dsh)) || (R > 0 && !binning_state))
    return W2W_ERR_INVALID;
  return backward_impl(s, means3D, scales, rotations, shs, nullptr, radii, geom_state, R, binning_state,
                       image_state, out_alpha, dL_dcolor, dL_ddepth, dL_dalpha, grad_mode, scratch, scratch_bytes,
                       dL_dmeans2D, dL_dcolors, dL_dopacity, dL_dmeans3D, dL_dcov3D, dL_dsh, dL_dscales,
                       dL_drotations, stream);
}

int w2w_backward_raw_densify(const w2w_settings* s, const float* means3D, const float* svec, const float* quaternion,
                     const float* opacity_logit, const float* sh_dc, const float* sh_ac, const int* radii,
                     const void* geom_state, long long R, const void* binning_state, const void* image_state,
                     const float* out_alpha, const float* dL_dcolor, const float* dL_ddepth, const float* dL_dalpha,
                     void* scratch, size_t scratch_bytes, float* dL_dmeans2D, float* dL_dcolors,
                     float* dL_dopacity_logit, float* dL_dmeans3D, float* dL_dcov3D, float* dL_dsh_dc,
                     float* dL_dsh_ac, float* dL_dsvec, float* dL_dquaternion, float* dens_accum,
                             float* dens_counter, w2w_stream_t stream) {
  if (!settings_ok(s) || s->M < 1 || s->M > 16) return W2W_ERR_INVALID;
  const int P = s->P;
  if (P == 0) return W2W_OK;
  if (!means3D || !svec || !quaternion || !opacity_logit || !sh_dc || (s->M > 1 && (!sh_ac || !dL_dsh_ac)) ||
      !radii || !geom_state || !image_state || !out_alpha || !dL_dcolor ||
      !dL_dmeans2D || !dL_dcolors || !dL_dopacity_logit || !dL_dmeans3D || !dL_dcov3D || !dL_dsh_dc || !dL_dsvec ||
      !dL_dquaternion || (R > 0 && !binning_state))
    return W2W_ERR_INVALID;
  if ((dens_accum == nullptr) != (dens_counter == nullptr)) return W2W_ERR_INVALID;
  const RawGrads raw{svec, quaternion, opacity_logit, sh_dc, sh_ac, dL_dsh_dc, dL_dsh_ac, dens_accum, dens_counter};
  return backward_impl(s, means3D, nullptr, nullptr, nullptr, &raw, radii, geom_state, R, binning_state, image_state,
                       out_alpha, dL_dcolor, dL_ddepth, dL_dalpha, 0, scratch, scratch_bytes, dL_dmeans2D,
                       dL_dcolors, dL_dopacity_logit, dL_dmeans3D, dL_dcov3D, nullptr, dL_dsvec, dL_dquaternion,
                       stream);
}

int w2w_backward_raw(const w2w_settings* s, const float* means3D, const float* svec, const float* quaternion,
                     const float* opacity_logit, const float* sh_dc, const float* sh_ac, const int* radii,
                     const void* geom_state, long long R, const void* binning_state, const void* image_state,
                     const float* out_alpha, const float* dL_dcolor, const float* dL_ddepth, const float* dL_dalpha,
                     void* scratch, size_t scratch_bytes, float* dL_dmeans2D, float* dL_dcolors,
                     float* dL_dopacity_logit, float* dL_dmeans3D, float* dL_dcov3D, float* dL_dsh_dc,
                     float* dL_dsh_ac, float* dL_dsvec, float* dL_dquaternion, w2w_stream_t stream) {
  return w2w_backward_raw_densify(s, means3D, svec, quaternion, opacity_logit, sh_dc, sh_ac, radii, geom_state, R,
                                  binning_state, image_state, out_alpha, dL_dcolor, dL_ddepth, dL_dalpha, scratch,
                                  scratch_bytes, dL_dmeans2D, dL_dcolors, dL_dopacity_logit, dL_dmeans3D, dL_dcov3D,
                                  dL_dsh_dc, dL_dsh_ac, dL_dsvec, dL_dquaternion, nullptr, nullptr, stream);
}

size_t w2w_sort_scratch_bytes(long long n) {
  size_t a, b, c, d, e, f;
  return sort_scratch_layout(n, &a, &b, &c, &d, &e, &f);
}

int w2w_sort_pairs_u64(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out, uint32_t* vals_out,
                       long long n, int begin_bit, int end_bit, void* scratch, size_t scratch_bytes,
                       w2w_stream_t stream) {
  if (n < 0 || begin_bit < 0 || end_bit > 64 || end_bit < begin_bit) return W2W_ERR_INVALID;
  if (n == 0) return W2W_OK;
  if (!keys_in || !vals_in || !keys_out || !vals_out || keys_in == keys_out || vals_in == vals_out)
    return W2W_ERR_INVALID;
  if (n >= (1LL << 30)) return W2W_ERR_CAPACITY;
  size_t kt, vt, hi, stt, ct, er;
  const size_t need = sort_scratch_layout(n, &kt, &vt, &hi, &stt, &ct, &er);
  if (!scratch || scratch_bytes < need) return W2W_ERR_SCRATCH;
  cudaStream_t st = S(stream);
  cudaMemsetAsync(at<uint32_t>(scratch, er), 0, 4, st);
  SortArgs so{};
  so.n = n; so.key64 = 1; so.begin_bit = begin_bit; so.bits = end_bit - begin_bit;
  so.keys_in = keys_in; so.vals_in = vals_in;
  so.keys_out = keys_out; so.vals_out = vals_out;
  so.keys_tmp = at<void>(scratch, kt); so.vals_tmp = at<uint32_t>(scratch, vt);
  so.hist = at<uint32_t>(scratch, hi);
  so.status = at<uint32_t>(scratch, stt);
  so.counters = at<uint32_t>(scratch, ct);
  so.error = at<uint32_t>(scratch, er);
  so.tile_shift = 0; so.num_tiles = 0; so.tile_hist = nullptr; so.ranges = nullptr;
  so.spin_limit = spin_limit();
  so.unpublished_tile = unpublished_tile(kWaitSort);
  launch_sort(so, st);
  return finish(so.error, st);
}

size_t w2w_scan_scratch_bytes(long long n) { return align256(scan_scratch_bytes(n)); }

int w2w_scan_u32(const uint32_t* in, uint32_t* out, long long n, int exclusive, void* scratch,
                 size_t scratch_bytes, w2w_stream_t stream) {
  if (n < 0) return W2W_ERR_INVALID;
  if (n == 0) return W2W_OK;
  if (!in || !out) return W2W_ERR_INVALID;
  if (!scratch || scratch_bytes < w2w_scan_scratch_bytes(n)) return W2W_ERR_SCRATCH;
  launch_scan(in, out, n, exclusive, scratch, S(stream));
  return finish(static_cast<unsigned char*>(scratch) + 4, S(stream));
}

int w2w_scan_u32_noalloc(const uint32_t* in, uint32_t* out, long long n, int exclusive, w2w_stream_t stream) {
  if (n < 0) return W2W_ERR_INVALID;
  if (n == 0) return W2W_OK;
  if (!in || !out) return W2W_ERR_INVALID;
  if (n > scan_noalloc_max()) {
    std::fprintf(stderr,
                 "w2w_scan_u32_noalloc: %lld elements exceed the %lld this entry point's fixed scratch holds; "
                 "use w2w_scan_u32 with a caller-provided scratch buffer\n",
                 n, scan_noalloc_max());
    return W2W_ERR_CAPACITY;
  }
  int rc = 0;
  void* scratch = scan_noalloc_scratch(&rc);
  if (rc != 0 || scratch == nullptr) return W2W_ERR_CUDA;
  launch_scan(in, out, n, exclusive, scratch, S(stream));
  return finish(static_cast<unsigned char*>(scratch) + 4, S(stream));
}

int w2w_activate_forward(long long P, int K, const float* opacity_logit, const float* svec, const float* quaternion,
                         const float* sh_dc, const float* sh_ac, float* opacity, float* scales, float* rotations,
                         float* shs, w2w_stream_t stream) {
  if (P < 0 || K < 0) return W2W_ERR_INVALID;
  if (P * 3 * (K + 1LL) >= (1LL << 31)) return W2W_ERR_CAPACITY;
  if (P == 0) return W2W_OK;
  if (!opacity_logit || !svec || !quaternion || !sh_dc || (K > 0 && !sh_ac) || !opacity || !scales ||
      !rotations || !shs)
    return W2W_ERR_INVALID;
  ActivateArgs a{P, K, opacity_logit, svec, quaternion, sh_dc, sh_ac, opacity, scales, rotations, shs};
  launch_activate(a, S(stream));
  return check_launch();
}

int w2w_activate_backward(long long P, int K, const float* g_opacity, const float* g_scales,
                          const float* g_rotations, const float* g_shs, const float* opacity, const float* scales,
                          const float* quaternion, float* d_opacity_logit, float* d_svec, float* d_quaternion,
                          float* d_sh_dc, float* d_sh_ac, w2w_stream_t stream) {
  if (P < 0 || K < 0) return W2W_ERR_INVALID;
  if (P * 3 * (K + 1LL) >= (1LL << 31)) return W2W_ERR_CAPACITY;
  if (P == 0) return W2W_OK;
  if (!g_opacity || !g_scales || !g_rotations || !g_shs || !opacity || !scales || !quaternion ||
      !d_opacity_logit || !d_svec || !d_quaternion || !d_sh_dc || (K > 0 && !d_sh_ac))
    return W2W_ERR_INVALID;
  ActivateBackwardArgs a{P, K, g_opacity, g_scales, g_rotations, g_shs, opacity, scales, quaternion,
                         d_opacity_logit, d_svec, d_quaternion, d_sh_dc, d_sh_ac};
  launch_activate_backward(a, S(stream));
  return check_launch();
}

int w2w_voxel_field(const float* means, const float* covs, const float* opacities, int n, int resolution,
                    int num_blocks, float relax_ratio, float* occ, w2w_stream_t stream) {
  if (n < 0 || resolution < 2 || resolution > 2048 || num_blocks < 1 || num_blocks > 1000 ||
      !(relax_ratio >= 0.0f && relax_ratio <= 64.0f) || !occ)
    return W2W_ERR_INVALID;
  if (n > 0 && (!means || !covs || !opacities)) return W2W_ERR_INVALID;
  cudaStream_t st = S(stream);
  const size_t voxels = size_t(resolution) * resolution * resolution;
  if (n == 0) {
    cudaMemsetAsync(occ, 0, voxels * 4, st);
    return check_launch();
  }
  const int nb = num_blocks + 1;  // the last voxel of an axis falls in block num_blocks
  const int nblocks = nb * nb * nb;
  std::vector<void*> bufs;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMallocAsync(&p, bytes > 0 ? bytes : 1, st) != cudaSuccess) return nullptr;
    bufs.push_back(p);
    return p;
  };
  auto release = [&]() {
    for (void* p : bufs) cudaFreeAsync(p, st);
    bufs.clear();
  };
  VoxelArgs a{};
  a.P = n; a.R = resolution; a.B = num_blocks;
  a.bs = 2.0f / float(num_blocks);
  a.relax = relax_ratio;
  a.means = means; a.covs = covs; a.opacities = opacities; a.occ = occ;
  a.rec = static_cast<float4*>(alloc(size_t(n) * 48));
  a.count = static_cast<uint32_t*>(alloc(size_t(n) * 4));
  uint32_t* offsets = static_cast<uint32_t*>(alloc(size_t(n) * 4));
  void* scan_scratch = alloc(scan_scratch_bytes(n));
  if (!a.rec || !a.count || !offsets || !scan_scratch) { release(); return W2W_ERR_CUDA; }
  a.offsets = offsets;
  launch_voxel_prepare(a, st);
  launch_scan(a.count, offsets, n, 1, scan_scratch, st);
  uint32_t tail[2] = {0, 0};
  cudaMemcpyAsync(&tail[0], offsets + (n - 1), 4, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&tail[1], a.count + (n - 1), 4, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) { release(); return check_launch(); }
  const long long pairs = (long long)tail[0] + tail[1];
  if (pairs >= (1LL << 30)) { release(); return W2W_ERR_CAPACITY; }
  if (pairs == 0) {
    cudaMemsetAsync(occ, 0, voxels * 4, st);
    release();
    return check_launch();
  }
  a.keys = static_cast<uint32_t*>(alloc(size_t(pairs) * 4));
  a.vals = static_cast<uint32_t*>(alloc(size_t(pairs) * 4));
  uint32_t* keys_out = static_cast<uint32_t*>(alloc(size_t(pairs) * 4));
  uint32_t* vals_out = static_cast<uint32_t*>(alloc(size_t(pairs) * 4));
  size_t kt, vt, hi, stt, ct, er;
  const size_t sbytes = sort_scratch_layout(pairs, &kt, &vt, &hi, &stt, &ct, &er);
  void* sort_scratch = alloc(sbytes);
  uint32_t* tile_hist = static_cast<uint32_t*>(alloc(size_t(nblocks) * 4));
  uint2* ranges = static_cast<uint2*>(alloc(size_t(nblocks) * 8));
  if (!a.keys || !a.vals || !keys_out || !vals_out || !sort_scratch || !tile_hist || !ranges) {
    release();
    return W2W_ERR_CUDA;
  }
  launch_voxel_emit(a, st);
  cudaMemsetAsync(at<uint32_t>(sort_scratch, er), 0, 4, st);
  SortArgs so{};
  so.n = pairs; so.key64 = 0; so.begin_bit = 0; so.bits = ceil_log2(uint32_t(nblocks));
  so.keys_in = a.keys; so.vals_in = a.vals; so.keys_out = keys_out; so.vals_out = vals_out;
  so.keys_tmp = at<void>(sort_scratch, kt); so.vals_tmp = at<uint32_t>(sort_scratch, vt);
  so.hist = at<uint32_t>(sort_scratch, hi); so.status = at<uint32_t>(sort_scratch, stt);
  so.counters = at<uint32_t>(sort_scratch, ct); so.error = at<uint32_t>(sort_scratch, er);
  so.tile_shift = 0; so.num_tiles = nblocks; so.tile_hist = tile_hist; so.ranges = ranges;
  so.spin_limit = spin_limit();
  so.unpublished_tile = unpublished_tile(kWaitSort);
  launch_sort(so, st);
  launch_voxel_field(a, vals_out, ranges, st);
  uint32_t err = 0;
  cudaMemcpyAsync(&err, so.error, 4, cudaMemcpyDeviceToHost, st);
  const cudaError_t se = cudaStreamSynchronize(st);
  release();
  if (se != cudaSuccess) return check_launch();
  if (err & kErrTimeout) return W2W_ERR_TIMEOUT;
  if (err) return W2W_ERR_CAPACITY;
  return check_launch();
}

int w2w_compute_voxel_field(float* h_occ, const float* h_means, const float* h_covs, const float* h_opacities,
                            int n, int resolution, int num_blocks, float relax_ratio) {
  if (!h_occ || n < 0 || resolution < 2 || resolution > 2048 || (n > 0 && (!h_means || !h_covs || !h_opacities)))
    return W2W_ERR_INVALID;
  const size_t voxels = size_t(resolution) * resolution * resolution;
  float *d_occ = nullptr, *d_in = nullptr;
  if (cudaMalloc(&d_occ, voxels * 4) != cudaSuccess) return W2W_ERR_CUDA;
  const size_t nn = size_t(n);
  if (cudaMalloc(&d_in, (nn * 10 > 0 ? nn * 10 : 1) * 4) != cudaSuccess) {
    cudaFree(d_occ);
    return W2W_ERR_CUDA;
  }
  if (n > 0) {
    cudaMemcpy(d_in, h_means, nn * 12, cudaMemcpyHostToDevice);
    cudaMemcpy(d_in + 3 * nn, h_covs, nn * 24, cudaMemcpyHostToDevice);
    cudaMemcpy(d_in + 9 * nn, h_opacities, nn * 4, cudaMemcpyHostToDevice);
  }
  int rc = w2w_voxel_field(d_in, d_in + 3 * nn, d_in + 9 * nn, n, resolution, num_blocks, relax_ratio, d_occ,
                           nullptr);
  if (rc == W2W_OK && cudaMemcpy(h_occ, d_occ, voxels * 4, cudaMemcpyDeviceToHost) != cudaSuccess) rc = W2W_ERR_CUDA;
  cudaFree(d_occ);
  cudaFree(d_in);
  return rc;
}

int w2w_group_sum(const float* src, int width, int num_groups, const uint32_t* tables, int num_items, float* dst,
                  long long total_rows, w2w_stream_t stream) {
  if (width <= 0 || num_groups < 0 || num_items < 0 || total_rows < 0) return W2W_ERR_INVALID;
  if (num_groups == 0 || total_rows == 0) return W2W_OK;
  if (!src || !tables || !dst) return W2W_ERR_INVALID;
  launch_group_sum(src, width, num_groups, tables, num_items, dst, total_rows, S(stream));
  return check_launch();
}

int w2w_densification_stats(long long P, const float* dL_dmeans2D, const int* radii, float* accum, float* counter,
                            w2w_stream_t stream) {
  if (P < 0) return W2W_ERR_INVALID;
  if (P == 0) return W2W_OK;
  if (!dL_dmeans2D || !radii || !accum || !counter) return W2W_ERR_INVALID;
  launch_densify_stats(P, dL_dmeans2D, radii, accum, counter, S(stream));
  return check_launch();
}

int w2w_tile_ranges(const uint64_t* sorted_keys, long long n, int tile_shift, uint32_t* ranges, int ntiles,
                    w2w_stream_t stream) {
  if (n < 0 || ntiles <= 0 || !ranges || (n > 0 && !sorted_keys) || tile_shift < 0 || tile_shift > 63)
    return W2W_ERR_INVALID;
  cudaStream_t st = S(stream);
  cudaMemsetAsync(ranges, 0, sizeof(uint2) * size_t(ntiles), st);
  if (n > 0) {
    stage_begin(kStOther, st);
    ranges_from_sorted<<<int((n + 255) / 256), 256, 0, st>>>(sorted_keys, n, tile_shift,
                                                              reinterpret_cast<uint2*>(ranges), ntiles);
    stage_end(kStOther, st, 1);
  }
  return check_launch();
}

int w2w_blend(const w2w_settings* s, const void* geom_state, const uint32_t* ranges, const uint32_t* point_list,
              void* image_state, float* out_color, float* out_depth, float* out_alpha, w2w_stream_t stream) {
  if (!settings_ok(s) || !geom_state || !ranges || !image_state || !out_color || !out_depth || !out_alpha)
    return W2W_ERR_INVALID;
  const ImageLayout IL(s->width, s->height);
  // keep the ranges in the image state so it is complete for a backward pass
  uint2* own = at<uint2>(image_state, IL.ranges);
  if (reinterpret_cast<const void*>(own) != reinterpret_cast<const void*>(ranges))
    cudaMemcpyAsync(own, ranges, sizeof(uint2) * size_t(num_tiles(s->width, s->height)), cudaMemcpyDeviceToDevice,
                    S(stream));
  BlendArgs b{};
  b.W = s->width; b.H = s->height;
  b.ranges = own;
  b.point_list = point_list;
  b.record = at<float>(geom_state, GeomLayout(s->P).record);
  b.num_records = uint32_t(s->P);
  b.bg = s->background;
  b.out_color = out_color; b.out_depth = out_depth; b.out_alpha = out_alpha;
  b.n_contrib = at<uint32_t>(image_state, IL.n_contrib);
  b.T_final = at<float>(image_state, IL.T_final);
  b.tile_max = at<uint32_t>(image_state, IL.tile_max);
  b.order = at<uint32_t>(image_state, IL.order);
  b.order_bwd = at<uint32_t>(image_state, IL.order_bwd);
  b.queue = at<uint32_t>(image_state, IL.queue);
  b.spin_limit = spin_limit();
  launch_blend(b, S(stream));
  return check_launch();
}

int w2w_binning_keys64_layout(const void* binning_state, long long R, long long layout_count, int W, int H,
                              uint64_t* out, w2w_stream_t stream) {
  if (R < 0 || layout_count < R || !out || (R > 0 && !binning_state)) return W2W_ERR_INVALID;
  if (R == 0) return W2W_OK;
  const BinLayout BL(layout_count, num_tiles(W, H));
  const BinHeader* h = at<BinHeader>(binning_state, BL.header);
  BinHeader hh;
  cudaStream_t st = S(stream);
  if (cudaMemcpyAsync(&hh, h, sizeof(hh), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return W2W_ERR_CUDA;
  const int blocks = int((R + 255) / 256);
  stage_begin(kStOther, st);
  if (hh.key64) expand_keys<uint64_t><<<blocks, 256, 0, st>>>(h, at<uint64_t>(binning_state, BL.keysA), R, out);
  else expand_keys<uint32_t><<<blocks, 256, 0, st>>>(h, at<uint32_t>(binning_state, BL.keysA), R, out);
  stage_end(kStOther, st, 1);
  return check_launch();
}

int w2w_binning_keys64(const void* binning_state, long long R, int W, int H, uint64_t* out, w2w_stream_t stream) {
  return w2w_binning_keys64_layout(binning_state, R, R, W, H, out, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched calls: many views of many scenes in one launch per stage.  Items'
// elements (per-view copies of their scene's Gaussians), tiles and pixels are
// laid out back to back; keys are (global tile, depth) so one sort serves all
// items and each tile's list is exactly the one its item alone would give.
// ---------------------------------------------------------------------------
namespace {

struct BatchTotals {
  long long elems = 0, pixels = 0;
  int tiles = 0, M = -1;
  bool ok = true;
};

BatchTotals batch_totals(const w2w_batch_item* items, int n) {
  BatchTotals t;
  if (!items || n <= 0) { t.ok = false; return t; }
  for (int v = 0; v < n; ++v) {
    const w2w_batch_item& it = items[v];
    if (it.P < 0 || it.width <= 0 || it.height <= 0 || it.M < 0 || it.degree < 0 || it.width >= 65535 * kTile ||
        it.height >= 65535 * kTile || (it.P > 0 && (!it.means3D || !it.scales || !it.rotations || !it.opacities ||
                                                      (it.M > 0 && !it.shs)))) {
      t.ok = false;
      return t;
    }
    if (t.M < 0) t.M = it.M;
    if (it.M != t.M) { t.ok = false; return t; }  // one SH row length per batch
    t.elems += it.P;
    t.pixels += (long long)it.width * it.height;
    t.tiles += num_tiles(it.width, it.height);
  }
  if (t.elems >= (1LL << 30) || t.tiles >= (1 << 30)) t.ok = false;
  return t;
}

struct BatchGeomLayout {
  size_t items, item_end, total;
  BatchGeomLayout(long long E, int n) {
    const size_t g = GeomLayout(E).total;
    items = g;
    item_end = align256(items + size_t(n) * sizeof(BatchItem));
    total = align256(item_end + size_t(n) * 4);
  }
};

std::vector<BatchItem> device_items(const w2w_batch_item* items, int n) {
  std::vector<BatchItem> d(static_cast<size_t>(n));
  uint32_t eb = 0, tb = 0;
  unsigned long long pb = 0;
  for (int v = 0; v < n; ++v) {
    const w2w_batch_item& it = items[v];
    BatchItem& b = d[size_t(v)];
    std::memset(&b, 0, sizeof(b));
    b.means3D = it.means3D; b.scales = it.scales; b.rotations = it.rotations; b.opacities = it.opacities;
    b.shs = it.shs;
    b.P = it.P; b.M = it.M; b.degree = it.degree; b.W = it.width; b.H = it.height;
    b.gw = tiles_x(it.width);
    b.tiles = num_tiles(it.width, it.height);
    b.focal_x = it.focal_x; b.tan_fovx = it.tan_fovx; b.tan_fovy = it.tan_fovy;
    b.scale_modifier = it.scale_modifier;
    b.h_x = float(it.width) / (2.0f * it.tan_fovx);
    b.h_y = float(it.height) / (2.0f * it.tan_fovy);
    std::memcpy(b.view, it.viewmatrix, sizeof(b.view));
    std::memcpy(b.proj, it.projmatrix, sizeof(b.proj));
    std::memcpy(b.campos, it.campos, 3 * sizeof(float));
    std::memcpy(b.bg, it.background, 3 * sizeof(float));
    b.elem_base = eb;
    b.tile_base = tb;
    b.pix_base = pb;
    eb += uint32_t(it.P);
    tb += uint32_t(b.tiles);
    pb += (unsigned long long)it.width * it.height;
  }
  return d;
}

}  // namespace

extern "C" {

size_t w2w_batch_geometry_state_bytes(const w2w_batch_item* items, int n) {
  const BatchTotals t = batch_totals(items, n);
  return t.ok ? BatchGeomLayout(t.elems, n).total : 0;
}

size_t w2w_batch_image_state_bytes(const w2w_batch_item* items, int n) {
  const BatchTotals t = batch_totals(items, n);
  return t.ok ? ImageLayout(size_t(t.pixels), size_t(t.tiles)).total : 0;
}

size_t w2w_batch_binning_state_bytes(long long R, const w2w_batch_item* items, int n) {
  const BatchTotals t = batch_totals(items, n);
  return (t.ok && R >= 0) ? BinLayout(R, t.tiles).total : 0;
}

size_t w2w_batch_backward_scratch_bytes(const w2w_batch_item* items, int n) {
  const BatchTotals t = batch_totals(items, n);
  return t.ok ? align256(size_t(t.elems) * 16) + align256(size_t(t.elems) * 4) : 0;
}

int w2w_batch_forward_geometry(const w2w_batch_item* items, int n, int compat_spill, int* radii, void* geom_state,
                               w2w_geometry_info* info, w2w_stream_t stream) {
  const BatchTotals t = batch_totals(items, n);
  if (!t.ok || !info || !geom_state || (t.elems > 0 && !radii)) return W2W_ERR_INVALID;
  std::memset(info, 0, sizeof(*info));
  const long long E = t.elems;
  const GeomLayout L(E);
  const BatchGeomLayout BL(E, n);
  cudaStream_t st = S(stream);
  const std::vector<BatchItem> host = device_items(items, n);
  BatchItem* dev_items = at<BatchItem>(geom_state, BL.items);
  if (cudaMemcpyAsync(dev_items, host.data(), sizeof(BatchItem) * size_t(n), cudaMemcpyHostToDevice, st) !=
      cudaSuccess)
    return W2W_ERR_CUDA;
  if (E == 0) return W2W_OK;
  cudaMemsetAsync(geom_state, 0, L.depth, st);  // header + scan status
  cudaMemsetAsync(at<uint32_t>(geom_state, BL.item_end), 0, size_t(n) * 4, st);
  PreprocessArgs a{};
  a.P = int(E); a.compat_spill = compat_spill;
  a.items = dev_items; a.num_items = n; a.item_end = at<uint32_t>(geom_state, BL.item_end);
  // the 16-coefficient vector path needs every item's rows 16-byte aligned
  bool sh16 = t.M == 16;
  for (int v = 0; v < n && sh16; ++v)
    if (items[v].P > 0 && (reinterpret_cast<uintptr_t>(items[v].shs) & 15) != 0) sh16 = false;
  a.M = sh16 ? 16 : 0;
  a.shs = sh16 ? items[0].shs : nullptr;
  a.radii = radii;
  a.header = at<GeomHeader>(geom_state, L.header);
  a.scan_status = at<unsigned long long>(geom_state, L.scan_status);
  a.depth = at<float>(geom_state, L.depth);
  a.clamped = at<uint8_t>(geom_state, L.clamped);
  a.means2D = at<float>(geom_state, L.means2D);
  a.cov3D = at<float>(geom_state, L.cov3D);
  a.conic = at<float>(geom_state, L.conic);
  a.rgb = at<float>(geom_state, L.rgb);
  a.tiles = at<uint32_t>(geom_state, L.tiles);
  a.offsets = at<uint32_t>(geom_state, L.offsets);
  a.rect = at<uint32_t>(geom_state, L.rect);
  a.prev_reach = at<uint32_t>(geom_state, L.prev_reach);
  a.record = at<float>(geom_state, L.record);
  a.bwd_record = at<float>(geom_state, L.bwd_record);
  a.spin_limit = spin_limit();
  a.unpublished_tile = unpublished_tile(kWaitPreprocess);
  launch_preprocess(a, st);
  int rc = check_launch();
  if (rc) return rc;
  GeomHeader h;
  if (cudaMemcpyAsync(&h, a.header, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return W2W_ERR_CUDA;
  info->num_rendered = h.num_rendered;
  info->depth_min_bits = ~h.depth_min;
  info->depth_max_bits = h.depth_max;
  info->error = h.error;
  if (h.error & kErrTimeout) return W2W_ERR_TIMEOUT;
  if (h.error & kErrCapacity) return W2W_ERR_CAPACITY;
  return W2W_OK;
}

int w2w_batch_forward_render(const w2w_batch_item* items, int n, const void* geom_state,
                             const w2w_geometry_info* info, void* binning_state, void* image_state, float* out_color,
                             float* out_depth, float* out_alpha, w2w_stream_t stream) {
  const BatchTotals t = batch_totals(items, n);
  if (!t.ok || !info || !geom_state || !image_state || !out_color || !out_depth || !out_alpha) return W2W_ERR_INVALID;
  const long long R = info->num_rendered;
  if (R < 0 || R >= (1LL << 30)) return W2W_ERR_CAPACITY;
  if (R > 0 && !binning_state) return W2W_ERR_INVALID;
  cudaStream_t st = S(stream);
  const long long E = t.elems;
  const int T = t.tiles;
  const ImageLayout IL(size_t(t.pixels), size_t(T));
  const BatchGeomLayout BGL(E, n);
  const BatchItem* dev_items = at<BatchItem>(geom_state, BGL.items);
  uint2* ranges = at<uint2>(image_state, IL.ranges);
  const uint32_t* point_list = nullptr;
  const void* err_word = nullptr;  // the binning header's error word
  if (R == 0) {
    cudaMemsetAsync(ranges, 0, sizeof(uint2) * size_t(T), st);
  } else {
    const GeomLayout GL(E);
    const BinLayout BL(R, T);
    const KeyPlan kp = plan_keys_tiles(*info, T);
    const int passes = sort_passes(kp.bits);
    BinHeader* bh = at<BinHeader>(binning_state, BL.header);
    err_word = &bh->error;
    stage_begin(kStOther, st);
    write_bin_header<<<1, 1, 0, st>>>(bh, kp, uint32_t(R), uint32_t(passes), nullptr, nullptr);
    stage_end(kStOther, st, 1);
    const bool odd = (passes % 2) == 1;
    void* keysA = at<void>(binning_state, BL.keysA);
    void* keysB = at<void>(binning_state, BL.keysB);
    uint32_t* valsA = at<uint32_t>(binning_state, BL.valsA);
    uint32_t* valsB = at<uint32_t>(binning_state, BL.valsB);
    DuplicateArgs d{};
    d.P = int(E); d.gw = 0; d.R = uint32_t(R); d.key64 = kp.key64; d.depth_bits = uint32_t(kp.depth_bits);
    d.items = dev_items; d.num_items = n; d.item_end = at<uint32_t>(geom_state, BGL.item_end);
    d.tiles = at<uint32_t>(geom_state, GL.tiles);
    d.offsets = at<uint32_t>(geom_state, GL.offsets);
    d.rect = at<uint32_t>(geom_state, GL.rect);
    d.prev_reach = at<uint32_t>(geom_state, GL.prev_reach);
    d.depth = at<float>(geom_state, GL.depth);
    d.keys = odd ? keysB : keysA;
    d.vals = odd ? valsB : valsA;
    launch_duplicate(d, st);
    SortArgs so{};
    so.n = R; so.key64 = kp.key64; so.begin_bit = 0; so.bits = kp.bits;
    so.keys_in = d.keys; so.vals_in = d.vals;
    so.match_rank = 1;  // emitted Gaussian by Gaussian: few distinct digits per warp
    so.keys_out = keysA; so.vals_out = valsA;
    so.keys_tmp = keysB; so.vals_tmp = valsB;
    so.hist = at<uint32_t>(binning_state, BL.hist);
    so.status = at<uint32_t>(binning_state, BL.status);
    so.counters = bh->tile_counter;
    so.error = &bh->error;
    so.tile_shift = kp.depth_bits;
    so.num_tiles = T;
    so.tile_hist = at<uint32_t>(binning_state, BL.tile_hist);
    so.ranges = ranges;
    // hist, tile_hist and the used status words are contiguous; the tile
    // counters were cleared by write_bin_header
    so.clear_span = at<void>(binning_state, BL.hist);
    so.clear_bytes = BL.status - BL.hist + size_t(passes > 0 ? passes : 1) * kMaxBins * 4 *
                     size_t((R + sort_tile_keys(kp.key64) - 1) / sort_tile_keys(kp.key64));
    so.spin_limit = spin_limit();
    so.unpublished_tile = unpublished_tile(kWaitSort);
    launch_sort(so, st);
    point_list = valsA;
  }
  BlendArgs b{};
  b.W = 0; b.H = 0;
  b.items = dev_items; b.num_items = n; b.total_tiles = T;
  b.ranges = ranges;
  b.point_list = point_list;
  b.record = R > 0 ? at<float>(geom_state, GeomLayout(E).record) : nullptr;
  b.num_records = uint32_t(E);
  if (R > 0) {
    const BinLayout BL(R, T);
    b.mask_top = at<uint8_t>(binning_state, BL.masks);
    b.mask_bottom = b.mask_top + R;
    b.masks_valid = &at<BinHeader>(binning_state, BL.header)->masks_valid;
  }
  b.bg = nullptr;
  b.out_color = out_color; b.out_depth = out_depth; b.out_alpha = out_alpha;
  b.n_contrib = at<uint32_t>(image_state, IL.n_contrib);
  b.T_final = at<float>(image_state, IL.T_final);
  b.tile_max = at<uint32_t>(image_state, IL.tile_max);
  b.order = at<uint32_t>(image_state, IL.order);
  b.order_bwd = at<uint32_t>(image_state, IL.order_bwd);
  b.queue = at<uint32_t>(image_state, IL.queue);
  b.error = const_cast<uint32_t*>(static_cast<const uint32_t*>(err_word));
  b.spin_limit = spin_limit();
  launch_blend(b, st);
  return finish(err_word, st);
}

// The per-Gaussian pass's arguments of a batched backward: the item table and
// geometry state, and the per-element accumulators the per-pixel pass fills
// (acc_cov and acc_depth in the scratch; dL_dmeans2D, dL_dcolors, dL_dopacity).
static void batch_gaussian_args(int n, long long E, int M, const void* geom_state, const int* radii, int grad_mode,
                                void* scratch, float* dL_dmeans2D, float* dL_dcolors, float* dL_dopacity,
                                BackwardArgs& a) {
  const GeomLayout GL(E);
  const BatchGeomLayout BGL(E, n);
  a = BackwardArgs{};
  a.P = int(E); a.W = 0; a.H = 0; a.degree = 0; a.M = M; a.grad_mode = grad_mode;
  a.items = at<BatchItem>(geom_state, BGL.items); a.num_items = n;
  a.shs = nullptr;
  a.radii = radii;
  a.cov3D = at<float>(geom_state, GL.cov3D);
  a.clamped = at<uint8_t>(geom_state, GL.clamped);
  a.record = at<float>(geom_state, GL.record);
  a.bwd_record = at<float>(geom_state, GL.bwd_record);
  a.dL_dmean2D = dL_dmeans2D; a.dL_dopacity = dL_dopacity; a.dL_dcolors = dL_dcolors;
  a.acc_cov = static_cast<float*>(scratch);
  a.acc_depth = at<float>(scratch, align256(size_t(E) * 16));
}

// The batched backward's common part: argument checks, the per-element
// accumulators cleared, the per-pixel pass launched; `a` is left ready for a
// per-Gaussian pass.  Returns W2W_OK, an error, or 1 when there is no element.
static int batch_backward_begin(const w2w_batch_item* items, int n, const void* geom_state, long long R,
                                const void* binning_state, const void* image_state, const int* radii,
                                const float* out_alpha, const float* dL_dcolor, const float* dL_ddepth,
                                const float* dL_dalpha, int grad_mode, void* scratch, size_t scratch_bytes,
                                float* dL_dmeans2D, float* dL_dcolors, float* dL_dopacity, cudaStream_t st,
                                BackwardArgs& a) {
  const BatchTotals t = batch_totals(items, n);
  if (!t.ok || (grad_mode != 0 && grad_mode != 1)) return W2W_ERR_INVALID;
  const long long E = t.elems;
  if (E == 0) return 1;
  // dL_ddepth / dL_dalpha may be null: no loss reaches depth / alpha (read as zero)
  if (!geom_state || !image_state || !radii || !out_alpha || !dL_dcolor || !dL_dmeans2D || !dL_dcolors ||
      !dL_dopacity || (R > 0 && !binning_state))
    return W2W_ERR_INVALID;
  if (!scratch || scratch_bytes < w2w_batch_backward_scratch_bytes(items, n)) return W2W_ERR_SCRATCH;
  const int T = t.tiles;
  const ImageLayout IL(size_t(t.pixels), size_t(T));
  cudaMemsetAsync(scratch, 0, w2w_batch_backward_scratch_bytes(items, n), st);
  cudaMemsetAsync(dL_dmeans2D, 0, sizeof(float) * 3 * size_t(E), st);
  cudaMemsetAsync(dL_dcolors, 0, sizeof(float) * 3 * size_t(E), st);
  cudaMemsetAsync(dL_dopacity, 0, sizeof(float) * size_t(E), st);
  batch_gaussian_args(n, E, t.M, geom_state, radii, grad_mode, scratch, dL_dmeans2D, dL_dcolors, dL_dopacity, a);
  a.total_tiles = T;
  a.ranges = at<uint2>(image_state, IL.ranges);
  a.point_list = R > 0 ? at<uint32_t>(binning_state, BinLayout(R, T).valsA) : nullptr;
  if (R > 0) {
    const BinLayout BL(R, T);
    a.mask_top = at<uint8_t>(binning_state, BL.masks);
    a.mask_bottom = a.mask_top + R;
    a.masks_valid = &at<BinHeader>(binning_state, BL.header)->masks_valid;
  }
  a.n_contrib = at<uint32_t>(image_state, IL.n_contrib);
  a.tile_max = at<uint32_t>(image_state, IL.tile_max);
  a.order_bwd = at<uint32_t>(image_state, IL.order_bwd);
  a.T_final = at<float>(image_state, IL.T_final);
  a.out_alpha = out_alpha;
  a.dL_dcolor = dL_dcolor; a.dL_ddepth = dL_ddepth; a.dL_dalpha = dL_dalpha;
  if (R > 0) launch_backward_render(a, st);
  return W2W_OK;
}

// The grouped outputs' arguments (both grouped entry points).
static bool group_outputs_ok(const BatchTotals& t, const uint32_t* group_tables, int num_groups, long long group_rows,
                             const float* g_means3D, const float* g_opacity, const float* g_scales,
                             const float* g_rotations, const float* g_sh) {
  return group_tables && num_groups > 0 && group_rows > 0 && group_rows <= t.elems && g_means3D && g_opacity &&
         g_scales && g_rotations && (t.M == 0 || g_sh);
}

static void set_group_outputs(BackwardArgs& a, const uint32_t* group_tables, int num_groups, long long group_rows,
                              float* g_means3D, float* g_opacity, float* g_scales, float* g_rotations, float* g_sh) {
  a.group_tables = group_tables; a.num_groups = num_groups; a.group_rows = group_rows;
  a.g_means3D = g_means3D; a.g_opacity = g_opacity; a.g_scales = g_scales; a.g_rotations = g_rotations;
  a.g_sh = g_sh;
}

int w2w_batch_backward(const w2w_batch_item* items, int n, const void* geom_state, long long R,
                       const void* binning_state, const void* image_state, const int* radii, const float* out_alpha,
                       const float* dL_dcolor, const float* dL_ddepth, const float* dL_dalpha, int grad_mode,
                       void* scratch, size_t scratch_bytes, float* dL_dmeans2D, float* dL_dcolors, float* dL_dopacity,
                       float* dL_dmeans3D, float* dL_dcov3D, float* dL_dsh, float* dL_dscales, float* dL_drotations,
                       w2w_stream_t stream) {
  const BatchTotals t = batch_totals(items, n);
  if (t.ok && t.elems > 0 && (!dL_dmeans3D || !dL_dcov3D || !dL_dscales || !dL_drotations || (t.M > 0 && !dL_dsh)))
    return W2W_ERR_INVALID;
  BackwardArgs a;
  const int rc = batch_backward_begin(items, n, geom_state, R, binning_state, image_state, radii, out_alpha,
                                      dL_dcolor, dL_ddepth, dL_dalpha, grad_mode, scratch, scratch_bytes,
                                      dL_dmeans2D, dL_dcolors, dL_dopacity, S(stream), a);
  if (rc != W2W_OK) return rc == 1 ? W2W_OK : rc;
  a.dL_dmeans3D = dL_dmeans3D; a.dL_dcov3D = dL_dcov3D; a.dL_dsh = dL_dsh; a.dL_dscales = dL_dscales;
  a.dL_drotations = dL_drotations;
  launch_backward_gaussians(a, S(stream));
  return check_launch();
}

int w2w_batch_backward_grouped(const w2w_batch_item* items, int n, const void* geom_state, long long R,
                               const void* binning_state, const void* image_state, const int* radii,
                               const float* out_alpha, const float* dL_dcolor, const float* dL_ddepth,
                               const float* dL_dalpha, int grad_mode, void* scratch, size_t scratch_bytes,
                               const uint32_t* group_tables, int num_groups, long long group_rows,
                               float* dL_dmeans2D, float* dL_dcolors, float* dL_dopacity, float* g_means3D,
                               float* g_opacity, float* g_scales, float* g_rotations, float* g_sh,
                               w2w_stream_t stream) {
  const BatchTotals t = batch_totals(items, n);
  if (t.ok && t.elems > 0 &&
      !group_outputs_ok(t, group_tables, num_groups, group_rows, g_means3D, g_opacity, g_scales, g_rotations, g_sh))
    return W2W_ERR_INVALID;
  BackwardArgs a;
  const int rc = batch_backward_begin(items, n, geom_state, R, binning_state, image_state, radii, out_alpha,
                                      dL_dcolor, dL_ddepth, dL_dalpha, grad_mode, scratch, scratch_bytes,
                                      dL_dmeans2D, dL_dcolors, dL_dopacity, S(stream), a);
  if (rc != W2W_OK) return rc == 1 ? W2W_OK : rc;
  set_group_outputs(a, group_tables, num_groups, group_rows, g_means3D, g_opacity, g_scales, g_rotations, g_sh);
  launch_backward_groups(a, S(stream));
  return check_launch();
}

int w2w_batch_gaussians_grouped(const w2w_batch_item* items, int n, const void* geom_state, const int* radii,
                                int grad_mode, void* scratch, size_t scratch_bytes, const float* dL_dmeans2D,
                                const float* dL_dcolors, const float* dL_dopacity, const uint32_t* group_tables,
                                int num_groups, long long group_rows, float* g_means3D, float* g_opacity,
                                float* g_scales, float* g_rotations, float* g_sh, w2w_stream_t stream) {
  const BatchTotals t = batch_totals(items, n);
  if (!t.ok || (grad_mode != 0 && grad_mode != 1)) return W2W_ERR_INVALID;
  if (t.elems == 0) return W2W_OK;
  if (!geom_state || !radii || !dL_dmeans2D || !dL_dcolors || !dL_dopacity ||
      !group_outputs_ok(t, group_tables, num_groups, group_rows, g_means3D, g_opacity, g_scales, g_rotations, g_sh))
    return W2W_ERR_INVALID;
  if (!scratch || scratch_bytes < w2w_batch_backward_scratch_bytes(items, n)) return W2W_ERR_SCRATCH;
  BackwardArgs a;
  // the pass only reads the per-element accumulators
  batch_gaussian_args(n, t.elems, t.M, geom_state, radii, grad_mode, scratch, const_cast<float*>(dL_dmeans2D),
                      const_cast<float*>(dL_dcolors), const_cast<float*>(dL_dopacity), a);
  set_group_outputs(a, group_tables, num_groups, group_rows, g_means3D, g_opacity, g_scales, g_rotations, g_sh);
  launch_backward_groups(a, S(stream));
  return check_launch();
}

}  // extern "C"
