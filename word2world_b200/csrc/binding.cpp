// Torch binding: the drop-in `rasterize_gaussians` / `rasterize_gaussians_backward`
// pair with the reference extension's positional signatures and return tuples
// (reference ext.cpp:5-7, rasterize_points.h:15-56, rasterize_points.cu:88-246),
// plus the stage entry points used by tests and benchmarks.  Tensor checks and
// allocation live here; all computation is the C ABI of libw2w_raster.so
// (include/w2w_raster.h), enqueued on torch's current stream.
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/extension.h>

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/w2w_raster.h"

using torch::Tensor;

namespace {

void check(int rc, const char* what) {
  if (rc != W2W_OK) {
    std::ostringstream os;
    os << what << " failed: " << w2w_status_string(rc) << " (status " << rc << ")";
    throw std::runtime_error(os.str());
  }
}

Tensor f32(const Tensor& t, const char* name, const torch::Device& dev) {
  TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor");
  TORCH_CHECK(t.device() == dev, name, " must be on ", dev);
  TORCH_CHECK(t.scalar_type() == torch::kFloat32, name, " must be float32");
  return t.contiguous();
}

w2w_stream_t cur_stream() {
  return reinterpret_cast<w2w_stream_t>(c10::cuda::getCurrentCUDAStream().stream());
}

// Deferred device error checks.  A render returns before its sort has run,
// so the sort's error word (a lookback wait that ran out, an index out of
// range) cannot be read without stalling the host.  Instead, each render
// enqueues a 4-byte copy of the word into a pinned host slot on its own stream,
// followed by an event; every later call into this module polls the finished
// events without blocking and raises if a word was set, and
// check_device_errors() waits for all of them first.
class DeferredChecks {
 public:
  void add(const void* dev_word, cudaStream_t st, const char* what) {
    std::lock_guard<std::mutex> lk(mu_);
    if (free_.empty()) grow();
    Entry e = free_.back();
    free_.pop_back();
    *e.slot = 0u;
    if (cudaMemcpyAsync(e.slot, dev_word, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaEventRecord(e.ev, st) != cudaSuccess) {
      free_.push_back(e);
      throw std::runtime_error(std::string(what) + ": could not enqueue the error-word read");
    }
    e.what = what;
    pending_.push_back(e);
  }

  // Raises on the first finished entry whose word is set (wait: finish all first).
  void poll(bool wait) {
    std::string msg;
    {
      std::lock_guard<std::mutex> lk(mu_);
      std::vector<Entry> keep;
      for (Entry& e : pending_) {
        const cudaError_t q = wait ? cudaEventSynchronize(e.ev) : cudaEventQuery(e.ev);
        if (q == cudaErrorNotReady) {
          keep.push_back(e);
          continue;
        }
        if (q != cudaSuccess) {
          cudaGetLastError();
          if (msg.empty()) msg = e.what + ": CUDA error while reading the device error word";
        } else if (*e.slot != 0u && msg.empty()) {
          const uint32_t w = *e.slot;
          msg = e.what + ": device error word " + std::to_string(w) +
                ((w & 2u) ? " (a bounded device wait timed out; results invalid)"
                          : " (capacity exceeded or an index out of range; results invalid)");
        }
        free_.push_back(e);
      }
      pending_.swap(keep);
    }
    if (!msg.empty()) throw std::runtime_error(msg);
  }

 private:
  struct Entry {
    uint32_t* slot;
    cudaEvent_t ev;
    std::string what;
  };
  void grow() {
    constexpr int kSlots = 256;
    void* p = nullptr;
    if (cudaHostAlloc(&p, kSlots * sizeof(uint32_t), cudaHostAllocDefault) != cudaSuccess)
      throw std::runtime_error("could not allocate pinned error-word slots");
    for (int i = 0; i < kSlots; ++i) {
      Entry e{static_cast<uint32_t*>(p) + i, nullptr, std::string()};
      if (cudaEventCreateWithFlags(&e.ev, cudaEventDisableTiming) != cudaSuccess)
        throw std::runtime_error("could not create an event for the error-word read");
      free_.push_back(e);
    }
  }
  std::mutex mu_;
  std::vector<Entry> pending_, free_;
};

DeferredChecks& deferred() {
  static DeferredChecks* d = new DeferredChecks();  // lives until exit (its pinned slots too)
  return *d;
}

// The binning state's error word, read after the render (deferred).
void defer_bin_check(const Tensor& bin, int64_t R, int W, int H, cudaStream_t st, const char* what) {
  if (R <= 0) return;
  const size_t off = w2w_binning_offset(R, W, H, "header");  // the header starts with the error word
  deferred().add(static_cast<const unsigned char*>(bin.data_ptr()) + off, st, what);
}

// ---- planned forward --------------------------------------------------------
// Per image shape (device, P, H, W): the largest instance count and the most
// key depth bits seen so far.  Once a shape has been rendered, later renders
// of it launch their whole forward before reading the instance count back
// (w2w_forward_render_planned); a view that does not fit renders again with
// the exact plan.  The "planned_forward" tuning knob (default 1) turns this
// off; the "binning" knob's path always takes the exact plan.
struct PlanState {
  long long capacity = 0;
  int depth_bits = -1;
};
std::mutex g_plan_mu;
std::map<std::tuple<int, int64_t, int, int>, PlanState> g_plans;

int tune_index(const char* name) {
  for (int k = 0; k < w2w_tune_count(); ++k)
    if (std::string(w2w_tune_name(k)) == name) return k;
  return -1;
}

bool planned_enabled() {
  static const int planned = tune_index("planned_forward"), binning = tune_index("binning");
  return planned >= 0 && w2w_tune_get(planned) == 1 && (binning < 0 || w2w_tune_get(binning) == 0);
}

// This thread's pinned header slot and event on the current device (the slot
// is read only after the event, within the same call).
struct HeaderSlot {
  void* pinned = nullptr;
  cudaEvent_t ev = nullptr;
};
HeaderSlot& header_slot(int dev) {
  thread_local std::map<int, HeaderSlot> slots;
  HeaderSlot& h = slots[dev];
  if (h.pinned == nullptr) {
    if (cudaHostAlloc(&h.pinned, 64, cudaHostAllocDefault) != cudaSuccess)
      throw std::runtime_error("could not allocate a pinned header slot");
    if (cudaEventCreateWithFlags(&h.ev, cudaEventDisableTiming) != cudaSuccess)
      throw std::runtime_error("could not create the header event");
  }
  return h;
}

// The forward after its geometry arguments are set: `geom_async(header_host)`
// launches the projection pass and the header copy, `geom_sync(info)` is the
// synchronous geometry call of the exact plan.  Allocates the binning state
// into `bin`, renders, returns R.
template <typename GeomAsync, typename GeomSync>
int64_t planned_forward(w2w_settings& st, const Tensor& geom, const Tensor& img, const Tensor& color,
                        const Tensor& depth, const Tensor& alpha, Tensor& bin, const torch::TensorOptions& bopt,
                        int dev, GeomAsync geom_async, GeomSync geom_sync, w2w_stream_t stream, const char* what) {
  const int W = st.width, H = st.height;
  w2w_geometry_info info{};
  auto render_exact = [&]() {
    bin = torch::empty({int64_t(w2w_binning_state_bytes(info.num_rendered, W, H))}, bopt);
    pybind11::gil_scoped_release nogil;
    check(w2w_forward_render(&st, geom.data_ptr(), &info, bin.data_ptr(), img.data_ptr(), color.data_ptr<float>(),
                             depth.data_ptr<float>(), alpha.data_ptr<float>(), stream),
          "w2w_forward_render");
  };
  if (st.P == 0 || !planned_enabled()) {
    {
      pybind11::gil_scoped_release nogil;
      check(geom_sync(&info), what);
    }
    render_exact();
    return info.num_rendered;
  }
  const auto key = std::make_tuple(dev, int64_t(st.P), H, W);
  PlanState ps;
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    ps = g_plans[key];
  }
  HeaderSlot& hs = header_slot(dev);
  {
    pybind11::gil_scoped_release nogil;
    check(geom_async(hs.pinned), what);
    if (cudaEventRecord(hs.ev, reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
      throw std::runtime_error(std::string(what) + ": could not record the header event");
  }
  bool fits = false;
  if (ps.capacity > 0) {
    bin = torch::empty({int64_t(w2w_binning_state_bytes(ps.capacity, W, H))}, bopt);
    pybind11::gil_scoped_release nogil;
    check(w2w_forward_render_planned(&st, geom.data_ptr(), ps.capacity, ps.depth_bits, bin.data_ptr(),
                                     img.data_ptr(), color.data_ptr<float>(), depth.data_ptr<float>(),
                                     alpha.data_ptr<float>(), stream),
          "w2w_forward_render_planned");
  }
  {
    pybind11::gil_scoped_release nogil;
    if (cudaEventSynchronize(hs.ev) != cudaSuccess) throw std::runtime_error(std::string(what) + ": CUDA error");
  }
  check(w2w_geometry_info_from_header(hs.pinned, &info), what);
  const int need = w2w_depth_bits_needed(&info);
  if (ps.capacity > 0) fits = info.num_rendered <= ps.capacity && need <= ps.depth_bits;
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    PlanState& p = g_plans[key];
    // the capacity follows the counts: it grows to a larger view, and shrinks
    // back when a view uses less than a quarter of it (a plan sized for one
    // outsized view would make every later view clear and launch for it)
    if (info.num_rendered > p.capacity || info.num_rendered < p.capacity / 4)
      p.capacity = w2w_planned_capacity(info.num_rendered);
    if (need > p.depth_bits) p.depth_bits = need;
  }
  if (!fits) render_exact();  // the planned launches (if any) processed no instance
  return info.num_rendered;
}

// The instance count a binning state handed back by the forward is laid out
// for (R, or a planned render's capacity).
int64_t layout_count(int64_t R, const Tensor& binningBuffer, int W, int H) {
  const long long L = w2w_binning_layout_count(R, size_t(binningBuffer.numel()), W, H);
  TORCH_CHECK(L >= R, "binningBuffer does not match R");
  return L;
}

struct Camera {
  Tensor view, proj, campos, bg;
};

Camera camera(const Tensor& viewmatrix, const Tensor& projmatrix, const Tensor& campos,
              const c10::optional<Tensor>& background, const torch::Device& dev) {
  Camera c;
  c.view = f32(viewmatrix, "viewmatrix", dev);
  c.proj = f32(projmatrix, "projmatrix", dev);
  c.campos = f32(campos, "campos", dev);
  TORCH_CHECK(c.view.numel() == 16 && c.proj.numel() == 16, "view/projection matrices must have 16 elements");
  TORCH_CHECK(c.campos.numel() == 3, "campos must have 3 elements");
  if (background.has_value() && background->defined() && background->numel() > 0) {
    c.bg = f32(*background, "background", dev);
    TORCH_CHECK(c.bg.numel() == 3, "background must have 3 elements");
  } else {
    c.bg = torch::ones({3}, torch::TensorOptions().dtype(torch::kFloat32).device(dev));
  }
  return c;
}

std::tuple<int64_t, Tensor, Tensor, Tensor, Tensor, Tensor, Tensor, Tensor> rasterize_gaussians(
    const Tensor& sh, double focal_y, const Tensor& scales, const Tensor& means3D, const Tensor& projmatrix,
    int64_t degree, const Tensor& opacity, const Tensor& rotations, const Tensor& campos, const Tensor& viewmatrix,
    double focal_x, int64_t image_height, int64_t image_width, const c10::optional<Tensor>& background,
    bool compat_spill) {
  (void)focal_y;  // the reference forward uses focal_x on both axes (projection.cu:100-101)
  deferred().poll(false);
  TORCH_CHECK(means3D.dim() == 2 && means3D.size(1) == 3, "means3D must be [P, 3]");
  const auto dev = means3D.device();
  const int64_t P = means3D.size(0);
  c10::cuda::CUDAGuard guard(dev);
  Tensor m = f32(means3D, "means3D", dev);
  Tensor s = f32(scales, "scales", dev);
  Tensor r = f32(rotations, "rotations", dev);
  Tensor o = f32(opacity, "opacity", dev);
  TORCH_CHECK(s.dim() == 2 && s.size(0) == P && s.size(1) == 3, "scales must be [P, 3]");
  TORCH_CHECK(r.dim() == 2 && r.size(0) == P && r.size(1) == 4, "rotations must be [P, 4]");
  TORCH_CHECK(o.numel() == P, "opacity must have P elements");
  int64_t M = 0;
  Tensor shc;
  if (sh.numel() > 0) {
    shc = f32(sh, "sh", dev);
    TORCH_CHECK(shc.dim() == 3 && shc.size(0) == P && shc.size(2) == 3, "sh must be [P, M, 3]");
    M = shc.size(1);
  }
  TORCH_CHECK(image_height > 0 && image_width > 0, "image size must be positive");
  TORCH_CHECK(degree >= 0 && degree <= 3, "sh_degree must be in [0, 3]");
  Camera cam = camera(viewmatrix, projmatrix, campos, background, dev);
  const auto fopt = torch::TensorOptions().dtype(torch::kFloat32).device(dev);
  const auto bopt = torch::TensorOptions().dtype(torch::kUInt8).device(dev);
  const int W = int(image_width), H = int(image_height);
  Tensor color = torch::empty({3, H, W}, fopt);
  Tensor depth = torch::empty({1, H, W}, fopt);
  Tensor alpha = torch::empty({1, H, W}, fopt);
  Tensor radii = torch::empty({P}, torch::TensorOptions().dtype(torch::kInt32).device(dev));
  Tensor geom = torch::empty({int64_t(w2w_geometry_state_bytes(int(P)))}, bopt);
  Tensor img = torch::empty({int64_t(w2w_image_state_bytes(W, H))}, bopt);
  w2w_settings st{};
  st.P = int(P); st.degree = int(degree); st.M = int(M); st.width = W; st.height = H;
  st.focal_x = float(focal_x);
  st.tan_fovx = st.tan_fovy = 1.0f;
  st.scale_modifier = 1.0f;
  st.compat_spill = compat_spill ? 1 : 0;
  st.viewmatrix = cam.view.data_ptr<float>();
  st.projmatrix = cam.proj.data_ptr<float>();
  st.campos = cam.campos.data_ptr<float>();
  st.background = cam.bg.data_ptr<float>();
  const w2w_stream_t stream = cur_stream();
  const float* shp = M > 0 ? shc.data_ptr<float>() : nullptr;
  Tensor bin;
  const int64_t R = planned_forward(
      st, geom, img, color, depth, alpha, bin, bopt, dev.index(),
      [&](void* header) {
        return w2w_forward_geometry_async(&st, m.data_ptr<float>(), s.data_ptr<float>(), r.data_ptr<float>(),
                                          o.data_ptr<float>(), shp, radii.data_ptr<int>(), geom.data_ptr(), header,
                                          stream);
      },
      [&](w2w_geometry_info* info) {
        return w2w_forward_geometry(&st, m.data_ptr<float>(), s.data_ptr<float>(), r.data_ptr<float>(),
                                    o.data_ptr<float>(), shp, radii.data_ptr<int>(), geom.data_ptr(), info, stream);
      },
      stream, "w2w_forward_geometry");
  defer_bin_check(bin, R, W, H, reinterpret_cast<cudaStream_t>(stream), "w2w_forward_render");
  return std::make_tuple(R, color, depth, alpha, radii, geom, bin, img);
}

std::tuple<Tensor, Tensor, Tensor, Tensor, Tensor, Tensor, Tensor, Tensor> rasterize_gaussians_backward(
    const Tensor& background, const Tensor& means3D, const Tensor& radii, const Tensor& colors_precomp,
    const Tensor& scales, const Tensor& rotations, double scale_modifier, const Tensor& cov3D_precomp,
    const Tensor& viewmatrix, const Tensor& projmatrix, double tan_fovx, double tan_fovy,
    const Tensor& dL_dout_color, const Tensor& dL_dout_depth, const Tensor& dL_dout_alpha, const Tensor& sh,
    int64_t degree, const Tensor& campos, const Tensor& geomBuffer, int64_t R, const Tensor& binningBuffer,
    const Tensor& imageBuffer, const Tensor& alpha, bool debug, int64_t grad_mode) {
  TORCH_CHECK(means3D.dim() == 2 && means3D.size(1) == 3, "means3D must be [P, 3]");
  TORCH_CHECK(colors_precomp.numel() == 0 && cov3D_precomp.numel() == 0,
              "precomputed colours / covariances are not supported: the forward always derives them from "
              "SH coefficients, scales and rotations (as the reference forward does)");
  TORCH_CHECK(grad_mode == 0 || grad_mode == 1, "grad_mode must be 0 (reference) or 1 (exact)");
  deferred().poll(debug);
  const auto dev = means3D.device();
  c10::cuda::CUDAGuard guard(dev);
  const int64_t P = means3D.size(0);
  Tensor m = f32(means3D, "means3D", dev);
  Tensor s = f32(scales, "scales", dev);
  Tensor r = f32(rotations, "rotations", dev);
  Tensor g = f32(dL_dout_color, "dL_dout_color", dev);
  TORCH_CHECK(g.dim() == 3 && g.size(0) == 3, "dL_dout_color must be [3, H, W]");
  const int H = int(g.size(1)), W = int(g.size(2));
  Tensor gd = f32(dL_dout_depth, "dL_dout_depth", dev);
  Tensor ga = f32(dL_dout_alpha, "dL_dout_alpha", dev);
  Tensor al = f32(alpha, "alpha", dev);
  // an empty depth / alpha gradient means none (no loss on that output)
  TORCH_CHECK((gd.numel() == 0 || gd.numel() == int64_t(H) * W) && (ga.numel() == 0 || ga.numel() == int64_t(H) * W) &&
                  al.numel() == int64_t(H) * W,
              "depth / alpha gradients (or empty) and alpha must be [1, H, W]");
  TORCH_CHECK(radii.is_cuda() && radii.scalar_type() == torch::kInt32 && radii.numel() == P, "radii must be int32 [P]");
  Tensor rad = radii.contiguous();
  int64_t M = 0;
  Tensor shc;
  if (sh.numel() > 0) {
    shc = f32(sh, "sh", dev);
    TORCH_CHECK(shc.dim() == 3 && shc.size(0) == P && shc.size(2) == 3, "sh must be [P, M, 3]");
    M = shc.size(1);
  }
  TORCH_CHECK(geomBuffer.numel() >= int64_t(w2w_geometry_state_bytes(int(P))), "geomBuffer does not match P");
  TORCH_CHECK(imageBuffer.numel() >= int64_t(w2w_image_state_bytes(W, H)), "imageBuffer does not match H, W");
  const int64_t LR = layout_count(R, binningBuffer, W, H);  // R, or a planned render's capacity
  Camera cam = camera(viewmatrix, projmatrix, campos, background, dev);
  const auto fopt = torch::TensorOptions().dtype(torch::kFloat32).device(dev);
  Tensor dmean2D = torch::empty({P, 3}, fopt), dcolors = torch::empty({P, 3}, fopt),
         dopac = torch::empty({P, 1}, fopt), dmean3D = torch::empty({P, 3}, fopt),
         dcov3D = torch::empty({P, 6}, fopt), dsh = torch::empty({P, M, 3}, fopt),
         dscales = torch::empty({P, 3}, fopt), drot = torch::empty({P, 4}, fopt);
  Tensor scratch = torch::empty({int64_t(w2w_backward_scratch_bytes(int(P)))},
                                torch::TensorOptions().dtype(torch::kUInt8).device(dev));
  w2w_settings st{};
  st.P = int(P); st.degree = int(degree); st.M = int(M); st.width = W; st.height = H;
  st.tan_fovx = float(tan_fovx); st.tan_fovy = float(tan_fovy);
  st.focal_x = float(W / (2.0 * tan_fovx));
  st.scale_modifier = float(scale_modifier);
  st.viewmatrix = cam.view.data_ptr<float>();
  st.projmatrix = cam.proj.data_ptr<float>();
  st.campos = cam.campos.data_ptr<float>();
  st.background = cam.bg.data_ptr<float>();
  const w2w_stream_t stream = cur_stream();
  {
    pybind11::gil_scoped_release nogil;
    check(w2w_backward(&st, m.data_ptr<float>(), s.data_ptr<float>(), r.data_ptr<float>(),
                       M > 0 ? shc.data_ptr<float>() : nullptr, rad.data_ptr<int>(), geomBuffer.data_ptr(), LR,
                       binningBuffer.data_ptr(), imageBuffer.data_ptr(), al.data_ptr<float>(), g.data_ptr<float>(),
                       gd.numel() ? gd.data_ptr<float>() : nullptr, ga.numel() ? ga.data_ptr<float>() : nullptr,
                       int(grad_mode), scratch.data_ptr(),
                       size_t(scratch.numel()), dmean2D.data_ptr<float>(), dcolors.data_ptr<float>(),
                       dopac.data_ptr<float>(), dmean3D.data_ptr<float>(), dcov3D.data_ptr<float>(),
                       M > 0 ? dsh.data_ptr<float>() : nullptr, dscales.data_ptr<float>(), drot.data_ptr<float>(),
                       stream),
          "w2w_backward");
    if (debug) {
      const int e = w2w_state_error(geomBuffer.data_ptr(), 0, stream);
      if (e != 0) throw std::runtime_error("rasterizer device error word set: " + std::to_string(e));
    }
  }
  return std::make_tuple(dmean2D, dcolors, dopac, dmean3D, dcov3D, dsh, dscales, drot);
}

// ---- stages ---------------------------------------------------------------

// check_errors: read the scratch's error word back (synchronises the stream).
std::tuple<Tensor, Tensor> sort_pairs_u64(const Tensor& keys, const Tensor& vals, int64_t begin_bit, int64_t end_bit,
                                          bool check_errors) {
  TORCH_CHECK(keys.is_cuda() && keys.scalar_type() == torch::kInt64, "keys must be a CUDA int64 tensor (raw u64 bits)");
  TORCH_CHECK(vals.is_cuda() && vals.scalar_type() == torch::kInt32 && vals.numel() == keys.numel(),
              "vals must be a CUDA int32 tensor with one value per key");
  c10::cuda::CUDAGuard guard(keys.device());
  Tensor k = keys.contiguous(), v = vals.contiguous();
  const int64_t n = k.numel();
  Tensor ko = torch::empty_like(k), vo = torch::empty_like(v);
  Tensor scratch = torch::empty({int64_t(w2w_sort_scratch_bytes(n))}, k.options().dtype(torch::kUInt8));
  check(w2w_sort_pairs_u64(reinterpret_cast<const uint64_t*>(k.data_ptr<int64_t>()),
                           reinterpret_cast<const uint32_t*>(v.data_ptr<int>()),
                           reinterpret_cast<uint64_t*>(ko.data_ptr<int64_t>()), reinterpret_cast<uint32_t*>(vo.data_ptr<int>()),
                           n, int(begin_bit), int(end_bit), scratch.data_ptr(), size_t(scratch.numel()), cur_stream()),
        "w2w_sort_pairs_u64");
  if (check_errors && n > 0) check(w2w_scratch_error(scratch.data_ptr(), cur_stream()), "w2w_sort_pairs_u64");
  return std::make_tuple(ko, vo);
}

// Renderer.render on raw parameters (Renderer.py:164-192): the activation
// preamble runs inside the projection pass; outputs as rasterize_gaussians.
std::tuple<int64_t, Tensor, Tensor, Tensor, Tensor, Tensor, Tensor, Tensor> rasterize_gaussians_raw(
    const Tensor& means3D, const Tensor& sh_dc, const Tensor& sh_ac, const Tensor& opacity_logit, const Tensor& svec,
    const Tensor& quaternion, const Tensor& viewmatrix, const Tensor& projmatrix, const Tensor& campos,
    double focal_x, int64_t degree, int64_t image_height, int64_t image_width, const c10::optional<Tensor>& background,
    bool compat_spill) {
  deferred().poll(false);
  TORCH_CHECK(means3D.dim() == 2 && means3D.size(1) == 3, "means3D must be [P, 3]");
  const auto dev = means3D.device();
  const int64_t P = means3D.size(0);
  c10::cuda::CUDAGuard guard(dev);
  Tensor m = f32(means3D, "means3D", dev), dc = f32(sh_dc, "sh_dc", dev), ac = f32(sh_ac, "sh_ac", dev);
  Tensor lo = f32(opacity_logit, "opacity", dev), sv = f32(svec, "svec", dev), q = f32(quaternion, "quaternion", dev);
  TORCH_CHECK(dc.numel() == 3 * P && ac.dim() == 3 && ac.size(0) == P && ac.size(2) == 3 && ac.size(1) <= 15,
              "sh_dc [P,1,3] and sh_ac [P,K,3] (K <= 15) expected");
  TORCH_CHECK(lo.numel() == P && sv.numel() == 3 * P && q.numel() == 4 * P, "opacity [P,1], svec [P,3], quaternion [P,4]");
  TORCH_CHECK(image_height > 0 && image_width > 0 && degree >= 0 && degree <= 3, "bad image size or degree");
  const int64_t M = ac.size(1) + 1;
  Camera cam = camera(viewmatrix, projmatrix, campos, background, dev);
  const auto fopt = torch::TensorOptions().dtype(torch::kFloat32).device(dev);
  const auto bopt = torch::TensorOptions().dtype(torch::kUInt8).device(dev);
  const int W = int(image_width), H = int(image_height);
  Tensor color = torch::empty({3, H, W}, fopt), depth = torch::empty({1, H, W}, fopt), alpha = torch::empty({1, H, W}, fopt);
  Tensor radii = torch::empty({P}, torch::TensorOptions().dtype(torch::kInt32).device(dev));
  Tensor geom = torch::empty({int64_t(w2w_geometry_state_bytes(int(P)))}, bopt);
  Tensor img = torch::empty({int64_t(w2w_image_state_bytes(W, H))}, bopt);
  w2w_settings st{};
  st.P = int(P); st.degree = int(degree); st.M = int(M); st.width = W; st.height = H;
  st.focal_x = float(focal_x);
  st.tan_fovx = st.tan_fovy = 1.0f;
  st.scale_modifier = 1.0f;
  st.compat_spill = compat_spill ? 1 : 0;
  st.viewmatrix = cam.view.data_ptr<float>(); st.projmatrix = cam.proj.data_ptr<float>();
  st.campos = cam.campos.data_ptr<float>(); st.background = cam.bg.data_ptr<float>();
  const w2w_stream_t stream = cur_stream();
  Tensor bin;
  const int64_t R = planned_forward(
      st, geom, img, color, depth, alpha, bin, bopt, dev.index(),
      [&](void* header) {
        return w2w_forward_geometry_raw_async(&st, m.data_ptr<float>(), sv.data_ptr<float>(), q.data_ptr<float>(),
                                              lo.data_ptr<float>(), dc.data_ptr<float>(), ac.data_ptr<float>(),
                                              radii.data_ptr<int>(), geom.data_ptr(), header, stream);
      },
      [&](w2w_geometry_info* info) {
        return w2w_forward_geometry_raw(&st, m.data_ptr<float>(), sv.data_ptr<float>(), q.data_ptr<float>(),
                                        lo.data_ptr<float>(), dc.data_ptr<float>(), ac.data_ptr<float>(),
                                        radii.data_ptr<int>(), geom.data_ptr(), info, stream);
      },
      stream, "w2w_forward_geometry_raw");
  defer_bin_check(bin, R, W, H, reinterpret_cast<cudaStream_t>(stream), "w2w_forward_render");
  return std::make_tuple(R, color, depth, alpha, radii, geom, bin, img);
}

// Gradients of rasterize_gaussians_raw's outputs with respect to its raw
// parameters (reference formulas): (means2D, means3D, sh_dc, sh_ac, opacity
// logits, svec, quaternion).
std::tuple<Tensor, Tensor, Tensor, Tensor, Tensor, Tensor, Tensor> rasterize_gaussians_backward_raw(
    const Tensor& background, const Tensor& means3D, const Tensor& sh_dc, const Tensor& sh_ac,
    const Tensor& opacity_logit, const Tensor& svec, const Tensor& quaternion, const Tensor& radii,
    const Tensor& viewmatrix, const Tensor& projmatrix, const Tensor& campos, double tan_fovx, double tan_fovy,
    int64_t degree, const Tensor& dL_dout_color, const Tensor& dL_dout_depth, const Tensor& dL_dout_alpha,
    const Tensor& geomBuffer, int64_t R, const Tensor& binningBuffer, const Tensor& imageBuffer, const Tensor& alpha,
    const c10::optional<Tensor>& dens_accum, const c10::optional<Tensor>& dens_counter) {
  deferred().poll(false);
  const auto dev = means3D.device();
  // densification statistics accumulated in the pass (renderer.DensificationStats' [P, 1] tensors)
  float* dacc = nullptr;
  float* dcnt = nullptr;
  if (dens_accum.has_value() && dens_counter.has_value()) {
    const Tensor& A = *dens_accum;
    const Tensor& Cn = *dens_counter;
    TORCH_CHECK(A.is_cuda() && Cn.is_cuda() && A.device() == dev && Cn.device() == dev &&
                    A.scalar_type() == torch::kFloat32 && Cn.scalar_type() == torch::kFloat32 &&
                    A.is_contiguous() && Cn.is_contiguous() && A.numel() == means3D.size(0) &&
                    Cn.numel() == means3D.size(0),
                "densification accumulators must be contiguous float32 [P] tensors on the means' device");
    dacc = A.data_ptr<float>();
    dcnt = Cn.data_ptr<float>();
  }
  c10::cuda::CUDAGuard guard(dev);
  const int64_t P = means3D.size(0);
  Tensor m = f32(means3D, "means3D", dev), dc = f32(sh_dc, "sh_dc", dev), ac = f32(sh_ac, "sh_ac", dev);
  Tensor lo = f32(opacity_logit, "opacity", dev), sv = f32(svec, "svec", dev), q = f32(quaternion, "quaternion", dev);
  Tensor g = f32(dL_dout_color, "dL_dout_color", dev);
  TORCH_CHECK(g.dim() == 3 && g.size(0) == 3, "dL_dout_color must be [3, H, W]");
  const int H = int(g.size(1)), W = int(g.size(2));
  Tensor gd = f32(dL_dout_depth, "dL_dout_depth", dev), ga = f32(dL_dout_alpha, "dL_dout_alpha", dev);
  Tensor al = f32(alpha, "alpha", dev);
  // an empty depth / alpha gradient means none (no loss on that output)
  TORCH_CHECK((gd.numel() == 0 || gd.numel() == int64_t(H) * W) && (ga.numel() == 0 || ga.numel() == int64_t(H) * W) &&
                  al.numel() == int64_t(H) * W,
              "depth / alpha gradients (or empty) and alpha must be [1, H, W]");
  TORCH_CHECK(radii.is_cuda() && radii.scalar_type() == torch::kInt32 && radii.numel() == P, "radii must be int32 [P]");
  TORCH_CHECK(geomBuffer.numel() >= int64_t(w2w_geometry_state_bytes(int(P))), "geomBuffer does not match P");
  TORCH_CHECK(imageBuffer.numel() >= int64_t(w2w_image_state_bytes(W, H)), "imageBuffer does not match H, W");
  const int64_t LR = layout_count(R, binningBuffer, W, H);  // R, or a planned render's capacity
  Tensor rad = radii.contiguous();
  const int64_t K = ac.size(1);
  Camera cam = camera(viewmatrix, projmatrix, campos, background, dev);
  const auto fopt = torch::TensorOptions().dtype(torch::kFloat32).device(dev);
  Tensor dmean2D = torch::empty({P, 3}, fopt), dcolors = torch::empty({P, 3}, fopt),
         dlogit = torch::empty({P, 1}, fopt), dmean3D = torch::empty({P, 3}, fopt),
         dcov3D = torch::empty({P, 6}, fopt), ddc = torch::empty({P, 1, 3}, fopt), dac = torch::empty({P, K, 3}, fopt),
         dsvec = torch::empty({P, 3}, fopt), dquat = torch::empty({P, 4}, fopt);
  Tensor scratch = torch::empty({int64_t(w2w_backward_scratch_bytes(int(P)))},
                                torch::TensorOptions().dtype(torch::kUInt8).device(dev));
  w2w_settings st{};
  st.P = int(P); st.degree = int(degree); st.M = int(K + 1); st.width = W; st.height = H;
  st.tan_fovx = float(tan_fovx); st.tan_fovy = float(tan_fovy);
  st.focal_x = float(W / (2.0 * tan_fovx));
  st.scale_modifier = 1.0f;
  st.viewmatrix = cam.view.data_ptr<float>(); st.projmatrix = cam.proj.data_ptr<float>();
  st.campos = cam.campos.data_ptr<float>(); st.background = cam.bg.data_ptr<float>();
  const w2w_stream_t stream = cur_stream();
  {
    pybind11::gil_scoped_release nogil;
    check(w2w_backward_raw_densify(&st, m.data_ptr<float>(), sv.data_ptr<float>(), q.data_ptr<float>(), lo.data_ptr<float>(),
                           dc.data_ptr<float>(), ac.data_ptr<float>(), rad.data_ptr<int>(), geomBuffer.data_ptr(), LR,
                           binningBuffer.data_ptr(), imageBuffer.data_ptr(), al.data_ptr<float>(), g.data_ptr<float>(),
                           gd.numel() ? gd.data_ptr<float>() : nullptr, ga.numel() ? ga.data_ptr<float>() : nullptr,
                           scratch.data_ptr(), size_t(scratch.numel()),
                           dmean2D.data_ptr<float>(), dcolors.data_ptr<float>(), dlogit.data_ptr<float>(),
                           dmean3D.data_ptr<float>(), dcov3D.data_ptr<float>(), ddc.data_ptr<float>(),
                           dac.data_ptr<float>(), dsvec.data_ptr<float>(), dquat.data_ptr<float>(), dacc, dcnt,
                           stream),
          "w2w_backward_raw");
  }
  return std::make_tuple(dmean2D, dmean3D, ddc, dac, dlogit, dsvec, dquat);
}

// Renderer.render's activation preamble (Renderer.py:164-167), fused.
std::tuple<Tensor, Tensor, Tensor, Tensor> activate(const Tensor& opacity_logit, const Tensor& svec,
                                                    const Tensor& quaternion, const Tensor& sh_dc,
                                                    const Tensor& sh_ac) {
  const auto dev = opacity_logit.device();
  c10::cuda::CUDAGuard guard(dev);
  Tensor o = f32(opacity_logit, "opacity", dev), s = f32(svec, "svec", dev), q = f32(quaternion, "quaternion", dev);
  Tensor dc = f32(sh_dc, "sh_dc", dev), ac = f32(sh_ac, "sh_ac", dev);
  const int64_t P = o.size(0);
  TORCH_CHECK(o.numel() == P && s.numel() == 3 * P && q.numel() == 4 * P && dc.numel() == 3 * P,
              "opacity [P,1], svec [P,3], quaternion [P,4], sh_dc [P,1,3] expected");
  TORCH_CHECK(ac.dim() == 3 && ac.size(0) == P && ac.size(2) == 3, "sh_ac [P,K,3] expected");
  const int64_t K = ac.size(1);
  Tensor op = torch::empty_like(o), sc = torch::empty_like(s), rot = torch::empty_like(q);
  Tensor shs = torch::empty({P, K + 1, 3}, o.options());
  check(w2w_activate_forward(P, int(K), o.data_ptr<float>(), s.data_ptr<float>(), q.data_ptr<float>(),
                             dc.data_ptr<float>(), ac.data_ptr<float>(), op.data_ptr<float>(), sc.data_ptr<float>(),
                             rot.data_ptr<float>(), shs.data_ptr<float>(), cur_stream()),
        "w2w_activate_forward");
  return std::make_tuple(op, sc, rot, shs);
}

std::tuple<Tensor, Tensor, Tensor, Tensor, Tensor> activate_backward(const Tensor& g_opacity, const Tensor& g_scales,
                                                                     const Tensor& g_rotations, const Tensor& g_shs,
                                                                     const Tensor& opacity, const Tensor& scales,
                                                                     const Tensor& quaternion) {
  const auto dev = opacity.device();
  c10::cuda::CUDAGuard guard(dev);
  Tensor go = f32(g_opacity, "g_opacity", dev), gs = f32(g_scales, "g_scales", dev);
  Tensor gr = f32(g_rotations, "g_rotations", dev), gsh = f32(g_shs, "g_shs", dev);
  Tensor o = f32(opacity, "opacity", dev), s = f32(scales, "scales", dev), q = f32(quaternion, "quaternion", dev);
  const int64_t P = o.size(0);
  TORCH_CHECK(gsh.dim() == 3 && gsh.size(0) == P && gsh.size(2) == 3, "g_shs [P,K+1,3] expected");
  TORCH_CHECK(go.numel() == P && gs.numel() == 3 * P && gr.numel() == 4 * P && s.numel() == 3 * P &&
                  q.numel() == 4 * P, "gradient shapes do not match the parameters");
  const int64_t K = gsh.size(1) - 1;
  Tensor dlogit = torch::empty_like(o), dsvec = torch::empty_like(s), dq = torch::empty_like(q);
  Tensor ddc = torch::empty({P, 1, 3}, o.options()), dac = torch::empty({P, K, 3}, o.options());
  check(w2w_activate_backward(P, int(K), go.data_ptr<float>(), gs.data_ptr<float>(), gr.data_ptr<float>(),
                              gsh.data_ptr<float>(), o.data_ptr<float>(), s.data_ptr<float>(), q.data_ptr<float>(),
                              dlogit.data_ptr<float>(), dsvec.data_ptr<float>(), dq.data_ptr<float>(),
                              ddc.data_ptr<float>(), dac.data_ptr<float>(), cur_stream()),
        "w2w_activate_backward");
  return std::make_tuple(dlogit, dsvec, dq, ddc, dac);
}

// gaussians_handler.collect_densification_info (gaussians_handler.py:116-118), fused.
void densification_stats(const Tensor& dL_dmeans2D, const Tensor& radii, Tensor& accum, Tensor& counter) {
  const auto dev = dL_dmeans2D.device();
  c10::cuda::CUDAGuard guard(dev);
  Tensor g = f32(dL_dmeans2D, "dL_dmeans2D", dev);
  TORCH_CHECK(radii.is_cuda() && radii.device() == dev && radii.scalar_type() == torch::kInt32,
              "radii must be an int32 CUDA tensor on the gradient's device");
  Tensor r = radii.contiguous();
  const int64_t P = r.numel();
  TORCH_CHECK(g.numel() == 3 * P, "dL_dmeans2D must be [P,3]");
  for (const Tensor* t : {&accum, &counter}) {
    TORCH_CHECK(t->is_cuda() && t->device() == dev && t->scalar_type() == torch::kFloat32 && t->is_contiguous() &&
                    t->numel() == P, "accum and counter must be contiguous float32 [P] or [P,1] on the same device");
  }
  check(w2w_densification_stats(P, g.data_ptr<float>(), r.data_ptr<int>(), accum.data_ptr<float>(),
                                counter.data_ptr<float>(), cur_stream()),
        "w2w_densification_stats");
}

// Voxel occupancy field (compute_voxel_field.cu:25-124): [R, R, R], x fastest
// in memory, as the reference wrapper reshapes it (compute_voxel_field_wrapper.py:101).
Tensor voxel_field(const Tensor& means, const Tensor& covs, const Tensor& opacities, int64_t resolution,
                   int64_t num_blocks, double relax_ratio) {
  const auto dev = means.device();
  c10::cuda::CUDAGuard guard(dev);
  Tensor m = f32(means, "means", dev), c = f32(covs, "covs", dev), o = f32(opacities, "opacities", dev);
  const int64_t n = m.numel() / 3;
  TORCH_CHECK(m.numel() == 3 * n && c.numel() == 6 * n && o.numel() == n,
              "means [N,3], covs [N,6] (xx, xy, xz, yy, yz, zz), opacities [N] expected");
  Tensor occ = torch::empty({resolution, resolution, resolution}, m.options());
  check(w2w_voxel_field(m.data_ptr<float>(), c.data_ptr<float>(), o.data_ptr<float>(), int(n), int(resolution),
                        int(num_blocks), float(relax_ratio), occ.data_ptr<float>(), cur_stream()),
        "w2w_voxel_field");
  return occ;
}

// check_errors: read the scratch's error word back (synchronises the stream).
Tensor scan_u32(const Tensor& x, bool exclusive, bool check_errors) {
  TORCH_CHECK(x.is_cuda() && x.scalar_type() == torch::kInt32, "x must be a CUDA int32 tensor (raw u32 bits)");
  c10::cuda::CUDAGuard guard(x.device());
  Tensor xi = x.contiguous();
  Tensor out = torch::empty_like(xi);
  const int64_t n = xi.numel();
  Tensor scratch = torch::empty({int64_t(w2w_scan_scratch_bytes(n))}, xi.options().dtype(torch::kUInt8));
  check(w2w_scan_u32(reinterpret_cast<const uint32_t*>(xi.data_ptr<int>()), reinterpret_cast<uint32_t*>(out.data_ptr<int>()),
                     n, exclusive ? 1 : 0, scratch.data_ptr(), size_t(scratch.numel()), cur_stream()),
        "w2w_scan_u32");
  if (check_errors && n > 0) check(w2w_scratch_error(scratch.data_ptr(), cur_stream()), "w2w_scan_u32");
  return out;
}

Tensor tile_ranges(const Tensor& sorted_keys, int64_t tile_shift, int64_t ntiles) {
  TORCH_CHECK(sorted_keys.is_cuda() && sorted_keys.scalar_type() == torch::kInt64, "keys must be CUDA int64");
  c10::cuda::CUDAGuard guard(sorted_keys.device());
  Tensor k = sorted_keys.contiguous();
  Tensor out = torch::empty({ntiles, 2}, k.options().dtype(torch::kInt32));
  check(w2w_tile_ranges(reinterpret_cast<const uint64_t*>(k.data_ptr<int64_t>()), k.numel(), int(tile_shift),
                        reinterpret_cast<uint32_t*>(out.data_ptr<int>()), int(ntiles), cur_stream()),
        "w2w_tile_ranges");
  return out;
}

std::tuple<Tensor, Tensor, Tensor, Tensor> blend(const Tensor& geomBuffer, int64_t P, const Tensor& ranges,
                                                 const Tensor& point_list, int64_t image_height, int64_t image_width,
                                                 const c10::optional<Tensor>& background) {
  const auto dev = geomBuffer.device();
  c10::cuda::CUDAGuard guard(dev);
  const int W = int(image_width), H = int(image_height);
  TORCH_CHECK(ranges.is_cuda() && ranges.scalar_type() == torch::kInt32 &&
                  ranges.numel() == 2 * int64_t((W + 15) / 16) * ((H + 15) / 16),
              "ranges must be int32 [tiles, 2]");
  TORCH_CHECK(point_list.is_cuda() && point_list.scalar_type() == torch::kInt32, "point_list must be CUDA int32");
  TORCH_CHECK(geomBuffer.numel() >= int64_t(w2w_geometry_state_bytes(int(P))), "geomBuffer does not match P");
  Tensor rg = ranges.contiguous(), pl = point_list.contiguous();
  Tensor bg = background.has_value() && background->numel() > 0
                  ? f32(*background, "background", dev)
                  : torch::ones({3}, torch::TensorOptions().dtype(torch::kFloat32).device(dev));
  const auto fopt = torch::TensorOptions().dtype(torch::kFloat32).device(dev);
  Tensor color = torch::empty({3, H, W}, fopt), depth = torch::empty({1, H, W}, fopt),
         alpha = torch::empty({1, H, W}, fopt);
  Tensor img = torch::empty({int64_t(w2w_image_state_bytes(W, H))}, fopt.dtype(torch::kUInt8));
  w2w_settings st{};
  st.P = int(P); st.width = W; st.height = H;
  st.viewmatrix = bg.data_ptr<float>();  // unused by the blend; any device pointer
  st.projmatrix = bg.data_ptr<float>();
  st.campos = bg.data_ptr<float>();
  st.background = bg.data_ptr<float>();
  check(w2w_blend(&st, geomBuffer.data_ptr(), reinterpret_cast<const uint32_t*>(rg.data_ptr<int>()),
                  pl.numel() ? reinterpret_cast<const uint32_t*>(pl.data_ptr<int>()) : nullptr, img.data_ptr(),
                  color.data_ptr<float>(), depth.data_ptr<float>(), alpha.data_ptr<float>(), cur_stream()),
        "w2w_blend");
  return std::make_tuple(color, depth, alpha, img);
}

Tensor binning_keys64(const Tensor& binningBuffer, int64_t R, int64_t image_height, int64_t image_width) {
  c10::cuda::CUDAGuard guard(binningBuffer.device());
  Tensor out = torch::empty({R}, binningBuffer.options().dtype(torch::kInt64));
  check(w2w_binning_keys64_layout(binningBuffer.data_ptr(), R,
                                 layout_count(R, binningBuffer, int(image_width), int(image_height)),
                                 int(image_width), int(image_height),
                           reinterpret_cast<uint64_t*>(out.data_ptr<int64_t>()), cur_stream()),
        "w2w_binning_keys64");
  return out;
}

int64_t state_error(const Tensor& buf, int64_t which) {
  c10::cuda::CUDAGuard guard(buf.device());
  return w2w_state_error(buf.data_ptr(), int(which), cur_stream());
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.doc() = "sm_100a Gaussian rasterizer (drop-in for cudaForwardBackwardRenderer._C)";
  m.def("rasterize_gaussians", &rasterize_gaussians, py::arg("sh"), py::arg("focal_y"), py::arg("scales"),
        py::arg("means3D"), py::arg("projmatrix"), py::arg("sh_degree"), py::arg("opacity"), py::arg("rotations"),
        py::arg("campos"), py::arg("viewmatrix"), py::arg("focal_x"), py::arg("image_height") = 800,
        py::arg("image_width") = 800, py::arg("background") = py::none(), py::arg("compat_spill") = true);
  m.def("rasterize_gaussians_backward", &rasterize_gaussians_backward, py::arg("background"), py::arg("means3D"),
        py::arg("radii"), py::arg("colors_precomp"), py::arg("scales"), py::arg("rotations"),
        py::arg("scale_modifier"), py::arg("cov3D_precomp"), py::arg("viewmatrix"), py::arg("projmatrix"),
        py::arg("tan_fovx"), py::arg("tan_fovy"), py::arg("dL_dout_color"), py::arg("dL_dout_depth"),
        py::arg("dL_dout_alpha"), py::arg("sh"), py::arg("degree"), py::arg("campos"), py::arg("geomBuffer"),
        py::arg("R"), py::arg("binningBuffer"), py::arg("imageBuffer"), py::arg("alpha"), py::arg("debug"),
        py::arg("grad_mode") = 0);
  m.def("sort_pairs_u64", &sort_pairs_u64, py::arg("keys"), py::arg("vals"), py::arg("begin_bit"), py::arg("end_bit"),
        py::arg("check_errors") = true);
  m.def("scan_u32", &scan_u32, py::arg("x"), py::arg("exclusive"), py::arg("check_errors") = true);
  m.def("check_device_errors", []() {
    // waits for every pending error-word read of earlier renders; raises on a set word
    pybind11::gil_scoped_release nogil;
    deferred().poll(true);
  });
  m.def("poll_device_errors", []() { deferred().poll(false); });
  m.def("test_set_spin_limit", [](int64_t limit) { return int64_t(w2w_test_set_spin_limit(unsigned(limit))); });
  m.def("test_unpublished_tile", [](int64_t stage, int64_t tile) {
    return int64_t(w2w_test_unpublished_tile(int(stage), tile));
  });
  m.def("set_error_check", [](bool on) { return w2w_set_error_check(on ? 1 : 0) != 0; });
  m.def("tune_knobs", []() {
    py::dict d;
    for (int k = 0; k < w2w_tune_count(); ++k) d[py::str(w2w_tune_name(k))] = w2w_tune_get(k);
    return d;
  });
  m.def("tune_set", [](const std::string& name, int64_t value) {
    for (int k = 0; k < w2w_tune_count(); ++k)
      if (name == w2w_tune_name(k)) {
        const int prev = w2w_tune_set(k, int(value));
        if (prev < 0) throw std::invalid_argument("invalid value for tuning knob " + name);
        return int64_t(prev);
      }
    throw std::invalid_argument("unknown tuning knob " + name);
  });
  m.def("activate", &activate);
  m.def("rasterize_gaussians_raw", &rasterize_gaussians_raw);
  m.def("rasterize_gaussians_backward_raw", &rasterize_gaussians_backward_raw, py::arg("background"),
        py::arg("means3D"), py::arg("sh_dc"), py::arg("sh_ac"), py::arg("opacity_logit"), py::arg("svec"),
        py::arg("quaternion"), py::arg("radii"), py::arg("viewmatrix"), py::arg("projmatrix"), py::arg("campos"),
        py::arg("tan_fovx"), py::arg("tan_fovy"), py::arg("degree"), py::arg("dL_dout_color"),
        py::arg("dL_dout_depth"), py::arg("dL_dout_alpha"), py::arg("geomBuffer"), py::arg("R"),
        py::arg("binningBuffer"), py::arg("imageBuffer"), py::arg("alpha"), py::arg("dens_accum") = py::none(),
        py::arg("dens_counter") = py::none());
  m.def("densification_stats", &densification_stats);
  m.def("voxel_field", &voxel_field);
  m.def("activate_backward", &activate_backward);
  m.def("tile_ranges", &tile_ranges);
  m.def("blend", &blend, py::arg("geomBuffer"), py::arg("P"), py::arg("ranges"), py::arg("point_list"),
        py::arg("image_height"), py::arg("image_width"), py::arg("background") = py::none());
  m.def("binning_keys64", &binning_keys64);
  m.def("planned_capacity", [](int64_t R) { return int64_t(w2w_planned_capacity(R)); });
  m.def("binning_layout_count", [](int64_t R, const Tensor& binningBuffer, int64_t H, int64_t W) {
    return layout_count(R, binningBuffer, int(W), int(H));
  });
  m.def("state_error", &state_error);
  m.def("geometry_state_bytes", [](int64_t P) { return int64_t(w2w_geometry_state_bytes(int(P))); });
  m.def("image_state_bytes", [](int64_t W, int64_t H) { return int64_t(w2w_image_state_bytes(int(W), int(H))); });
  m.def("binning_state_bytes", [](int64_t R, int64_t W, int64_t H) {
    return int64_t(w2w_binning_state_bytes(R, int(W), int(H)));
  });
  m.def("geometry_offset", [](int64_t P, const std::string& n) { return int64_t(w2w_geometry_offset(int(P), n.c_str())); });
  m.def("image_offset", [](int64_t W, int64_t H, const std::string& n) {
    return int64_t(w2w_image_offset(int(W), int(H), n.c_str()));
  });
  m.def("binning_offset", [](int64_t R, int64_t W, int64_t H, const std::string& n) {
    return int64_t(w2w_binning_offset(R, int(W), int(H), n.c_str()));
  });
  m.def("binning_info", [](const Tensor& binningBuffer, int64_t R, int64_t H, int64_t W) {
    // the sort plan recorded in a binning state's header (reads 64 bytes back)
    py::dict d;
    if (R <= 0) return d;
    const int64_t off = int64_t(w2w_binning_offset(R, int(W), int(H), "header"));
    Tensor h = binningBuffer.narrow(0, off, 64).cpu().contiguous();
    const uint32_t* u = reinterpret_cast<const uint32_t*>(h.data_ptr());
    d["key64"] = u[1]; d["depth_bits"] = u[2]; d["tile_bits"] = u[4]; d["passes"] = u[5];
    return d;
  });
  m.def("throughput_probe", [](int64_t kind, int64_t iters, int64_t blocks, const Tensor& out) {
    // enqueues the probe on the current stream; returns its instruction count
    c10::cuda::CUDAGuard guard(out.device());
    long long ops = 0;
    check(w2w_throughput_probe(int(kind), iters, int(blocks), out.data_ptr<float>(), &ops, cur_stream()),
          "w2w_throughput_probe");
    return int64_t(ops);
  });
  m.def("version", &w2w_version);
  m.def("launch_count", []() { return (unsigned long long)w2w_launch_count(); });
  m.def("stage_timing", [](bool on) { return w2w_stage_timing(on ? 1 : 0) != 0; });
  m.def("stage_timing_only", [](const std::vector<std::string>& names) {
    unsigned mask = 0;
    for (const auto& nm : names)
      for (int i = 0; i < w2w_stage_count(); ++i)
        if (nm == w2w_stage_name(i)) mask |= 1u << i;
    return w2w_stage_timing_mask(mask);
  });
  m.def("stage_times", []() {
    const int n = w2w_stage_count();
    std::vector<double> ms(n);
    std::vector<long long> cnt(n);
    {
      pybind11::gil_scoped_release nogil;
      w2w_stage_times(ms.data(), cnt.data(), n);
    }
    py::dict d;
    for (int i = 0; i < n; ++i)
      d[py::str(w2w_stage_name(i))] = py::make_tuple(ms[i], cnt[i]);
    return d;
  });
}
