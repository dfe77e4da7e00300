// Launch accounting and optional per-stage device timing.
//
// Every kernel launch of the library is counted.  When stage timing is
// enabled, each stage's launches are bracketed by CUDA events recorded on the
// launching stream; w2w_stage_times() waits for them and accumulates
// milliseconds and launch counts per stage.
#include <atomic>
#include <mutex>
#include <vector>

#include "../../include/w2w_raster.h"
#include "kernels.h"

namespace w2w {
namespace {

const char* kStageNames[kNumStages] = {"preprocess", "duplicate", "sort_histogram", "sort_onesweep", "blend",
                                       "backward_render", "backward_gaussians", "scan", "other", "depth_sort",
                                       "binning"};

std::atomic<unsigned long long> g_launches{0};
std::atomic<unsigned> g_mask{0};  // bit s: stage s records events

struct Pending {
  int stage;
  int kernels;
  cudaEvent_t start, stop;
};

std::mutex g_mu;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_free;
double g_ms[kNumStages] = {0};
long long g_count[kNumStages] = {0};
thread_local cudaEvent_t t_start = nullptr;

cudaEvent_t take_event() {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_free.empty()) {
    cudaEvent_t e = g_free.back();
    g_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

}  // namespace

void stage_begin(int stage, cudaStream_t s) {
  if (!((g_mask.load(std::memory_order_relaxed) >> stage) & 1u)) return;
  t_start = take_event();
  cudaEventRecord(t_start, s);
}

void stage_end(int stage, cudaStream_t s, int kernels) {
  g_launches.fetch_add(static_cast<unsigned long long>(kernels), std::memory_order_relaxed);
  if (!((g_mask.load(std::memory_order_relaxed) >> stage) & 1u) || t_start == nullptr) return;
  cudaEvent_t stop = take_event();
  cudaEventRecord(stop, s);
  std::lock_guard<std::mutex> lk(g_mu);
  g_pending.push_back(Pending{stage, kernels, t_start, stop});
  t_start = nullptr;
}

std::atomic<uint32_t> g_spin_limit{kSpinLimit};
std::atomic<long long> g_unpublished[kNumWaitStages] = {{-1}, {-1}, {-1}};

uint32_t spin_limit() { return g_spin_limit.load(std::memory_order_relaxed); }

namespace {
const char* kTuneNames[kNumTuneKnobs] = {"blend_warps", "backward_split", "backward_ways",
                                         "binning",     "blend_queue",    "preprocess_blocks",
                                         "planned_forward", "blend_stage"};
// defaults: 4-warp blend CTAs, the heaviest half-SM-count tiles' backward
// walks split in two (backward_split 2 measured 3.09 against 3.21 ms per 4-view
// step for 4, same B200), radix sort, per-tile blend, 4 projection CTAs per SM,
// planned forward on, blend batches copied with cp.async (five 4-warp CTAs per
// SM: 1416-1423 against 1388-1396 views/s for the 4-view step with the views
// on their own streams; alone the kernel takes 0.218 against 0.199 ms, so a
// single-stream caller's autotuning may pick 0)
std::atomic<int> g_tune[kNumTuneKnobs] = {{4}, {2}, {2}, {0}, {0}, {4}, {1}, {1}};
bool tune_valid(int knob, int v) {
  switch (knob) {
    case kTuneBlendWarps: return v == 4 || v == 8;
    case kTuneBwdSplit: return v >= 0 && v <= 16;
    case kTuneBwdWays: return v == 2 || v == 3;
    case kTuneBinning: return v == 0 || v == 1;
    case kTuneBlendQueue: return v == 0 || v == 1;
    case kTunePreBlocks: return v >= 2 && v <= 4;
    case kTunePlanned: return v == 0 || v == 1;
    case kTuneBlendStage: return v == 0 || v == 1;
    default: return false;
  }
}
}  // namespace

int tune_value(int knob) {
  return (knob >= 0 && knob < kNumTuneKnobs) ? g_tune[knob].load(std::memory_order_relaxed) : 0;
}

long long unpublished_tile(int stage) {
  return (stage >= 0 && stage < kNumWaitStages) ? g_unpublished[stage].load(std::memory_order_relaxed) : -1;
}

}  // namespace w2w

extern "C" {

int w2w_tune_count(void) { return w2w::kNumTuneKnobs; }

const char* w2w_tune_name(int knob) {
  return (knob >= 0 && knob < w2w::kNumTuneKnobs) ? w2w::kTuneNames[knob] : "";
}

int w2w_tune_get(int knob) { return w2w::tune_value(knob); }

int w2w_tune_set(int knob, int value) {
  if (!w2w::tune_valid(knob, value)) return -1;
  return w2w::g_tune[knob].exchange(value);
}

unsigned w2w_test_set_spin_limit(unsigned limit) {
  return w2w::g_spin_limit.exchange(limit == 0u ? w2w::kSpinLimit : limit);
}

long long w2w_test_unpublished_tile(int stage, long long tile) {
  if (stage < 0 || stage >= w2w::kNumWaitStages) return -2;
  return w2w::g_unpublished[stage].exchange(tile < 0 ? -1 : tile);
}

unsigned long long w2w_launch_count(void) { return w2w::g_launches.load(); }

int w2w_stage_timing(int enable) {
  return w2w::g_mask.exchange(enable ? (1u << w2w::kNumStages) - 1u : 0u) != 0u;
}

unsigned w2w_stage_timing_mask(unsigned mask) {
  return w2w::g_mask.exchange(mask & ((1u << w2w::kNumStages) - 1u));
}

int w2w_stage_count(void) { return w2w::kNumStages; }

const char* w2w_stage_name(int i) { return (i >= 0 && i < w2w::kNumStages) ? w2w::kStageNames[i] : ""; }

int w2w_stage_times(double* ms, long long* launches, int n) {
  using namespace w2w;
  std::vector<Pending> p;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    p.swap(g_pending);
  }
  for (const Pending& e : p) {
    float t = 0.f;
    if (cudaEventSynchronize(e.stop) == cudaSuccess && cudaEventElapsedTime(&t, e.start, e.stop) == cudaSuccess) {
      g_ms[e.stage] += t;
      g_count[e.stage] += e.kernels;
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (const Pending& e : p) {
      g_free.push_back(e.start);
      g_free.push_back(e.stop);
    }
  }
  const int k = n < kNumStages ? n : kNumStages;
  for (int i = 0; i < k; ++i) {
    if (ms) ms[i] = g_ms[i];
    if (launches) launches[i] = g_count[i];
  }
  for (int i = 0; i < kNumStages; ++i) {
    g_ms[i] = 0;
    g_count[i] = 0;
  }
  return k;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Arithmetic throughput probe: the FP32 and SFU issue rates of this GPU, the
// denominators of the per-pixel passes' roofline (their unit is an evaluated
// Gaussian-pixel pair: FP32 instructions plus one exponential and one
// division each).  Every thread runs kChains independent dependency chains,
// so each warp scheduler always has independent instructions to issue.
// ---------------------------------------------------------------------------
namespace w2w {
namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) fma_probe_kernel(long long iters, float a, float* out) {
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = float(threadIdx.x + c);
  for (long long i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = __fmaf_rn(x[c], a, 0.5f);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 1234.5f) out[threadIdx.x] = s;  // keeps the chains live; never true for the probe's inputs
}

__device__ __forceinline__ float ex2_approx(float v) {
  float r;
  asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

__global__ void __launch_bounds__(256) sfu_probe_kernel(long long iters, float a, float* out) {
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = a * 1e-3f * float(threadIdx.x + c);
  for (long long i = 0; i < iters; ++i) {
    // x stays in [0.5, 1]: one MUFU instruction per step (the sign is an operand modifier)
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = ex2_approx(-x[c]);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 1234.5f) out[threadIdx.x] = s;
}

}  // namespace
}  // namespace w2w

extern "C" int w2w_throughput_probe(int kind, long long iters, int blocks, float* out, long long* ops,
                                    w2w_stream_t stream) {
  using namespace w2w;
  if ((kind != 0 && kind != 1) || iters <= 0 || blocks <= 0 || !out) return W2W_ERR_INVALID;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // a multiplier just below 1 keeps the chains finite and normal
  if (kind == 0) fma_probe_kernel<<<blocks, 256, 0, st>>>(iters, 0.999999f, out);
  else sfu_probe_kernel<<<blocks, 256, 0, st>>>(iters, 0.999999f, out);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (ops) *ops = (long long)blocks * 256 * iters * kChains;
  return cudaGetLastError() == cudaSuccess ? W2W_OK : W2W_ERR_CUDA;
}
