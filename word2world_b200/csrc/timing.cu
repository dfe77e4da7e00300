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
                                       "backward_render", "backward_gaussians", "scan", "other"};

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

}  // namespace w2w

extern "C" {

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
