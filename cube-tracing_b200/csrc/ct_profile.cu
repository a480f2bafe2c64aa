// ct_profile.cu -- see ct_profile.cuh.
#include <atomic>
#include <mutex>
#include <vector>
#include "ct.h"
#include "ct_profile.cuh"

const char *const ct_kernel_names[CT_K_COUNT] = {
    "k_trace_primary", "k_di_gen0",         "k_di_gen1",      "k_di_resolve0", "k_spatial_select",
    "k_spatial_sample", "k_spatial_resolve", "k_trace_shadow", "k_taa",         "k_queries",
    "k_pt_start",       "k_pt_extend",       "k_pt_shade",     "k_pt_temporal", "k_pt_spatial",
    "k_edit",           "k_pt_finish",      "k_trace_prev",   "k_adjoint_forward", "k_adjoint_backward",
    "k_pt_replay",      "k_nrc_encode",      "k_nrc_mlp",      "k_nrc_trace"};

namespace {
struct Pending {
  int kernel;
  cudaEvent_t a, b;
};
std::atomic<bool> g_on{false};
std::mutex g_mu;
std::vector<Pending> g_pending;     // launches whose events have not been read
std::vector<cudaEvent_t> g_pool;    // recycled events
double g_ms[CT_K_COUNT];
uint64_t g_launches[CT_K_COUNT];

cudaEvent_t take_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}
}  // namespace

bool ct_profile_on() { return g_on.load(std::memory_order_relaxed); }

int ct_profile_begin(int kernel, cudaStream_t s) {
  if (!ct_profile_on()) return -1;
  std::lock_guard<std::mutex> lk(g_mu);
  Pending p{kernel, take_event(), take_event()};
  if (!p.a || !p.b) return -1;
  cudaEventRecord(p.a, s);
  g_pending.push_back(p);
  return (int)g_pending.size() - 1;
}

void ct_profile_end(int token, cudaStream_t s) {
  if (token < 0) return;
  std::lock_guard<std::mutex> lk(g_mu);
  if ((size_t)token < g_pending.size()) cudaEventRecord(g_pending[token].b, s);
}

extern "C" ct_status ct_profile_enable(int enable) {
  g_on.store(enable != 0);
  return CT_OK;
}

extern "C" ct_status ct_profile_read(ct_kernel_time *out, uint32_t capacity, uint32_t *count, int reset) {
  if (!count || (capacity && !out)) return CT_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_mu);
  ct_status st = CT_OK;
  for (const Pending &p : g_pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(p.b) != cudaSuccess || cudaEventElapsedTime(&ms, p.a, p.b) != cudaSuccess) {
      st = CT_ERR_CUDA;
    } else {
      g_ms[p.kernel] += ms;
      g_launches[p.kernel]++;
    }
    g_pool.push_back(p.a);
    g_pool.push_back(p.b);
  }
  g_pending.clear();
  uint32_t n = 0;
  for (int k = 0; k < CT_K_COUNT; k++) {
    if (!g_launches[k]) continue;
    if (n < capacity) {
      out[n].name = ct_kernel_names[k];
      out[n].total_ms = g_ms[k];
      out[n].launches = g_launches[k];
    }
    n++;
  }
  *count = n;
  if (reset) {
    for (int k = 0; k < CT_K_COUNT; k++) {
      g_ms[k] = 0.0;
      g_launches[k] = 0;
    }
  }
  return st;
}
