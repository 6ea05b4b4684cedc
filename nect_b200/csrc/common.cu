// Error state and version of libnectb.
#include "common.cuh"

namespace nectb {

namespace {
thread_local char g_last_error[512] = {0};
}

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

void clear_error() { g_last_error[0] = 0; }

}  // namespace nectb

extern "C" const char* nectb_version(void) { return "nectb 0.1 sm_100a"; }
extern "C" const char* nectb_last_error(void) { return nectb::g_last_error; }

// ---- per-kernel event profiler and NVTX ranges ----------------------------
#include <nvtx3/nvToolsExt.h>

#include <mutex>
#include <vector>

namespace nectb {
namespace {
struct ProfRec {
  int slot;
  cudaEvent_t a, b;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof_pending;
std::vector<cudaEvent_t> g_prof_free;
int g_prof_launches[NECTB_PROFILE_SLOTS];
double g_prof_ms[NECTB_PROFILE_SLOTS];
// NVTX range names of the slots (ncu --nvtx --nvtx-include "nectb backward/")
const char* const kProfNames[NECTB_PROFILE_SLOTS] = {
    "nectb ray preparation", "nectb forward", "nectb backward", "nectb adam", "nectb sampling",
    "nectb model and queries", "nectb staged scatter", "nectb ray ordering", "nectb time slice"};

cudaEvent_t prof_event() {
  if (!g_prof_free.empty()) {
    cudaEvent_t e = g_prof_free.back();
    g_prof_free.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

// The NVTX range brackets the launches of the scope on the host thread
// (a no-op unless a tool is attached); the events time them on the stream
// while profiling is enabled.
ProfScope::ProfScope(int slot, cudaStream_t s) : slot_(slot), s_(s), a_(nullptr) {
  nvtxRangePushA(kProfNames[slot]);
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on) return;
  a_ = prof_event();
  cudaEventRecord((cudaEvent_t)a_, s_);
}

ProfScope::~ProfScope() {
  if (a_) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    cudaEvent_t b = prof_event();
    cudaEventRecord(b, s_);
    g_prof_pending.push_back({slot_, (cudaEvent_t)a_, b});
  }
  nvtxRangePop();
}

}  // namespace nectb

extern "C" int nectb_profile_enable(int32_t enable) {
  std::lock_guard<std::mutex> lk(nectb::g_prof_mu);
  nectb::g_prof_on = enable != 0;
  return NECTB_OK;
}

extern "C" int nectb_profile_collect(int32_t* launches, double* total_ms) {
  using namespace nectb;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto& r : g_prof_pending) {
    cudaEventSynchronize(r.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    if (r.slot >= 0 && r.slot < NECTB_PROFILE_SLOTS) {
      g_prof_launches[r.slot] += 1;
      g_prof_ms[r.slot] += ms;
    }
    g_prof_free.push_back(r.a);
    g_prof_free.push_back(r.b);
  }
  g_prof_pending.clear();
  for (int i = 0; i < NECTB_PROFILE_SLOTS; ++i) {
    if (launches) launches[i] = g_prof_launches[i];
    if (total_ms) total_ms[i] = g_prof_ms[i];
    g_prof_launches[i] = 0;
    g_prof_ms[i] = 0.0;
  }
  return NECTB_OK;
}

namespace nectb {
namespace {
std::mutex g_tuning_mu;
NectbTuning g_tuning = {kFwdMaxWarpgroups, 3, 0, 4, int64_t(48) << 20, 1.0f, 3.0f, 1, 1};
}  // namespace

NectbTuning current_tuning() {
  std::lock_guard<std::mutex> lk(g_tuning_mu);
  return g_tuning;
}
}  // namespace nectb

extern "C" int nectb_get_tuning(NectbTuning* tuning) {
  using namespace nectb;
  clear_error();
  NECTB_REQUIRE(tuning, "null tuning");
  *tuning = current_tuning();
  return NECTB_OK;
}

extern "C" int nectb_set_tuning(const NectbTuning* t) {
  using namespace nectb;
  clear_error();
  NECTB_REQUIRE(t, "null tuning");
  NECTB_REQUIRE(t->forward_blocks_per_sm >= 1 && t->forward_blocks_per_sm <= kFwdMaxWarpgroups,
                "forward_blocks_per_sm must be 1..%d", kFwdMaxWarpgroups);
  NECTB_REQUIRE(t->backward_blocks_per_sm >= 1 && t->backward_blocks_per_sm <= 3, "backward_blocks_per_sm must be 1..3");
  NECTB_REQUIRE(t->scatter_blocks_per_sm >= 0 && t->scatter_blocks_per_sm <= 8, "scatter_blocks_per_sm must be 0..8");
  NECTB_REQUIRE(t->staged_rounds >= 1 && t->staged_rounds <= 64, "staged_rounds must be 1..64");
  NECTB_REQUIRE(t->scatter_group_bytes >= (int64_t(1) << 20), "scatter_group_bytes must be at least 1 MiB");
  NECTB_REQUIRE(t->run_threshold_3d >= 0.f && t->run_threshold_3d <= 64.f && t->run_threshold_4d >= 0.f &&
                    t->run_threshold_4d <= 64.f,
                "run thresholds must be in [0, 64]");
  NECTB_REQUIRE(t->time_slice == 0 || t->time_slice == 1, "time_slice must be 0 or 1");
  NECTB_REQUIRE(t->encoding_store == 0 || t->encoding_store == 1, "encoding_store must be 0 or 1");
  std::lock_guard<std::mutex> lk(g_tuning_mu);
  g_tuning = *t;
  return NECTB_OK;
}
