// Event-based per-kernel-kind timing (used by the benchmark to time the
// dominant kernel inside the timed region on the stream it runs on).
#include <cuda_runtime.h>
#include <mutex>
#include <vector>
#include "common.h"

namespace qd {

namespace {
struct Pending {
  int kind;
  cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Pending> g_pending;
std::vector<std::pair<int, cudaEvent_t>> g_open;   // begun, not ended (per kind stack)
double g_ms[PK_COUNT] = {0};
int64_t g_n[PK_COUNT] = {0};
}  // namespace

bool prof_enabled() {
  std::lock_guard<std::mutex> lk(g_mu);
  return g_on;
}

void prof_begin(int kind, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_on) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, s);
  g_open.emplace_back(kind, e);
}

void prof_end(int kind, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_on) return;
  for (size_t i = g_open.size(); i-- > 0;) {
    if (g_open[i].first != kind) continue;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, s);
    g_pending.push_back(Pending{kind, g_open[i].second, e});
    g_open.erase(g_open.begin() + i);
    return;
  }
}

}  // namespace qd

extern "C" int qd_prof_enable(int on) {
  std::lock_guard<std::mutex> lk(qd::g_mu);
  qd::g_on = on != 0;
  return QD_OK;
}

extern "C" int qd_prof_read(double *ms, int64_t *launches, int reset) {
  std::lock_guard<std::mutex> lk(qd::g_mu);
  for (auto &p : qd::g_pending) {
    if (cudaEventSynchronize(p.b) != cudaSuccess) return QD_ERR_CUDA;
    float t = 0.f;
    if (cudaEventElapsedTime(&t, p.a, p.b) != cudaSuccess) return QD_ERR_CUDA;
    qd::g_ms[p.kind] += t;
    qd::g_n[p.kind] += 1;
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  qd::g_pending.clear();
  for (int k = 0; k < qd::PK_COUNT; ++k) {
    if (ms) ms[k] = qd::g_ms[k];
    if (launches) launches[k] = qd::g_n[k];
    if (reset) {
      qd::g_ms[k] = 0.0;
      qd::g_n[k] = 0;
    }
  }
  return QD_OK;
}
