// Reference-element tables in constant memory.  Each translation unit that
// includes this header owns its own copy of the symbol and uploads it on first
// use per device (host tables from tables.cpp).  The upload is a synchronous
// cudaMemcpyToSymbol, so the first call of an entry point on a device must not
// happen inside a stream capture.
#pragma once
#include <cuda_runtime.h>
#include <mutex>
#include "common.h"
#include "tables.h"

namespace {

__constant__ double c_tab[qd::kTableDoubles];

// packed layout per order: Mr, Sxx, Sxy, Syy (K*K each), then T (K*K*K)
template <int K> struct TabBase;
template <> struct TabBase<3> { static constexpr int v = 0; };
template <> struct TabBase<6> { static constexpr int v = 63; };
template <> struct TabBase<10> { static constexpr int v = 423; };

std::mutex g_tab_mu;
bool g_tab_ready[64] = {false};

int ensure_tables() {
  int dev = 0;
  QD_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return QD_ERR_LIMIT;
  std::lock_guard<std::mutex> lk(g_tab_mu);
  if (g_tab_ready[dev]) return QD_OK;
  static double host[qd::kTableDoubles];
  qd::TableOffsets off[4];
  qd::pack_tables(host, off);
  QD_CUDA_TRY(cudaMemcpyToSymbol(c_tab, host, sizeof(host)));
  g_tab_ready[dev] = true;
  return QD_OK;
}

}  // namespace
