// Host-side CSR pattern, per-row incident-element lists and the slot-sorted
// contribution plan consumed by the warp-per-row assembly kernel.
//
// The reference builds triplet lists and lets Eigen / scipy sum duplicates
// (backend/src/fem.cpp:116-151, qdsim_cython/solvers/schrodinger_solver.pyx:
// 131-190); here the duplicate-summing structure is computed once per mesh so
// that the GPU can assemble every matrix of that mesh without sorting or atomics.
#include <algorithm>
#include <cstring>
#include <vector>
#include "common.h"

namespace {

constexpr int kMaxRowLen = 128;      // slots per row the assembly kernel stages
constexpr int kMaxRowContrib = 255;  // m*k per row (uint8 contribution ids)
constexpr int kMaxRowAdj = 16;       // incident elements per row staged by the kernel

struct Plan {
  std::vector<int32_t> rowptr, col, adjptr, adj, cptr;
  std::vector<uint8_t> contrib, slotcnt;
};

int build_plan(int64_t num_nodes, int64_t num_elems, int k, const int32_t *elems,
               const int32_t *dof_map, int32_t n, Plan &P) {
  if (k != 3 && k != 6 && k != 10) return QD_ERR_INVALID;
  if (num_nodes <= 0 || num_elems < 0 || n < 0 || !elems || !dof_map) return QD_ERR_INVALID;
  if (num_elems >= (int64_t(1) << 27)) return QD_ERR_LIMIT;
  for (int64_t g = 0; g < num_nodes; ++g)
    if (dof_map[g] < -1 || dof_map[g] >= n) return QD_ERR_INVALID;
  // 1. incident (element, local) lists per reduced row, ascending element id
  P.adjptr.assign(n + 1, 0);
  for (int64_t e = 0; e < num_elems; ++e)
    for (int a = 0; a < k; ++a) {
      int32_t g = elems[e * k + a];
      if (g < 0 || g >= num_nodes) return QD_ERR_INVALID;
      int32_t r = dof_map[g];
      if (r >= 0) P.adjptr[r + 1]++;
    }
  for (int32_t r = 0; r < n; ++r) P.adjptr[r + 1] += P.adjptr[r];
  P.adj.assign(P.adjptr[n], 0);
  {
    std::vector<int32_t> fill(P.adjptr.begin(), P.adjptr.end() - 1);
    for (int64_t e = 0; e < num_elems; ++e)
      for (int a = 0; a < k; ++a) {
        int32_t r = dof_map[elems[e * k + a]];
        if (r >= 0) P.adj[fill[r]++] = int32_t((e << 4) | a);
      }
  }
  // 2. sorted unique columns per row and 3. slot-sorted contribution ids
  P.rowptr.assign(n + 1, 0);
  P.cptr.assign(n + 1, 0);
  std::vector<int32_t> cols;
  cols.reserve(size_t(P.adjptr[n]) * k / 2 + 16);
  std::vector<uint8_t> contrib;
  std::vector<uint8_t> slotcnt;
  contrib.reserve(size_t(P.adjptr[n]) * k);
  int32_t rc[kMaxRowContrib + 1];   // column of each (t, b)
  int32_t uniq[kMaxRowLen];
  for (int32_t r = 0; r < n; ++r) {
    const int32_t t0 = P.adjptr[r], m = P.adjptr[r + 1] - t0;
    if (m * k > kMaxRowContrib || m > kMaxRowAdj) return QD_ERR_LIMIT;
    int L = 0;
    for (int t = 0; t < m; ++t) {
      const int64_t e = P.adj[t0 + t] >> 4;
      for (int b = 0; b < k; ++b) {
        int32_t c = dof_map[elems[e * k + b]];
        rc[t * k + b] = c;
        if (c < 0) continue;
        // insertion into sorted unique list
        int pos = int(std::lower_bound(uniq, uniq + L, c) - uniq);
        if (pos < L && uniq[pos] == c) continue;
        if (L >= kMaxRowLen) return QD_ERR_LIMIT;
        std::memmove(uniq + pos + 1, uniq + pos, sizeof(int32_t) * (L - pos));
        uniq[pos] = c;
        ++L;
      }
    }
    P.rowptr[r + 1] = P.rowptr[r] + L;
    if (int64_t(P.rowptr[r + 1]) > INT32_MAX - kMaxRowLen) return QD_ERR_LIMIT;
    cols.insert(cols.end(), uniq, uniq + L);
    // contributions in (slot, t, b) order
    uint8_t cnt[kMaxRowLen];
    std::memset(cnt, 0, sizeof(cnt));
    std::vector<std::pair<int, int>> tmp;
    tmp.reserve(m * k);
    for (int t = 0; t < m; ++t)
      for (int b = 0; b < k; ++b) {
        int32_t c = rc[t * k + b];
        if (c < 0) continue;
        int s = int(std::lower_bound(uniq, uniq + L, c) - uniq);
        tmp.emplace_back(s, t * k + b);
        cnt[s]++;
      }
    std::stable_sort(tmp.begin(), tmp.end(),
                     [](const std::pair<int, int> &x, const std::pair<int, int> &y) {
                       return x.first < y.first;
                     });
    for (auto &pr : tmp) contrib.push_back(uint8_t(pr.second));
    P.cptr[r + 1] = P.cptr[r] + int32_t(tmp.size());
    slotcnt.insert(slotcnt.end(), cnt, cnt + L);
  }
  P.col.swap(cols);
  P.contrib.swap(contrib);
  P.slotcnt.swap(slotcnt);
  return QD_OK;
}

}  // namespace

extern "C" int qd_pattern_build(int64_t num_nodes, int64_t num_elems, int k,
                                const int32_t *h_elems, const int32_t *h_dof_map, int32_t n_dofs,
                                int64_t *nnz, int64_t *n_adj, int64_t *n_contrib,
                                int32_t *h_rowptr, int32_t *h_col, int32_t *h_adjptr,
                                int32_t *h_adj, int32_t *h_cptr, uint8_t *h_contrib,
                                uint8_t *h_slotcnt) {
  Plan P;
  int st = build_plan(num_nodes, num_elems, k, h_elems, h_dof_map, n_dofs, P);
  if (st != QD_OK) return st;
  if (nnz) *nnz = int64_t(P.col.size());
  if (n_adj) *n_adj = int64_t(P.adj.size());
  if (n_contrib) *n_contrib = int64_t(P.contrib.size());
  auto cp = [](auto *dst, const auto &src) {
    if (dst && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
  };
  cp(h_rowptr, P.rowptr);
  cp(h_col, P.col);
  cp(h_adjptr, P.adjptr);
  cp(h_adj, P.adj);
  cp(h_cptr, P.cptr);
  cp(h_contrib, P.contrib);
  cp(h_slotcnt, P.slotcnt);
  return QD_OK;
}

extern "C" int qd_node_adjacency(int64_t num_nodes, int64_t num_elems, int k,
                                 const int32_t *h_elems, int64_t *n_adj, int32_t *h_adjptr,
                                 int32_t *h_adj) {
  if (k != 3 && k != 6 && k != 10) return QD_ERR_INVALID;
  if (num_nodes <= 0 || num_elems < 0 || !h_elems) return QD_ERR_INVALID;
  if (num_elems >= (int64_t(1) << 27)) return QD_ERR_LIMIT;
  std::vector<int32_t> ptr(num_nodes + 1, 0);
  for (int64_t i = 0; i < num_elems * k; ++i) {
    int32_t g = h_elems[i];
    if (g < 0 || g >= num_nodes) return QD_ERR_INVALID;
    ptr[g + 1]++;
  }
  for (int64_t g = 0; g < num_nodes; ++g) ptr[g + 1] += ptr[g];
  if (n_adj) *n_adj = ptr[num_nodes];
  if (h_adjptr) std::memcpy(h_adjptr, ptr.data(), ptr.size() * sizeof(int32_t));
  if (h_adj) {
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t e = 0; e < num_elems; ++e)
      for (int a = 0; a < k; ++a) h_adj[fill[h_elems[e * k + a]]++] = int32_t((e << 4) | a);
  }
  return QD_OK;
}
