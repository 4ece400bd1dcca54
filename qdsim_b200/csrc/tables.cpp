#include "tables.h"
#include <cstring>

namespace qd {

void quadrature_rule(int order, std::vector<double> &lam, std::vector<double> &w) {
  lam.clear();
  w.clear();
  auto add_xe = [&](double xi, double eta, double wt) {
    lam.push_back(1.0 - xi - eta);
    lam.push_back(xi);
    lam.push_back(eta);
    w.push_back(wt);
  };
  if (order == 1) {
    // backend/src/fem.cpp:843-847 (interior 3-point rule, weight area/3)
    const double a = 1.0 / 6.0, b = 2.0 / 3.0;
    const double pts[3][3] = {{a, a, b}, {a, b, a}, {b, a, a}};
    for (auto &p : pts) {
      lam.insert(lam.end(), p, p + 3);
      w.push_back(1.0 / 3.0);
    }
    return;
  }
  if (order == 2) {
    // backend/src/fem.cpp:787-803 (7-point, degree 5)
    add_xe(1.0 / 3.0, 1.0 / 3.0, 0.225000000000000);
    add_xe(0.059715871789770, 0.470142064105115, 0.132394152788506);
    add_xe(0.470142064105115, 0.059715871789770, 0.132394152788506);
    add_xe(0.470142064105115, 0.470142064105115, 0.132394152788506);
    add_xe(0.797426985353087, 0.101286507323456, 0.125939180544827);
    add_xe(0.101286507323456, 0.797426985353087, 0.125939180544827);
    add_xe(0.101286507323456, 0.101286507323456, 0.125939180544827);
  } else {
    // backend/src/fem.cpp:807-832 (12-point, degree 6)
    const double a = 0.249286745170910, b = 0.501426509658179;
    const double c = 0.063089014491502, d = 0.873821971016996;
    const double e = 0.310352451033785, f = 0.636502499121399, g = 0.053145049844816;
    const double w1 = 0.116786275726379, w2 = 0.050844906370207, w3 = 0.082851075618374;
    add_xe(a, a, w1); add_xe(a, b, w1); add_xe(b, a, w1);
    add_xe(c, c, w2); add_xe(c, d, w2); add_xe(d, c, w2);
    add_xe(e, f, w3); add_xe(f, g, w3); add_xe(g, e, w3);
    add_xe(f, e, w3); add_xe(e, g, w3); add_xe(g, f, w3);
  }
  double s = 0.0;
  for (double x : w) s += x;
  for (double &x : w) x /= s;
}

void shape_functions(int order, const double lam[3], double *phi, double *d) {
  const double l0 = lam[0], l1 = lam[1], l2 = lam[2];
  const int k = order == 1 ? 3 : order == 2 ? 6 : 10;
  for (int i = 0; i < 3 * k; ++i) d[i] = 0.0;
  auto D = [&](int m, int i) -> double & { return d[m * k + i]; };
  if (order == 1) {
    phi[0] = l0; phi[1] = l1; phi[2] = l2;
    D(0, 0) = D(1, 1) = D(2, 2) = 1.0;
    return;
  }
  if (order == 2) {
    phi[0] = l0 * (2 * l0 - 1); phi[1] = l1 * (2 * l1 - 1); phi[2] = l2 * (2 * l2 - 1);
    phi[3] = 4 * l0 * l1; phi[4] = 4 * l1 * l2; phi[5] = 4 * l2 * l0;
    D(0, 0) = 4 * l0 - 1; D(1, 1) = 4 * l1 - 1; D(2, 2) = 4 * l2 - 1;
    D(0, 3) = 4 * l1; D(1, 3) = 4 * l0;
    D(1, 4) = 4 * l2; D(2, 4) = 4 * l1;
    D(2, 5) = 4 * l0; D(0, 5) = 4 * l2;
    return;
  }
  const double L[3] = {l0, l1, l2};
  for (int m = 0; m < 3; ++m) {
    phi[m] = 0.5 * L[m] * (3 * L[m] - 1) * (3 * L[m] - 2);
    D(m, m) = 0.5 * (27 * L[m] * L[m] - 18 * L[m] + 2);
  }
  // edges (i, j) carry nodes ni (nearer i) and nj (nearer j)
  const int E[3][4] = {{0, 1, 3, 4}, {1, 2, 5, 6}, {2, 0, 7, 8}};
  for (auto &ed : E) {
    const int i = ed[0], j = ed[1], ni = ed[2], nj = ed[3];
    const double li = L[i], lj = L[j];
    phi[ni] = 4.5 * li * lj * (3 * li - 1);
    phi[nj] = 4.5 * li * lj * (3 * lj - 1);
    D(i, ni) = 4.5 * lj * (6 * li - 1);
    D(j, ni) = 4.5 * li * (3 * li - 1);
    D(i, nj) = 4.5 * lj * (3 * lj - 1);
    D(j, nj) = 4.5 * li * (6 * lj - 1);
  }
  phi[9] = 27 * l0 * l1 * l2;
  D(0, 9) = 27 * l1 * l2; D(1, 9) = 27 * l0 * l2; D(2, 9) = 27 * l0 * l1;
}

RefTables make_tables(int order) {
  RefTables t;
  t.order = order;
  const int k = order == 1 ? 3 : order == 2 ? 6 : 10;
  t.k = k;
  std::vector<double> lam, w;
  quadrature_rule(order, lam, w);
  const int Q = int(w.size());
  t.Mr.assign(k * k, 0.0);
  t.Sxx.assign(k * k, 0.0);
  t.Sxy.assign(k * k, 0.0);
  t.Syy.assign(k * k, 0.0);
  t.T.assign(k * k * k, 0.0);
  std::vector<double> phi(k), d(3 * k), dxi(k), deta(k);
  for (int q = 0; q < Q; ++q) {
    shape_functions(order, &lam[3 * q], phi.data(), d.data());
    for (int i = 0; i < k; ++i) {
      dxi[i] = d[k + i] - d[i];        // xi = lambda1
      deta[i] = d[2 * k + i] - d[i];   // eta = lambda2
    }
    const double wq = w[q];
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) {
        t.Mr[i * k + j] += wq * phi[i] * phi[j];
        t.Sxx[i * k + j] += wq * dxi[i] * dxi[j];
        t.Sxy[i * k + j] += wq * (dxi[i] * deta[j] + deta[i] * dxi[j]);
        t.Syy[i * k + j] += wq * deta[i] * deta[j];
        for (int l = 0; l < k; ++l) t.T[(l * k + i) * k + j] += wq * phi[l] * phi[i] * phi[j];
      }
  }
  return t;
}

void pack_tables(double *dst, TableOffsets off[4]) {
  int pos = 0;
  for (int p = 1; p <= 3; ++p) {
    RefTables t = make_tables(p);
    auto put = [&](const std::vector<double> &v) {
      int at = pos;
      std::memcpy(dst + pos, v.data(), v.size() * sizeof(double));
      pos += int(v.size());
      return at;
    };
    off[p].Mr = put(t.Mr);
    off[p].Sxx = put(t.Sxx);
    off[p].Sxy = put(t.Sxy);
    off[p].Syy = put(t.Syy);
    off[p].T = put(t.T);
  }
}

}  // namespace qd
