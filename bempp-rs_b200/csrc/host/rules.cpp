// Quadrature rules of the assembler.
//
// Regular pairs: fully symmetric triangle rules selected by point count, as
// ndelement::quadrature::simplex_rule is used at src/boundary_assemblers.rs:419,434
// (table generated by gen_simplex_rules.py).
//
// Singular pairs: bempp-rs builds one rule per adjacency configuration with
// bempp_quadrature::duffy::triangle_duffy (bempp-quadrature 0.1.0, unvendored) at
// src/boundary_assemblers.rs:524-562.  The rules here restate the published construction
// of Sauter & Schwab, Boundary Element Methods (Springer 2011), section 5.2: the pair
// integral over That x That, That = {0 <= x2 <= x1 <= 1}, is split into 6 (identical
// cells), 5 (common edge) or 2 (common vertex) regions, each mapped from the unit 4-cube
// (xi, eta1, eta2, eta3) with Jacobian xi^3 eta1^2 eta2 (identical, edge) or xi^3 eta2
// (vertex) so that the 1/r singularity cancels; every axis uses n-point Gauss-Legendre.
// That's vertices P0=(0,0), P1=(1,0), P2=(1,1) (barycentric (1-x1, x1-x2, x2)) are
// mapped onto the cells' local vertices so that the shared vertex is P0 and the shared
// edge is P0-P1 in both cells.
#include <cmath>
#include <stdexcept>
#include <string>

#include "core.h"

namespace bempp_b200 {

namespace {
struct SimplexRuleEntry {
  int npoints;
  int degree;
  const double* points;
  const double* weights;
};
#include "simplex_rules_table.inc"
}  // namespace

void gauss_legendre_01(int n, std::vector<double>& x, std::vector<double>& w) {
  // Newton's method on the Legendre polynomial P_n, roots mapped from [-1,1] to [0,1].
  x.resize(n);
  w.resize(n);
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < n; ++i) {
    double t = std::cos(pi * (i + 0.75) / (n + 0.5));
    double dpn = 1.0;
    for (int it = 0; it < 100; ++it) {
      double pm1 = 1.0, pn = t;
      for (int j = 2; j <= n; ++j) {
        double pj = ((2 * j - 1) * t * pn - (j - 1) * pm1) / j;
        pm1 = pn;
        pn = pj;
      }
      if (n == 1) {
        pn = t;
        pm1 = 1.0;
      }
      dpn = n * (t * pn - pm1) / (t * t - 1.0);
      double step = pn / dpn;
      t -= step;
      if (std::fabs(step) < 1e-16) break;
    }
    x[n - 1 - i] = 0.5 * (t + 1.0);
    w[n - 1 - i] = 1.0 / ((1.0 - t * t) * dpn * dpn);
  }
}

bool has_simplex_rule(int npoints) {
  for (const auto& e : kSimplexRules)
    if (e.npoints == npoints) return true;
  return false;
}

RegularRule simplex_rule(int npoints) {
  for (const auto& e : kSimplexRules) {
    if (e.npoints != npoints) continue;
    if (npoints > kMaxRegularPoints)
      throw Error(kUnsupported, "regular rule larger than the kernels support");
    RegularRule r{};
    r.npts = npoints;
    for (int i = 0; i < npoints; ++i) {
      r.w[i] = e.weights[i];
      r.xi[2 * i] = e.points[2 * i];
      r.xi[2 * i + 1] = e.points[2 * i + 1];
      r.wf[i] = static_cast<float>(e.weights[i]);
      r.uf[i] = static_cast<float>(e.points[2 * i] - 1.0 / 3.0);
      r.vf[i] = static_cast<float>(e.points[2 * i + 1] - 1.0 / 3.0);
      const double x = e.points[2 * i], y = e.points[2 * i + 1];
      const double phi[3] = {1.0 - x - y, x, y};
      r.u[i] = x - 1.0 / 3.0;
      r.v[i] = y - 1.0 / 3.0;
      for (int b = 0; b < 3; ++b) {
        r.phi[b][i] = phi[b];
        r.phif[b][i] = static_cast<float>(phi[b]);
        r.wphi[b][i] = e.weights[i] * phi[b];
      }
    }
    return r;
  }
  std::string avail;
  for (const auto& e : kSimplexRules) avail += " " + std::to_string(e.npoints);
  throw Error(kUnsupported, "no symmetric triangle rule with " + std::to_string(npoints) +
                                " points (available:" + avail + ")");
}

const std::vector<std::vector<std::pair<int, int>>>& singular_configurations() {
  static const std::vector<std::vector<std::pair<int, int>>> configs = [] {
    std::vector<std::vector<std::pair<int, int>>> c;
    for (int i = 0; i < 3; ++i)  // vertex-adjacent
      for (int j = 0; j < 3; ++j) c.push_back({{i, j}});
    const int edges[3][2] = {{1, 2}, {0, 2}, {0, 1}};  // reference_cell::edges(Triangle)
    for (const auto& te : edges)                        // edge-adjacent, two orientations
      for (const auto& se : edges) {
        c.push_back({{te[0], se[0]}, {te[1], se[1]}});
        c.push_back({{te[1], se[0]}, {te[0], se[1]}});
      }
    c.push_back({{0, 0}, {1, 1}, {2, 2}});  // identical
    return c;
  }();
  return configs;
}

namespace {

// One region of a Sauter-Schwab decomposition: points of That x That and the Jacobian.
struct RegionPoint {
  double x1, x2, y1, y2, jac;
};

RegionPoint identical_region(int r, double xi, double a, double b, double c) {
  const double j = xi * xi * xi * a * a * b;
  switch (r) {
    case 0: return {xi, xi * (1 - a + a * b), xi * (1 - a * b * c), xi * (1 - a), j};
    case 1: return {xi * (1 - a * b * c), xi * (1 - a), xi, xi * (1 - a + a * b), j};
    case 2: return {xi, xi * a * (1 - b + b * c), xi * (1 - a * b), xi * a * (1 - b), j};
    case 3: return {xi * (1 - a * b), xi * a * (1 - b), xi, xi * a * (1 - b + b * c), j};
    case 4: return {xi * (1 - a * b * c), xi * a * (1 - b * c), xi, xi * a * (1 - b), j};
    default: return {xi, xi * a * (1 - b), xi * (1 - a * b * c), xi * a * (1 - b * c), j};
  }
}

RegionPoint edge_region(int r, double xi, double a, double b, double c) {
  const double j0 = xi * xi * xi * a * a;
  const double j = j0 * b;
  switch (r) {
    case 0: return {xi, xi * a * c, xi * (1 - a * b), xi * a * (1 - b), j0};
    case 1: return {xi, xi * a, xi * (1 - a * b * c), xi * a * b * (1 - c), j};
    case 2: return {xi * (1 - a * b), xi * a * (1 - b), xi, xi * a * b * c, j};
    case 3: return {xi * (1 - a * b * c), xi * a * b * (1 - c), xi, xi * a, j};
    default: return {xi * (1 - a * b * c), xi * a * (1 - b * c), xi, xi * a * b, j};
  }
}

RegionPoint vertex_region(int r, double xi, double a, double b, double c) {
  const double j = xi * xi * xi * b;
  if (r == 0) return {xi, xi * a, xi * b, xi * b * c, j};
  return {xi * b, xi * b * a, xi, xi * c, j};
}

// Point of That (x1, x2) -> reference-triangle coordinates of a cell whose local vertex
// perm[k] plays the role of P_k.
void to_reference(double x1, double x2, const int perm[3], double& u, double& v) {
  const double bary[3] = {1.0 - x1, x1 - x2, x2};
  u = v = 0.0;
  for (int k = 0; k < 3; ++k) {
    if (perm[k] == 1) u += bary[k];
    if (perm[k] == 2) v += bary[k];
  }
}

}  // namespace

DuffyRule duffy_rule(int config, int order) {
  const auto& cfgs = singular_configurations();
  if (config < 0 || config >= static_cast<int>(cfgs.size()))
    throw Error(kInvalidArgument, "bad singular configuration");
  if (order < 1) throw Error(kInvalidArgument, "singular quadrature order must be >= 1");
  const auto& pairs = cfgs[config];
  int tp[3], sp[3];
  const int shared = static_cast<int>(pairs.size());
  auto fill_rest = [](int* perm, int used) {
    int k = used;
    for (int v = 0; v < 3; ++v) {
      bool in = false;
      for (int u = 0; u < used; ++u) in = in || perm[u] == v;
      if (!in) perm[k++] = v;
    }
  };
  for (int s = 0; s < shared && s < 2; ++s) {
    tp[s] = pairs[s].first;
    sp[s] = pairs[s].second;
  }
  if (shared == 3) {
    for (int v = 0; v < 3; ++v) tp[v] = sp[v] = v;
  } else {
    fill_rest(tp, shared);
    fill_rest(sp, shared);
  }
  std::vector<double> gx, gw;
  gauss_legendre_01(order, gx, gw);
  const int nreg = shared == 3 ? 6 : (shared == 2 ? 5 : 2);
  DuffyRule r;
  const size_t n4 = static_cast<size_t>(order) * order * order * order;
  r.test_xi.reserve(2 * nreg * n4);
  r.trial_xi.reserve(2 * nreg * n4);
  r.w.reserve(nreg * n4);
  for (int reg = 0; reg < nreg; ++reg)
    for (int i0 = 0; i0 < order; ++i0)
      for (int i1 = 0; i1 < order; ++i1)
        for (int i2 = 0; i2 < order; ++i2)
          for (int i3 = 0; i3 < order; ++i3) {
            const double xi = gx[i0], a = gx[i1], b = gx[i2], c = gx[i3];
            RegionPoint p = shared == 3   ? identical_region(reg, xi, a, b, c)
                            : shared == 2 ? edge_region(reg, xi, a, b, c)
                                          : vertex_region(reg, xi, a, b, c);
            double u, v;
            to_reference(p.x1, p.x2, tp, u, v);
            r.test_xi.push_back(u);
            r.test_xi.push_back(v);
            to_reference(p.y1, p.y2, sp, u, v);
            r.trial_xi.push_back(u);
            r.trial_xi.push_back(v);
            r.w.push_back(gw[i0] * gw[i1] * gw[i2] * gw[i3] * p.jac);
          }
  return r;
}

}  // namespace bempp_b200
