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
#include <algorithm>
#include <cmath>
#include <functional>
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
      // degree 2: l (2 l - 1) at the vertices, 4 l_a l_b on edges [1,2], [0,2], [0,1]
      const double p2[6] = {phi[0] * (2.0 * phi[0] - 1.0), phi[1] * (2.0 * phi[1] - 1.0),
                            phi[2] * (2.0 * phi[2] - 1.0), 4.0 * phi[1] * phi[2],
                            4.0 * phi[0] * phi[2], 4.0 * phi[0] * phi[1]};
      for (int b = 0; b < 6; ++b) {
        r.phi2[b][i] = p2[b];
        r.wphi2[b][i] = e.weights[i] * p2[b];
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

// ------------------------------------------------------------------ quadrilaterals ---
// Quadrilateral rules (ndelement's reference square: v0 = (0,0), v1 = (1,0), v2 = (0,1),
// v3 = (1,1); edges [0,1], [0,2], [1,3], [2,3]).
//
// Regular: Gauss-Legendre tensor rules of n x n points on [0,1]^2 (weights sum to 1), n
// the smallest with n^2 >= the requested number of points (37, the default, gives 7 x 7).
//
// Singular (Sauter & Schwab, Boundary Element Methods, section 5.2, for squares), on a
// canonical configuration mapped onto the shared entity of each cell by a symmetry of the
// square, n-point Gauss-Legendre on every coordinate of [0,1]^4:
//   identical: z = x - y split by the signs of z1, z2 and by which of |z1|, |z2| is larger
//     (|z| = (xi, xi eta) or (xi eta, xi), Jacobian xi), y on the overlap of the square
//     and its shift, y_i = max(0, -z_i) + (1 - |z_i|) t_i: 8 regions;
//   edge (shared edge x2 = y2 = 0, x1 = y1 on it): (|x1 - y1|, x2, y2) in 3 pyramids by the
//     largest coordinate (Jacobian xi^2), 2 signs of x1 - y1, y1 on the overlap: 6 regions;
//   vertex (shared vertex x = y = 0): (x1, x2, y1, y2) in 4 pyramids by the largest
//     coordinate (Jacobian xi^3): 4 regions.
namespace {

const double kQV[4][2] = {{0.0, 0.0}, {1.0, 0.0}, {0.0, 1.0}, {1.0, 1.0}};
const int kQE[4][2] = {{0, 1}, {0, 2}, {1, 3}, {2, 3}};

// x -> o + x0 d + x1 m: the symmetry of the square taking (0,0) to vertex p and (1,0) to
// vertex q (q < 0: the reflection that keeps the axes)
struct SquareSymmetry {
  double o[2], d[2], m[2];
  SquareSymmetry(int p, int q) {
    o[0] = kQV[p][0];
    o[1] = kQV[p][1];
    const double sx = kQV[p][0] == 0.0 ? 1.0 : -1.0, sy = kQV[p][1] == 0.0 ? 1.0 : -1.0;
    if (q < 0) {
      d[0] = sx; d[1] = 0.0; m[0] = 0.0; m[1] = sy;
      return;
    }
    d[0] = kQV[q][0] - kQV[p][0];
    d[1] = kQV[q][1] - kQV[p][1];
    if (d[0] != 0.0) {
      m[0] = 0.0; m[1] = sy;
    } else {
      m[0] = sx; m[1] = 0.0;
    }
  }
  void apply(double a, double b, std::vector<double>& out) const {
    out.push_back(o[0] + a * d[0] + b * m[0]);
    out.push_back(o[1] + a * d[1] + b * m[1]);
  }
};

}  // namespace

int quad_gauss_order(size_t npoints) {
  int n = 1;
  while (static_cast<size_t>(n) * n < npoints) ++n;
  if (n > kMaxQuadGauss)
    throw Error(kUnsupported, "quadrilateral regular rules have at most " +
                                  std::to_string(kMaxQuadGauss * kMaxQuadGauss) + " points; " +
                                  std::to_string(npoints) + " asked");
  return n;
}

QuadGaussRule quad_gauss_rule(size_t npoints) {
  const int n = quad_gauss_order(npoints);
  std::vector<double> g, gw;
  gauss_legendre_01(n, g, gw);
  QuadGaussRule r{};
  r.n = n;
  for (int i = 0; i < n; ++i) {
    r.x[i] = g[i];
    r.w[i] = gw[i];
  }
  return r;
}

const std::vector<std::vector<std::pair<int, int>>>& quad_singular_configurations() {
  static const std::vector<std::vector<std::pair<int, int>>> configs = [] {
    std::vector<std::vector<std::pair<int, int>>> out;
    for (int t = 0; t < 4; ++t)
      for (int s = 0; s < 4; ++s) out.push_back({{t, s}});
    for (int te = 0; te < 4; ++te)
      for (int se = 0; se < 4; ++se) {
        out.push_back({{kQE[te][0], kQE[se][0]}, {kQE[te][1], kQE[se][1]}});
        out.push_back({{kQE[te][1], kQE[se][0]}, {kQE[te][0], kQE[se][1]}});
      }
    out.push_back({{0, 0}, {1, 1}, {2, 2}, {3, 3}});
    return out;
  }();
  return configs;
}

DuffyRule quad_duffy_rule(int config, int order) {
  const auto& configs = quad_singular_configurations();
  if (config < 0 || config >= static_cast<int>(configs.size()) || order < 1)
    throw Error(kInvalidArgument, "quadrilateral Duffy rule: bad configuration or order");
  const auto& pairs = configs[config];
  std::vector<double> g, gw;
  gauss_legendre_01(order, g, gw);
  const SquareSymmetry mt = pairs.size() == 4   ? SquareSymmetry(0, 1)
                            : pairs.size() == 2 ? SquareSymmetry(pairs[0].first, pairs[1].first)
                                                : SquareSymmetry(pairs[0].first, -1);
  const SquareSymmetry ms = pairs.size() == 4   ? SquareSymmetry(0, 1)
                            : pairs.size() == 2 ? SquareSymmetry(pairs[0].second, pairs[1].second)
                                                : SquareSymmetry(pairs[0].second, -1);
  DuffyRule r;
  auto push = [&](double x1, double x2, double y1, double y2, double w) {
    mt.apply(x1, x2, r.test_xi);
    ms.apply(y1, y2, r.trial_xi);
    r.w.push_back(w);
  };
  const int n = order;
  // region loops outermost, then the Gauss points of (xi, a, b, c)
  auto gauss4 = [&](const std::function<void(double, double, double, double, double)>& f) {
    for (int i0 = 0; i0 < n; ++i0)
      for (int i1 = 0; i1 < n; ++i1)
        for (int i2 = 0; i2 < n; ++i2)
          for (int i3 = 0; i3 < n; ++i3)
            f(g[i0], g[i1], g[i2], g[i3], gw[i0] * gw[i1] * gw[i2] * gw[i3]);
  };
  if (pairs.size() == 4) {
    for (int s1 = -1; s1 <= 1; s1 += 2)
      for (int s2 = -1; s2 <= 1; s2 += 2)
        for (int first = 1; first >= 0; --first)  // |z1| >= |z2| first
          gauss4([&](double xi, double a, double b, double c, double wq) {
            const double z1 = s1 * (first ? xi : xi * a), z2 = s2 * (first ? xi * a : xi);
            const double y1 = std::max(0.0, -z1) + (1.0 - std::fabs(z1)) * b;
            const double y2 = std::max(0.0, -z2) + (1.0 - std::fabs(z2)) * c;
            push(y1 + z1, y2 + z2, y1, y2,
                 wq * xi * (1.0 - std::fabs(z1)) * (1.0 - std::fabs(z2)));
          });
  } else if (pairs.size() == 2) {
    for (int s = -1; s <= 1; s += 2)
      for (int pyr = 0; pyr < 3; ++pyr)  // the largest of (|x1 - y1|, x2, y2)
        gauss4([&](double xi, double a, double b, double c, double wq) {
          double u[3];
          for (int k = 0, e = 0; k < 3; ++k) u[k] = k == pyr ? xi : xi * (e++ == 0 ? a : b);
          const double z = s * u[0];
          const double y1 = std::max(0.0, -z) + (1.0 - u[0]) * c;
          push(y1 + z, u[1], y1, u[2], wq * xi * xi * (1.0 - u[0]));
        });
  } else {
    for (int pyr = 0; pyr < 4; ++pyr)  // the largest of (x1, x2, y1, y2)
      gauss4([&](double xi, double a, double b, double c, double wq) {
        const double e[3] = {a, b, c};
        double u[4];
        for (int k = 0, j = 0; k < 4; ++k) u[k] = k == pyr ? xi : xi * e[j++];
        push(u[0], u[1], u[2], u[3], wq * xi * xi * xi);
      });
  }
  return r;
}

}  // namespace bempp_b200
