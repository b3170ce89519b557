// CPU FP64 assembly of Laplace and Helmholtz boundary operators on single-element
// quadrilateral grids.
//
// TEST INFRASTRUCTURE ONLY: the checker of the CUDA assembler's quadrilateral path; only
// the tests load it, the product never links or calls it.
//
// Same structure as the triangle oracle (oracle.cpp) and the reference
// (src/boundary_assemblers.rs): the regular part integrates every pair of cells that
// share no vertex with the tensor product of a regular rule on both cells, the singular
// part every ordered pair that shares a vertex (each pair once, grouped by its
// (test_local, trial_local) vertex pairing, trial local ascending, as
// get_pairs_if_smallest lists them) with the Duffy rule of that pairing; entries are
// added into the dense column-major output.  Restated from published mathematics, since
// the crates that hold them are not in the reference tree:
//   * degree-1 quadrilateral geometry (ndgrid): the bilinear map of the four vertices in
//     ndelement's order v0 = (0,0), v1 = (1,0), v2 = (0,1), v3 = (1,1), with its Jacobian,
//     Jacobian determinant and unit normal at every quadrature point;
//   * Lagrange degree 0 / 1 on the quadrilateral (ndelement): DP0; Q1 with the tensor
//     basis (1-x)(1-y), x(1-y), (1-x)y, xy, continuous (one DOF per vertex, first visit)
//     or discontinuous (four interior DOFs);
//   * regular rules: Gauss-Legendre tensor rules of n x n points on [0,1]^2, n the
//     smallest with n^2 >= the option's point count (the 37-point rule that ndelement
//     would give is not in the tree; a 7 x 7 rule stands for it);
//   * Duffy rules (bempp-quadrature `quadrilateral_duffy`): Sauter & Schwab, Boundary
//     Element Methods (Springer 2011), section 5.2, for quadrilaterals: identical cells
//     through the difference z = x - y (4 sign quadrants x 2 Duffy triangles, the
//     remaining coordinates on the overlap of the two squares), edge-adjacent cells
//     through (x1 - y1, x2, y2) (2 signs x 3 pyramids), vertex-adjacent cells through the
//     4-cube (4 pyramids), n-point Gauss-Legendre per coordinate; the canonical shared
//     vertex (0,0) / edge x2 = y2 = 0 is mapped onto each cell's shared entity by a
//     symmetry of the square.
// The hypersingular integrand uses the surface curl (J1 d0 phi - J0 d1 phi) / jdet, which
// holds for any parametrised surface (n x grad_surface phi).  No reference test holds a
// quadrilateral matrix; this restatement is checked by its own invariants (rules that
// integrate polynomials exactly, the closed-form Coulomb energy of a unit square) in
// tests/test_oracle_golden.py.

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace {

using cplx = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;

void gauss01(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = 0.0;
      for (int j = 1; j <= n; ++j) {
        double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
      }
      dp = n * (z * p0 - p1) / (z * z - 1.0);
      double dz = p0 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[n - 1 - i] = 0.5 * (1.0 + z);
    w[n - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);
  }
}

// reference coordinates of the quadrilateral's vertices and its edges
const double kVert[4][2] = {{0.0, 0.0}, {1.0, 0.0}, {0.0, 1.0}, {1.0, 1.0}};
const int kEdge[4][2] = {{0, 1}, {0, 2}, {1, 3}, {2, 3}};

struct Rule {
  std::vector<double> tp, sp, w;  // test / trial points (x0,y0,x1,...) and weights
  int n() const { return static_cast<int>(w.size()); }
};

// --- canonical Duffy rules on [0,1]^2 x [0,1]^2 ----------------------------------------
// identical cells: singular on x = y
Rule canonical_identical(int n) {
  std::vector<double> g, gw;
  gauss01(n, g, gw);
  Rule r;
  for (int s1 = -1; s1 <= 1; s1 += 2)
    for (int s2 = -1; s2 <= 1; s2 += 2)
      for (int ord = 0; ord < 2; ++ord)
        for (int a = 0; a < n; ++a)
          for (int b = 0; b < n; ++b)
            for (int c = 0; c < n; ++c)
              for (int d = 0; d < n; ++d) {
                const double xi = g[a], eta = g[b], t1 = g[c], t2 = g[d];
                const double big = xi, small = xi * eta;
                const double z1 = s1 * (ord == 0 ? big : small);
                const double z2 = s2 * (ord == 0 ? small : big);
                const double y1 = std::max(0.0, -z1) + (1.0 - std::fabs(z1)) * t1;
                const double y2 = std::max(0.0, -z2) + (1.0 - std::fabs(z2)) * t2;
                const double jac = xi * (1.0 - std::fabs(z1)) * (1.0 - std::fabs(z2));
                r.tp.push_back(y1 + z1);
                r.tp.push_back(y2 + z2);
                r.sp.push_back(y1);
                r.sp.push_back(y2);
                r.w.push_back(gw[a] * gw[b] * gw[c] * gw[d] * jac);
              }
  return r;
}

// edge-adjacent cells: shared edge x2 = y2 = 0 with x1 = y1 on it
Rule canonical_edge(int n) {
  std::vector<double> g, gw;
  gauss01(n, g, gw);
  Rule r;
  for (int s = -1; s <= 1; s += 2)
    for (int pyr = 0; pyr < 3; ++pyr)
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b)
          for (int c = 0; c < n; ++c)
            for (int d = 0; d < n; ++d) {
              const double xi = g[a], e1 = g[b], e2 = g[c], t = g[d];
              double az, x2, y2;  // |z|, x2, y2: the largest is xi
              if (pyr == 0) {
                az = xi; x2 = xi * e1; y2 = xi * e2;
              } else if (pyr == 1) {
                x2 = xi; az = xi * e1; y2 = xi * e2;
              } else {
                y2 = xi; az = xi * e1; x2 = xi * e2;
              }
              const double z = s * az;
              const double y1 = std::max(0.0, -z) + (1.0 - az) * t;
              r.tp.push_back(y1 + z);
              r.tp.push_back(x2);
              r.sp.push_back(y1);
              r.sp.push_back(y2);
              r.w.push_back(gw[a] * gw[b] * gw[c] * gw[d] * xi * xi * (1.0 - az));
            }
  return r;
}

// vertex-adjacent cells: shared vertex x = y = 0
Rule canonical_vertex(int n) {
  std::vector<double> g, gw;
  gauss01(n, g, gw);
  Rule r;
  for (int pyr = 0; pyr < 4; ++pyr)
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b)
        for (int c = 0; c < n; ++c)
          for (int d = 0; d < n; ++d) {
            const double xi = g[a];
            const double e[3] = {g[b], g[c], g[d]};
            double u[4];
            for (int i = 0, k = 0; i < 4; ++i) u[i] = i == pyr ? xi : xi * e[k++];
            r.tp.push_back(u[0]);
            r.tp.push_back(u[1]);
            r.sp.push_back(u[2]);
            r.sp.push_back(u[3]);
            r.w.push_back(gw[a] * gw[b] * gw[c] * gw[d] * xi * xi * xi);
          }
  return r;
}

// symmetry of the square taking canonical (0,0) to vertex p and canonical (1,0) to
// vertex q (an edge), or (0,0) to p alone (q < 0: the reflection that fixes the axes)
struct SquareMap {
  double o[2], d[2], m[2];  // x -> o + x1 d + x2 m
  void apply(const double* x, double* out) const {
    out[0] = o[0] + x[0] * d[0] + x[1] * m[0];
    out[1] = o[1] + x[0] * d[1] + x[1] * m[1];
  }
};

SquareMap square_map(int p, int q) {
  SquareMap s;
  s.o[0] = kVert[p][0];
  s.o[1] = kVert[p][1];
  if (q < 0) {
    s.d[0] = kVert[p][0] == 0.0 ? 1.0 : -1.0;
    s.d[1] = 0.0;
    s.m[0] = 0.0;
    s.m[1] = kVert[p][1] == 0.0 ? 1.0 : -1.0;
    return s;
  }
  s.d[0] = kVert[q][0] - kVert[p][0];
  s.d[1] = kVert[q][1] - kVert[p][1];
  if (s.d[0] != 0.0) {  // edge along x: the other neighbour of p is along y
    s.m[0] = 0.0;
    s.m[1] = kVert[p][1] == 0.0 ? 1.0 : -1.0;
  } else {
    s.m[0] = kVert[p][0] == 0.0 ? 1.0 : -1.0;
    s.m[1] = 0.0;
  }
  return s;
}

// The 49 vertex pairings of two quadrilaterals that share a vertex, an edge or are the
// same cell: (test_local, trial_local) pairs, trial local ascending.  Order: 16 vertex
// pairings (t * 4 + s), 32 edge pairings (16 + (test edge * 4 + trial edge) * 2 +
// orientation), the identical cell last.
std::vector<std::vector<std::pair<int, int>>> quad_configurations() {
  std::vector<std::vector<std::pair<int, int>>> out;
  for (int t = 0; t < 4; ++t)
    for (int s = 0; s < 4; ++s) out.push_back({{t, s}});
  for (int te = 0; te < 4; ++te)
    for (int se = 0; se < 4; ++se) {
      out.push_back({{kEdge[te][0], kEdge[se][0]}, {kEdge[te][1], kEdge[se][1]}});
      out.push_back({{kEdge[te][1], kEdge[se][0]}, {kEdge[te][0], kEdge[se][1]}});
    }
  out.push_back({{0, 0}, {1, 1}, {2, 2}, {3, 3}});
  return out;
}

Rule quad_duffy_rule(const std::vector<std::pair<int, int>>& pairs, int order) {
  Rule c;
  SquareMap mt, ms;
  if (pairs.size() == 4) {
    c = canonical_identical(order);
    mt = ms = square_map(0, 1);  // the identity
  } else if (pairs.size() == 2) {
    c = canonical_edge(order);
    mt = square_map(pairs[0].first, pairs[1].first);
    ms = square_map(pairs[0].second, pairs[1].second);
  } else {
    c = canonical_vertex(order);
    mt = square_map(pairs[0].first, -1);
    ms = square_map(pairs[0].second, -1);
  }
  Rule r;
  r.w = c.w;
  r.tp.resize(c.tp.size());
  r.sp.resize(c.sp.size());
  for (int i = 0; i < c.n(); ++i) {
    mt.apply(&c.tp[2 * i], &r.tp[2 * i]);
    ms.apply(&c.sp[2 * i], &r.sp[2 * i]);
  }
  return r;
}

// --- mesh, spaces, geometry -------------------------------------------------------------
struct QMesh {
  const double* pts;
  int64_t npts;
  const int64_t* cells;  // ncells x 4
  int64_t ncells;
  std::vector<std::vector<int64_t>> vertex_cells;
  void build() {
    vertex_cells.assign(npts, {});
    for (int64_t c = 0; c < ncells; ++c)
      for (int i = 0; i < 4; ++i) vertex_cells[cells[4 * c + i]].push_back(c);
  }
  int64_t v(int64_t c, int i) const { return cells[4 * c + i]; }
};

struct QSpace {
  int nbasis = 1;
  int64_t ndofs = 0;
  std::vector<int64_t> cell_dofs;
  int degree = 0;
};

QSpace make_qspace(const QMesh& m, int degree, bool continuous) {
  QSpace s;
  s.degree = degree;
  if (degree == 0) {
    s.nbasis = 1;
    s.ndofs = m.ncells;
    for (int64_t c = 0; c < m.ncells; ++c) s.cell_dofs.push_back(c);
  } else if (degree == 1) {
    s.nbasis = 4;
    s.cell_dofs.resize(4 * m.ncells);
    if (continuous) {
      std::vector<int64_t> vdof(m.npts, -1);
      int64_t size = 0;
      for (int64_t c = 0; c < m.ncells; ++c)
        for (int i = 0; i < 4; ++i) {
          int64_t v = m.v(c, i);
          if (vdof[v] < 0) vdof[v] = size++;
          s.cell_dofs[4 * c + i] = vdof[v];
        }
      s.ndofs = size;
    } else {
      for (int64_t i = 0; i < 4 * m.ncells; ++i) s.cell_dofs[i] = i;
      s.ndofs = 4 * m.ncells;
    }
  } else {
    throw std::runtime_error("oracle: quadrilateral spaces of degree 0 and 1 only");
  }
  return s;
}

void qtabulate(int degree, const double* xi, double v[4], double d0[4], double d1[4]) {
  if (degree == 0) {
    v[0] = 1.0;
    d0[0] = d1[0] = 0.0;
    return;
  }
  const double x = xi[0], y = xi[1];
  v[0] = (1 - x) * (1 - y); d0[0] = -(1 - y); d1[0] = -(1 - x);
  v[1] = x * (1 - y);       d0[1] = 1 - y;    d1[1] = -x;
  v[2] = (1 - x) * y;       d0[2] = -y;       d1[2] = 1 - x;
  v[3] = x * y;             d0[3] = y;        d1[3] = x;
}

struct PGeom {
  double x[3], j0[3], j1[3], n[3], jdet;
};

void qgeom(const QMesh& m, int64_t c, const double* xi, PGeom& g) {
  const double* a = m.pts + 3 * m.v(c, 0);
  const double* b = m.pts + 3 * m.v(c, 1);
  const double* d = m.pts + 3 * m.v(c, 2);
  const double* e = m.pts + 3 * m.v(c, 3);
  const double s = xi[0], t = xi[1];
  for (int i = 0; i < 3; ++i) {
    g.x[i] = a[i] * (1 - s) * (1 - t) + b[i] * s * (1 - t) + d[i] * (1 - s) * t + e[i] * s * t;
    g.j0[i] = (b[i] - a[i]) * (1 - t) + (e[i] - d[i]) * t;
    g.j1[i] = (d[i] - a[i]) * (1 - s) + (e[i] - b[i]) * s;
  }
  const double cx = g.j0[1] * g.j1[2] - g.j0[2] * g.j1[1];
  const double cy = g.j0[2] * g.j1[0] - g.j0[0] * g.j1[2];
  const double cz = g.j0[0] * g.j1[1] - g.j0[1] * g.j1[0];
  g.jdet = std::sqrt(cx * cx + cy * cy + cz * cz);
  g.n[0] = cx / g.jdet;
  g.n[1] = cy / g.jdet;
  g.n[2] = cz / g.jdet;
}

// entry contribution of one point pair (without the rule weight): jdet_x jdet_y times
// the integrand of src/boundary_assemblers/integrands/*.rs (Helmholtz hypersingular:
// src/helmholtz.rs:98-104)
template <typename T>
T point_integrand(int op, bool helm, double k, const PGeom& x, const PGeom& y, double pv,
                  double p0, double p1, double sv, double s0, double s1);

template <typename T>
T green(bool helm, double k, double r) {
  if constexpr (std::is_same_v<T, double>) {
    (void)helm;
    (void)k;
    return 1.0 / (4.0 * kPi * r);
  } else {
    return cplx(std::cos(k * r), std::sin(k * r)) / (4.0 * kPi * r);
  }
}

template <typename T>
T point_integrand(int op, bool helm, double k, const PGeom& x, const PGeom& y, double pv,
                  double p0, double p1, double sv, double s0, double s1) {
  double d[3] = {x.x[0] - y.x[0], x.x[1] - y.x[1], x.x[2] - y.x[2]};
  const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const T gval = green<T>(helm, k, r);
  const double jj = x.jdet * y.jdet;
  if (op == 0) return gval * pv * sv * jj;
  if (op == 1 || op == 2) {
    // grad_y G = G (1 - ikr) d / r^2 (Helmholtz), G d / r^2 (Laplace)
    T f;
    if constexpr (std::is_same_v<T, double>)
      f = gval / (r * r);
    else
      f = gval * cplx(1.0, -k * r) / (r * r);
    const double* nn = op == 1 ? y.n : x.n;
    const double dn = d[0] * nn[0] + d[1] * nn[1] + d[2] * nn[2];
    return (op == 1 ? 1.0 : -1.0) * f * dn * pv * sv * jj;
  }
  // hypersingular: G (curl phi . curl psi) jdet_x jdet_y; the jdet cancel the curls'
  double cc = 0.0;
  for (int i = 0; i < 3; ++i)
    cc += (x.j1[i] * p0 - x.j0[i] * p1) * (y.j1[i] * s0 - y.j0[i] * s1);
  T val = gval * cc;
  if (helm) {
    const double nn = x.n[0] * y.n[0] + x.n[1] * y.n[1] + x.n[2] * y.n[2];
    val += -k * k * gval * nn * pv * sv * jj;
  }
  return val;
}

bool qshare_vertex(const QMesh& m, int64_t a, int64_t b) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      if (m.v(a, i) == m.v(b, j)) return true;
  return false;
}

template <typename T>
void qassemble(const QMesh& m, const QSpace& ts, const QSpace& ss, int op, bool helm, double k,
               int nreg, int order, int parts, T* out) {
  const int64_t nt = ts.ndofs;
  const int ntb = ts.nbasis, nsb = ss.nbasis;
  if (parts & 1) {
    std::vector<double> g, gw;
    gauss01(nreg, g, gw);
    const int Q = nreg * nreg;
    std::vector<double> pts(2 * Q), wts(Q);
    for (int i = 0; i < nreg; ++i)
      for (int j = 0; j < nreg; ++j) {
        pts[2 * (i * nreg + j)] = g[i];
        pts[2 * (i * nreg + j) + 1] = g[j];
        wts[i * nreg + j] = gw[i] * gw[j];
      }
    // per trial cell its entries, added serially afterwards in trial-cell order: cells of
    // a continuous space share DOFs, so threads must not add into one column at once
    struct Trip {
      int64_t row, col;
      T val;
    };
    std::vector<std::vector<Trip>> per_cell(m.ncells);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t sc = 0; sc < m.ncells; ++sc) {
      std::vector<PGeom> sg(Q), tg(Q);
      std::vector<double> sv(4 * Q), s0(4 * Q), s1(4 * Q), tv(4 * Q), t0(4 * Q), t1(4 * Q);
      for (int q = 0; q < Q; ++q) {
        qgeom(m, sc, &pts[2 * q], sg[q]);
        qtabulate(ss.degree, &pts[2 * q], &sv[4 * q], &s0[4 * q], &s1[4 * q]);
        qtabulate(ts.degree, &pts[2 * q], &tv[4 * q], &t0[4 * q], &t1[4 * q]);
      }
      for (int64_t tc = 0; tc < m.ncells; ++tc) {
        if (qshare_vertex(m, tc, sc)) continue;
        for (int p = 0; p < Q; ++p) qgeom(m, tc, &pts[2 * p], tg[p]);
        for (int b = 0; b < nsb; ++b)
          for (int a = 0; a < ntb; ++a) {
            T e = T(0.0);
            for (int p = 0; p < Q; ++p)
              for (int q = 0; q < Q; ++q)
                e += point_integrand<T>(op, helm, k, tg[p], sg[q], tv[4 * p + a], t0[4 * p + a],
                                        t1[4 * p + a], sv[4 * q + b], s0[4 * q + b],
                                        s1[4 * q + b]) *
                     (wts[p] * wts[q]);
            per_cell[sc].push_back({ts.cell_dofs[tc * ntb + a], ss.cell_dofs[sc * nsb + b], e});
          }
      }
    }
    for (const auto& cell : per_cell)
      for (const Trip& tr : cell) out[tr.row + nt * tr.col] += tr.val;
  }
  if (parts & 2) {
    auto configs = quad_configurations();
    std::vector<Rule> rules;
    for (auto& c : configs) rules.push_back(quad_duffy_rule(c, order));
    std::vector<std::vector<std::pair<int64_t, int64_t>>> cell_pairs(configs.size());
    for (int64_t v = 0; v < m.npts; ++v)
      for (int64_t tcell : m.vertex_cells[v])
        for (int64_t scell : m.vertex_cells[v]) {
          std::vector<std::pair<int, int>> pairs;
          bool smallest = true;
          for (int si = 0; si < 4 && smallest; ++si)
            for (int ti = 0; ti < 4; ++ti)
              if (m.v(tcell, ti) == m.v(scell, si)) {
                if (m.v(tcell, ti) < v) {
                  smallest = false;
                  break;
                }
                pairs.push_back({ti, si});
              }
          if (!smallest) continue;
          size_t idx = std::find(configs.begin(), configs.end(), pairs) - configs.begin();
          if (idx == configs.size()) throw std::runtime_error("oracle: unknown quad adjacency");
          cell_pairs[idx].push_back({tcell, scell});
        }
    for (size_t ci = 0; ci < configs.size(); ++ci) {
      const Rule& r = rules[ci];
      for (auto& pr : cell_pairs[ci]) {
        for (int b = 0; b < nsb; ++b)
          for (int a = 0; a < ntb; ++a) {
            T e = T(0.0);
            for (int i = 0; i < r.n(); ++i) {
              PGeom x, y;
              qgeom(m, pr.first, &r.tp[2 * i], x);
              qgeom(m, pr.second, &r.sp[2 * i], y);
              double tv[4], t0[4], t1[4], sv[4], s0[4], s1[4];
              qtabulate(ts.degree, &r.tp[2 * i], tv, t0, t1);
              qtabulate(ss.degree, &r.sp[2 * i], sv, s0, s1);
              e += point_integrand<T>(op, helm, k, x, y, tv[a], t0[a], t1[a], sv[b], s0[b], s1[b]) *
                   r.w[i];
            }
            out[ts.cell_dofs[pr.first * ntb + a] + nt * ss.cell_dofs[pr.second * nsb + b]] += e;
          }
      }
    }
  }
}

thread_local std::string g_qerror;

}  // namespace

extern "C" {

const char* oracle_quad_last_error() { return g_qerror.c_str(); }

// Dense column-major assembly on a quadrilateral grid (cells: ncells x 4 point indices in
// ndelement's vertex order); the regular rule is the n x n Gauss tensor rule, n the
// smallest with n^2 >= q_regular.
int oracle_quad_assemble_dense(int helmholtz, int op, double k, const double* points,
                               int64_t npoints, const int64_t* cells, int64_t ncells,
                               int test_degree, int test_continuous, int trial_degree,
                               int trial_continuous, int q_regular, int q_singular,
                               int nthreads, int parts, void* out) {
  try {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    int n = 1;  // the smallest n with n^2 >= q_regular
    while (n * n < q_regular) ++n;
    QMesh m{points, npoints, cells, ncells, {}};
    m.build();
    QSpace ts = make_qspace(m, test_degree, test_continuous != 0);
    QSpace ss = make_qspace(m, trial_degree, trial_continuous != 0);
    if (helmholtz)
      qassemble<cplx>(m, ts, ss, op, true, k, n, q_singular, parts, static_cast<cplx*>(out));
    else
      qassemble<double>(m, ts, ss, op, false, k, n, q_singular, parts, static_cast<double*>(out));
    return 0;
  } catch (const std::exception& e) {
    g_qerror = e.what();
    return 1;
  }
}

int64_t oracle_quad_cell_dofs(const int64_t* cells, int64_t ncells, int64_t npoints, int degree,
                              int continuous, int64_t* cell_dofs) {
  QMesh m{nullptr, npoints, cells, ncells, {}};
  QSpace s = make_qspace(m, degree, continuous != 0);
  std::memcpy(cell_dofs, s.cell_dofs.data(), s.cell_dofs.size() * sizeof(int64_t));
  return s.ndofs;
}

// Duffy rule of quadrilateral configuration `config` (0..48, quad_configurations order);
// returns the number of points and fills the arrays when they are non-null.
int oracle_quad_duffy_rule(int config, int order, double* test_pts, double* trial_pts,
                           double* weights) {
  auto configs = quad_configurations();
  if (config < 0 || config >= static_cast<int>(configs.size())) return -1;
  Rule r = quad_duffy_rule(configs[config], order);
  if (test_pts) std::memcpy(test_pts, r.tp.data(), r.tp.size() * sizeof(double));
  if (trial_pts) std::memcpy(trial_pts, r.sp.data(), r.sp.size() * sizeof(double));
  if (weights) std::memcpy(weights, r.w.data(), r.w.size() * sizeof(double));
  return r.n();
}

}  // extern "C"
