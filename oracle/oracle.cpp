// CPU FP64 restatement of bempp-rs dense boundary-operator assembly.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA assembler: only the
// tests, the smoke check and the CPU-baseline leg of bench.py load it.  The product
// library never links or calls it.
//
// It restates, with the same loop structure and the same numerics, the path
//   BoundaryAssembler::assemble_into_memory       (src/boundary_assemblers.rs:176-214)
//   assemble_nonsingular_part / _batch_nonadjacent (src/boundary_assemblers.rs:396-521,689-773)
//   assemble_singular_part / make_cell_blocks      (src/boundary_assemblers.rs:234-393,564-606)
//   get_pairs_if_smallest / neighbours             (src/boundary_assemblers.rs:775-821)
//   Nonsingular/SingularCellPairAssembler          (src/boundary_assemblers/cell_pair_assemblers.rs)
//   integrands                                     (src/boundary_assemblers/integrands/*.rs)
//   operator factories                             (src/laplace.rs:34-78, src/helmholtz.rs:44-107)
//   DOF numbering and colouring                    (src/function.rs:281-445)
// The arithmetic of three unvendored crates is restated from published mathematics:
//   green-kernels (git main, no rev): G = 1/(4 pi r), e^{ikr}/(4 pi r); the derivative is
//     taken with respect to the target (= trial point y), as the call sites
//     src/boundary_assemblers/cell_pair_assemblers.rs:110-114,284-288 use it;
//   bempp-quadrature 0.1.0 `triangle_duffy`: Sauter & Schwab, Boundary Element Methods
//     (Springer 2011), section 5.2, regularising transformations for identical,
//     edge-adjacent and vertex-adjacent triangles with n-point Gauss-Legendre per axis;
//   ndelement (git main, no rev) `simplex_rule`: fully symmetric triangle rules by point
//     count (generated table, see gen_simplex_rules.py); Lagrange tabulation of degree 0, 1
//     and 2 with ndelement's DOF order on the reference triangle (vertices 0, 1, 2, then
//     the midpoints of edges 0 = [1,2], 1 = [0,2], 2 = [0,1]; nodal basis).
// Parity with bempp-rs itself is pinned by the bempp-cl golden matrices of
// tests/compare_to_bempp_cl.rs (absolute 1e-3 / 1e-4); the exact Duffy point sets of
// bempp-quadrature cannot be checked here (unpinned at the 1e-12 level).

#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace {

struct SimplexRuleEntry {
  int npoints;
  int degree;
  const double* points;
  const double* weights;
};
#include "simplex_rules_table.inc"

using cplx = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------
// Mesh topology and function spaces
// ---------------------------------------------------------------------------------------
struct Mesh {
  const double* pts;
  int64_t npts;
  const int64_t* cells;
  int64_t ncells;
  std::vector<std::vector<int64_t>> vertex_cells;  // upward connectivity, increasing cell
  void build() {
    vertex_cells.assign(npts, {});
    for (int64_t c = 0; c < ncells; ++c)
      for (int i = 0; i < 3; ++i) vertex_cells[cells[3 * c + i]].push_back(c);
  }
  int64_t v(int64_t c, int i) const { return cells[3 * c + i]; }
  // local edge i of cell c joins its vertices other than i (ndelement's reference
  // triangle: edges [1,2], [0,2], [0,1])
  std::pair<int64_t, int64_t> edge(int64_t c, int i) const {
    const int64_t a = v(c, (i + 1) % 3), b = v(c, (i + 2) % 3);
    return {std::min(a, b), std::max(a, b)};
  }
};

constexpr int kMaxBasis = 6;
inline int nbasis_of(int degree) { return degree == 0 ? 1 : degree == 1 ? 3 : 6; }

struct Space {
  int degree = 0;
  bool continuous = false;
  int nbasis = 1;
  int64_t ndofs = 0;
  std::vector<int64_t> cell_dofs;  // ncells * nbasis
};

// src/function.rs:365-445 (assign_dofs): cells in order, entities of each dimension in
// local order; the first visit of an entity allocates its DOFs.
Space make_space(const Mesh& m, int degree, bool continuous) {
  Space s;
  s.degree = degree;
  s.continuous = continuous;
  if (degree == 0) {
    s.nbasis = 1;
    s.ndofs = m.ncells;
    s.cell_dofs.resize(m.ncells);
    for (int64_t c = 0; c < m.ncells; ++c) s.cell_dofs[c] = c;
  } else if (degree == 1) {
    s.nbasis = 3;
    s.cell_dofs.resize(3 * m.ncells);
    if (continuous) {
      std::vector<int64_t> vdof(m.npts, -1);
      int64_t size = 0;
      for (int64_t c = 0; c < m.ncells; ++c)
        for (int i = 0; i < 3; ++i) {
          int64_t v = m.v(c, i);
          if (vdof[v] < 0) vdof[v] = size++;
          s.cell_dofs[3 * c + i] = vdof[v];
        }
      s.ndofs = size;
    } else {
      for (int64_t c = 0; c < 3 * m.ncells; ++c) s.cell_dofs[c] = c;
      s.ndofs = 3 * m.ncells;
    }
  } else if (degree == 2) {
    s.nbasis = 6;
    s.cell_dofs.resize(6 * m.ncells);
    if (continuous) {
      // per cell: its vertices, then its edges, each in local order
      std::vector<int64_t> vdof(m.npts, -1);
      std::map<std::pair<int64_t, int64_t>, int64_t> edof;
      int64_t size = 0;
      for (int64_t c = 0; c < m.ncells; ++c) {
        for (int i = 0; i < 3; ++i) {
          int64_t v = m.v(c, i);
          if (vdof[v] < 0) vdof[v] = size++;
          s.cell_dofs[6 * c + i] = vdof[v];
        }
        for (int i = 0; i < 3; ++i) {
          auto it = edof.find(m.edge(c, i));
          if (it == edof.end()) it = edof.emplace(m.edge(c, i), size++).first;
          s.cell_dofs[6 * c + 3 + i] = it->second;
        }
      }
      s.ndofs = size;
    } else {
      for (int64_t c = 0; c < 6 * m.ncells; ++c) s.cell_dofs[c] = c;
      s.ndofs = 6 * m.ncells;
    }
  } else {
    throw std::runtime_error("oracle: only degree 0, 1 and 2 Lagrange spaces");
  }
  return s;
}

// src/function.rs:281-351 (cell_colouring): greedy colouring over the lowest-dimensional
// entity that carries DOFs (vertices for P1, the cell itself for DP0/DP1).
std::vector<std::vector<int64_t>> colouring(const Mesh& m, const Space& s) {
  std::vector<std::vector<int64_t>> colours;
  bool vertex_based = s.continuous && s.degree >= 1;
  std::vector<std::vector<int>> entity_colours(vertex_based ? m.npts : m.ncells);
  for (int64_t c = 0; c < m.ncells; ++c) {
    std::vector<int64_t> ents;
    if (vertex_based)
      for (int i = 0; i < 3; ++i) ents.push_back(m.v(c, i));
    else
      ents.push_back(c);
    int col = 0;
    while (col < static_cast<int>(colours.size())) {
      bool found = false;
      for (int64_t e : ents)
        if (std::find(entity_colours[e].begin(), entity_colours[e].end(), col) !=
            entity_colours[e].end()) {
          found = true;
          break;
        }
      if (!found) break;
      ++col;
    }
    if (col == static_cast<int>(colours.size()))
      colours.push_back({c});
    else
      colours[col].push_back(c);
    for (int64_t e : ents) entity_colours[e].push_back(col);
  }
  return colours;
}

// ---------------------------------------------------------------------------------------
// Quadrature rules
// ---------------------------------------------------------------------------------------
void gauss_legendre01(int n, std::vector<double>& x, std::vector<double>& w) {
  // Newton iteration on P_n from the Chebyshev-like initial guess, mapped to [0, 1].
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

struct SimplexRule {
  std::vector<double> pts;  // 2 * n
  std::vector<double> wts;
};

SimplexRule simplex_rule(int npoints) {
  for (const auto& e : kSimplexRules)
    if (e.npoints == npoints) {
      SimplexRule r;
      r.pts.assign(e.points, e.points + 2 * npoints);
      r.wts.assign(e.weights, e.weights + npoints);
      return r;
    }
  throw std::runtime_error("oracle: no triangle rule with " + std::to_string(npoints) +
                           " points");
}

struct TestTrialRule {
  std::vector<double> test_pts, trial_pts, wts;
  int n() const { return static_cast<int>(wts.size()); }
};

// Reference-triangle coordinates of the point with barycentric coordinates mu with
// respect to local vertices (perm[0], perm[1], perm[2]); V0=(0,0), V1=(1,0), V2=(0,1).
inline void bary_to_ref(const double mu[3], const int perm[3], double* out) {
  out[0] = 0.0;
  out[1] = 0.0;
  for (int k = 0; k < 3; ++k) {
    if (perm[k] == 1) out[0] += mu[k];
    if (perm[k] == 2) out[1] += mu[k];
  }
}

// Sauter-Schwab regularising transformations on That = {0 <= x2 <= x1 <= 1} whose
// vertices P0=(0,0), P1=(1,0), P2=(1,1) give barycentric (1-x1, x1-x2, x2).  The shared
// vertex is P0, the shared edge is P0-P1.  `pairs` are (test_local, trial_local)
// vertex pairs sorted by trial local index (src/boundary_assemblers.rs:775-792).
TestTrialRule duffy_rule(const std::vector<std::pair<int, int>>& pairs, int order) {
  std::vector<double> g, gw;
  gauss_legendre01(order, g, gw);
  int tperm[3], sperm[3];
  int conn = static_cast<int>(pairs.size()) - 1;  // 0 vertex, 1 edge, 2 identical
  if (conn == 2) {
    for (int i = 0; i < 3; ++i) tperm[i] = sperm[i] = i;
  } else if (conn == 1) {
    tperm[0] = pairs[0].first;
    tperm[1] = pairs[1].first;
    tperm[2] = 3 - tperm[0] - tperm[1];
    sperm[0] = pairs[0].second;
    sperm[1] = pairs[1].second;
    sperm[2] = 3 - sperm[0] - sperm[1];
  } else {
    tperm[0] = pairs[0].first;
    sperm[0] = pairs[0].second;
    int k = 1;
    for (int i = 0; i < 3; ++i)
      if (i != tperm[0]) tperm[k++] = i;
    k = 1;
    for (int i = 0; i < 3; ++i)
      if (i != sperm[0]) sperm[k++] = i;
  }
  TestTrialRule r;
  auto push = [&](double x1, double x2, double y1, double y2, double w) {
    double mx[3] = {1.0 - x1, x1 - x2, x2};
    double my[3] = {1.0 - y1, y1 - y2, y2};
    double a[2], b[2];
    bary_to_ref(mx, tperm, a);
    bary_to_ref(my, sperm, b);
    r.test_pts.push_back(a[0]);
    r.test_pts.push_back(a[1]);
    r.trial_pts.push_back(b[0]);
    r.trial_pts.push_back(b[1]);
    r.wts.push_back(w);
  };
  int nregions = conn == 2 ? 6 : (conn == 1 ? 5 : 2);
  for (int reg = 0; reg < nregions; ++reg)
    for (int i0 = 0; i0 < order; ++i0)
      for (int i1 = 0; i1 < order; ++i1)
        for (int i2 = 0; i2 < order; ++i2)
          for (int i3 = 0; i3 < order; ++i3) {
            double xi = g[i0], e1 = g[i1], e2 = g[i2], e3 = g[i3];
            double wq = gw[i0] * gw[i1] * gw[i2] * gw[i3];
            if (conn == 2) {
              double w = wq * xi * xi * xi * e1 * e1 * e2;
              switch (reg) {
                case 0: push(xi, xi * (1 - e1 + e1 * e2), xi * (1 - e1 * e2 * e3), xi * (1 - e1), w); break;
                case 1: push(xi * (1 - e1 * e2 * e3), xi * (1 - e1), xi, xi * (1 - e1 + e1 * e2), w); break;
                case 2: push(xi, xi * e1 * (1 - e2 + e2 * e3), xi * (1 - e1 * e2), xi * e1 * (1 - e2), w); break;
                case 3: push(xi * (1 - e1 * e2), xi * e1 * (1 - e2), xi, xi * e1 * (1 - e2 + e2 * e3), w); break;
                case 4: push(xi * (1 - e1 * e2 * e3), xi * e1 * (1 - e2 * e3), xi, xi * e1 * (1 - e2), w); break;
                default: push(xi, xi * e1 * (1 - e2), xi * (1 - e1 * e2 * e3), xi * e1 * (1 - e2 * e3), w); break;
              }
            } else if (conn == 1) {
              double w0 = wq * xi * xi * xi * e1 * e1;
              double w = w0 * e2;
              switch (reg) {
                case 0: push(xi, xi * e1 * e3, xi * (1 - e1 * e2), xi * e1 * (1 - e2), w0); break;
                case 1: push(xi, xi * e1, xi * (1 - e1 * e2 * e3), xi * e1 * e2 * (1 - e3), w); break;
                case 2: push(xi * (1 - e1 * e2), xi * e1 * (1 - e2), xi, xi * e1 * e2 * e3, w); break;
                case 3: push(xi * (1 - e1 * e2 * e3), xi * e1 * e2 * (1 - e3), xi, xi * e1, w); break;
                default: push(xi * (1 - e1 * e2 * e3), xi * e1 * (1 - e2 * e3), xi, xi * e1 * e2, w); break;
              }
            } else {
              double w = wq * xi * xi * xi * e2;
              if (reg == 0)
                push(xi, xi * e1, xi * e2, xi * e2 * e3, w);
              else
                push(xi * e2, xi * e2 * e1, xi, xi * e3, w);
            }
          }
  return r;
}

// The 28 triangle-triangle adjacency configurations in the order the reference lists
// them (src/boundary_assemblers.rs:267-288): 9 vertex pairs, 18 edge pairs, 1 identical.
std::vector<std::vector<std::pair<int, int>>> singular_configurations() {
  std::vector<std::vector<std::pair<int, int>>> out;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out.push_back({{i, j}});
  const int edges[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  for (auto& te : edges)
    for (auto& se : edges) {
      out.push_back({{te[0], se[0]}, {te[1], se[1]}});
      out.push_back({{te[1], se[0]}, {te[0], se[1]}});
    }
  out.push_back({{0, 0}, {1, 1}, {2, 2}});
  return out;
}

// ---------------------------------------------------------------------------------------
// Geometry, kernels, integrands
// ---------------------------------------------------------------------------------------
struct CellGeom {
  double v0[3], t0[3], t1[3], n[3], jdet;
  void set(const Mesh& m, int64_t c) {
    const double* a = m.pts + 3 * m.v(c, 0);
    const double* b = m.pts + 3 * m.v(c, 1);
    const double* d = m.pts + 3 * m.v(c, 2);
    for (int i = 0; i < 3; ++i) {
      v0[i] = a[i];
      t0[i] = b[i] - a[i];
      t1[i] = d[i] - a[i];
    }
    double cx = t0[1] * t1[2] - t0[2] * t1[1];
    double cy = t0[2] * t1[0] - t0[0] * t1[2];
    double cz = t0[0] * t1[1] - t0[1] * t1[0];
    jdet = std::sqrt(cx * cx + cy * cy + cz * cz);
    n[0] = cx / jdet;
    n[1] = cy / jdet;
    n[2] = cz / jdet;
  }
  void point(const double* xi, double* x) const {
    for (int i = 0; i < 3; ++i) x[i] = v0[i] + xi[0] * t0[i] + xi[1] * t1[i];
  }
};

enum Op { kSingleLayer = 0, kDoubleLayer = 1, kAdjointDoubleLayer = 2, kHypersingular = 3 };

// basis tables: value, d/dxi0, d/dxi1 for basis b at reference point xi.  Degree 2: the
// nodal basis of the vertices and edge midpoints, with l0 = 1 - x - y, l1 = x, l2 = y:
// l_i (2 l_i - 1) at vertex i, then 4 l1 l2, 4 l0 l2, 4 l0 l1 at edges 0, 1, 2.
inline void tabulate(int degree, const double* xi, double val[kMaxBasis],
                     double d0[kMaxBasis], double d1[kMaxBasis]) {
  if (degree == 0) {
    val[0] = 1.0;
    d0[0] = 0.0;
    d1[0] = 0.0;
  } else if (degree == 1) {
    val[0] = 1.0 - xi[0] - xi[1];
    val[1] = xi[0];
    val[2] = xi[1];
    d0[0] = -1.0; d0[1] = 1.0; d0[2] = 0.0;
    d1[0] = -1.0; d1[1] = 0.0; d1[2] = 1.0;
  } else {
    const double l[3] = {1.0 - xi[0] - xi[1], xi[0], xi[1]};
    const double g0[3] = {-1.0, 1.0, 0.0}, g1[3] = {-1.0, 0.0, 1.0};  // grad l_i
    for (int i = 0; i < 3; ++i) {
      val[i] = l[i] * (2.0 * l[i] - 1.0);
      d0[i] = (4.0 * l[i] - 1.0) * g0[i];
      d1[i] = (4.0 * l[i] - 1.0) * g1[i];
    }
    const int ea[3] = {1, 0, 0}, eb[3] = {2, 2, 1};
    for (int e = 0; e < 3; ++e) {
      const int a = ea[e], b = eb[e];
      val[3 + e] = 4.0 * l[a] * l[b];
      d0[3 + e] = 4.0 * (l[a] * g0[b] + l[b] * g0[a]);
      d1[3 + e] = 4.0 * (l[a] * g1[b] + l[b] * g1[a]);
    }
  }
}

template <typename T>
struct KernelVals {
  T g;
  T grad[3];  // gradient with respect to the trial point y
};

template <typename T>
inline KernelVals<T> eval_kernel(double k, const double* x, const double* y);

template <>
inline KernelVals<double> eval_kernel<double>(double, const double* x, const double* y) {
  double d[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
  double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  KernelVals<double> kv;
  kv.g = 1.0 / (4.0 * kPi * r);
  double f = 1.0 / (4.0 * kPi * r * r * r);
  for (int i = 0; i < 3; ++i) kv.grad[i] = d[i] * f;
  return kv;
}

template <>
inline KernelVals<cplx> eval_kernel<cplx>(double k, const double* x, const double* y) {
  double d[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
  double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  cplx e(std::cos(k * r), std::sin(k * r));
  KernelVals<cplx> kv;
  kv.g = e / (4.0 * kPi * r);
  cplx f = e * cplx(1.0, -k * r) / (4.0 * kPi * r * r * r);
  for (int i = 0; i < 3; ++i) kv.grad[i] = d[i] * f;
  return kv;
}

template <typename T>
struct Integrand {
  int op;
  double k;
  // src/boundary_assemblers/integrands/*.rs; Helmholtz hypersingular adds
  // -k^2 * normal-normal term (src/helmholtz.rs:98-104)
  T eval(const KernelVals<T>& kv, int ta, int tb, const double* tv, const double* td0,
         const double* td1, const double* sv, const double* sd0, const double* sd1,
         const CellGeom& tg, const CellGeom& sg, bool helmholtz) const {
    switch (op) {
      case kSingleLayer:
        return kv.g * tv[ta] * sv[tb];
      case kDoubleLayer:
        return (kv.grad[0] * sg.n[0] + kv.grad[1] * sg.n[1] + kv.grad[2] * sg.n[2]) * tv[ta] *
               sv[tb];
      case kAdjointDoubleLayer:
        return -(kv.grad[0] * tg.n[0] + kv.grad[1] * tg.n[1] + kv.grad[2] * tg.n[2]) * tv[ta] *
               sv[tb];
      default: {
        double curl = 0.0;
        for (int c = 0; c < 3; ++c) {
          double a = tg.t1[c] * td0[ta] - tg.t0[c] * td1[ta];
          double b = sg.t1[c] * sd0[tb] - sg.t0[c] * sd1[tb];
          curl += a * b;
        }
        T val = kv.g * curl / tg.jdet / sg.jdet;
        if (helmholtz) {
          double nn = sg.n[0] * tg.n[0] + sg.n[1] * tg.n[1] + sg.n[2] * tg.n[2];
          val += -k * k * (kv.g * nn * tv[ta] * sv[tb]);
        }
        return val;
      }
    }
  }
};

bool share_vertex(const Mesh& m, int64_t a, int64_t b) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      if (m.v(a, i) == m.v(b, j)) return true;
  return false;
}

struct AssembleArgs {
  int helmholtz;
  int op;
  double k;
  int q_regular;
  int q_singular;
  int batch_size;
  int same_grid;
  int parts;  // bit 0: regular, bit 1: singular
  const int64_t* test_subset;
  int64_t n_subset;
};

template <typename T>
void assemble(const Mesh& m, const Space& test, const Space& trial, const AssembleArgs& a,
              T* out) {
  const int64_t nt = test.ndofs;
  Integrand<T> integ{a.op, a.k};
  const bool hel = a.helmholtz != 0;
  const int ntb = test.nbasis, nsb = trial.nbasis;

  if (a.parts & 1) {
    SimplexRule rule = simplex_rule(a.q_regular);
    const int Q = static_cast<int>(rule.wts.size());
    // tables: the reference tabulates the trial table at the test points
    // (src/boundary_assemblers.rs:464); identical rules on both sides make it the same.
    constexpr int B = kMaxBasis;
    std::vector<double> tv(Q * B), td0(Q * B), td1(Q * B), sv(Q * B), sd0(Q * B), sd1(Q * B);
    for (int p = 0; p < Q; ++p) {
      tabulate(test.degree, &rule.pts[2 * p], &tv[B * p], &td0[B * p], &td1[B * p]);
      tabulate(trial.degree, &rule.pts[2 * p], &sv[B * p], &sd0[B * p], &sd1[B * p]);
    }
    auto tcol = colouring(m, test);
    auto scol = colouring(m, trial);
    if (a.test_subset) {
      std::vector<char> keep(m.ncells, 0);
      for (int64_t i = 0; i < a.n_subset; ++i) keep[a.test_subset[i]] = 1;
      for (auto& c : tcol) {
        std::vector<int64_t> f;
        for (int64_t x : c)
          if (keep[x]) f.push_back(x);
        c.swap(f);
      }
    }
    const int bs = a.batch_size;
    for (const auto& tc : tcol)
      for (const auto& sc : scol) {
        std::vector<std::pair<int64_t, int64_t>> blocks;  // (test start, trial start)
        for (int64_t t0 = 0; t0 < static_cast<int64_t>(tc.size()); t0 += bs)
          for (int64_t s0 = 0; s0 < static_cast<int64_t>(sc.size()); s0 += bs)
            blocks.push_back({t0, s0});
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t bi = 0; bi < static_cast<int64_t>(blocks.size()); ++bi) {
          int64_t t0 = blocks[bi].first, s0 = blocks[bi].second;
          int64_t t1 = std::min<int64_t>(t0 + bs, tc.size());
          int64_t s1 = std::min<int64_t>(s0 + bs, sc.size());
          // test-geometry caching (cell_pair_assemblers.rs:194-259)
          std::vector<CellGeom> tgeo(t1 - t0);
          std::vector<double> tpts((t1 - t0) * Q * 3);
          for (int64_t i = t0; i < t1; ++i) {
            tgeo[i - t0].set(m, tc[i]);
            for (int p = 0; p < Q; ++p)
              tgeo[i - t0].point(&rule.pts[2 * p], &tpts[((i - t0) * Q + p) * 3]);
          }
          std::vector<KernelVals<T>> kmat(Q * Q);
          std::vector<double> spts(Q * 3);
          T local[kMaxBasis * kMaxBasis];
          for (int64_t j = s0; j < s1; ++j) {
            int64_t sc_cell = sc[j];
            CellGeom sg;
            sg.set(m, sc_cell);
            for (int q = 0; q < Q; ++q) sg.point(&rule.pts[2 * q], &spts[3 * q]);
            for (int64_t i = t0; i < t1; ++i) {
              int64_t tc_cell = tc[i];
              if (a.same_grid && share_vertex(m, tc_cell, sc_cell)) continue;
              const CellGeom& tg = tgeo[i - t0];
              const double* xp = &tpts[(i - t0) * Q * 3];
              for (int p = 0; p < Q; ++p)
                for (int q = 0; q < Q; ++q)
                  kmat[p * Q + q] = eval_kernel<T>(a.k, xp + 3 * p, &spts[3 * q]);
              // cell_pair_assemblers.rs:305-338: trial basis, test basis, test pt, trial pt
              for (int b = 0; b < nsb; ++b)
                for (int aa = 0; aa < ntb; ++aa) {
                  T e = T(0.0);
                  for (int p = 0; p < Q; ++p) {
                    double tw = rule.wts[p] * tg.jdet;
                    for (int q = 0; q < Q; ++q) {
                      e += integ.eval(kmat[p * Q + q], aa, b, &tv[B * p], &td0[B * p],
                                      &td1[B * p], &sv[B * q], &sd0[B * q], &sd1[B * q], tg,
                                      sg, hel) *
                           (rule.wts[q] * sg.jdet) * tw;
                    }
                  }
                  local[aa + ntb * b] = e;
                }
              for (int b = 0; b < nsb; ++b)
                for (int aa = 0; aa < ntb; ++aa)
                  out[test.cell_dofs[tc_cell * ntb + aa] +
                      nt * trial.cell_dofs[sc_cell * nsb + b]] += local[aa + ntb * b];
            }
          }
        }
      }
  }

  if ((a.parts & 2) && a.same_grid) {
    auto configs = singular_configurations();
    std::vector<TestTrialRule> rules;
    for (auto& c : configs) rules.push_back(duffy_rule(c, a.q_singular));
    // make_cell_blocks (src/boundary_assemblers.rs:564-606) with get_pairs_if_smallest
    std::vector<std::vector<std::pair<int64_t, int64_t>>> cell_pairs(configs.size());
    for (int64_t v = 0; v < m.npts; ++v)
      for (int64_t tcell : m.vertex_cells[v])
        for (int64_t scell : m.vertex_cells[v]) {
          std::vector<std::pair<int, int>> pairs;
          bool smallest = true;
          for (int si = 0; si < 3 && smallest; ++si)
            for (int ti = 0; ti < 3; ++ti)
              if (m.v(tcell, ti) == m.v(scell, si)) {
                if (m.v(tcell, ti) < v) {
                  smallest = false;
                  break;
                }
                pairs.push_back({ti, si});
              }
          if (!smallest) continue;
          size_t idx = std::find(configs.begin(), configs.end(), pairs) - configs.begin();
          cell_pairs[idx].push_back({tcell, scell});
        }
    struct Trip {
      int64_t row, col;
      T val;
    };
    std::vector<std::vector<Trip>> per_config(configs.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t ci = 0; ci < static_cast<int64_t>(configs.size()); ++ci) {
      const TestTrialRule& r = rules[ci];
      const int n = r.n();
      constexpr int B = kMaxBasis;
      std::vector<double> tv(n * B), td0(n * B), td1(n * B), sv(n * B), sd0(n * B), sd1(n * B);
      for (int i = 0; i < n; ++i) {
        tabulate(test.degree, &r.test_pts[2 * i], &tv[B * i], &td0[B * i], &td1[B * i]);
        tabulate(trial.degree, &r.trial_pts[2 * i], &sv[B * i], &sd0[B * i], &sd1[B * i]);
      }
      std::vector<KernelVals<T>> kv(n);
      for (auto& pr : cell_pairs[ci]) {
        CellGeom tg, sg;
        tg.set(m, pr.first);
        sg.set(m, pr.second);
        for (int i = 0; i < n; ++i) {
          double x[3], y[3];
          tg.point(&r.test_pts[2 * i], x);
          sg.point(&r.trial_pts[2 * i], y);
          kv[i] = eval_kernel<T>(a.k, x, y);
        }
        // cell_pair_assemblers.rs:129-151
        for (int b = 0; b < nsb; ++b)
          for (int aa = 0; aa < ntb; ++aa) {
            T e = T(0.0);
            for (int i = 0; i < n; ++i)
              e += integ.eval(kv[i], aa, b, &tv[B * i], &td0[B * i], &td1[B * i], &sv[B * i],
                              &sd0[B * i], &sd1[B * i], tg, sg, hel) *
                   (r.wts[i] * tg.jdet * sg.jdet);
            per_config[ci].push_back({test.cell_dofs[pr.first * ntb + aa],
                                      trial.cell_dofs[pr.second * nsb + b], e});
          }
      }
    }
    // serial dense add (src/boundary_assemblers.rs:208-213)
    for (auto& pc : per_config)
      for (auto& t : pc) out[t.row + nt * t.col] += t.val;
  }
}

thread_local std::string g_error;

}  // namespace

extern "C" {

const char* oracle_last_error() { return g_error.c_str(); }

// Dense assembly into `out` (column-major, n_test x n_trial; real f64 for Laplace,
// interleaved complex128 for Helmholtz).  `out` is accumulated into, not cleared.
// test_subset restricts the regular part to the listed test cells (NULL = all); it is
// how bench.py times a bounded sample.  Returns 0 on success.
int oracle_assemble_dense(int helmholtz, int op, double k, const double* points,
                          int64_t npoints, const int64_t* cells, int64_t ncells,
                          int test_degree, int test_continuous, int trial_degree,
                          int trial_continuous, int q_regular, int q_singular, int batch_size,
                          int nthreads, int parts, const int64_t* test_subset,
                          int64_t n_subset, void* out) {
  try {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    Mesh m{points, npoints, cells, ncells, {}};
    m.build();
    Space test = make_space(m, test_degree, test_continuous != 0);
    Space trial = make_space(m, trial_degree, trial_continuous != 0);
    AssembleArgs a{helmholtz, op, k, q_regular, q_singular, batch_size, 1, parts,
                   test_subset, n_subset};
    if (helmholtz)
      assemble<cplx>(m, test, trial, a, static_cast<cplx*>(out));
    else
      assemble<double>(m, test, trial, a, static_cast<double*>(out));
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

// DOF map of a degree-0/1/2 Lagrange space (src/function.rs:365-445); returns ndofs and
// writes ncells * nbasis DOF numbers.
int64_t oracle_cell_dofs(const int64_t* cells, int64_t ncells, int64_t npoints, int degree,
                         int continuous, int64_t* cell_dofs) {
  Mesh m{nullptr, npoints, cells, ncells, {}};
  Space s = make_space(m, degree, continuous != 0);
  std::memcpy(cell_dofs, s.cell_dofs.data(), s.cell_dofs.size() * sizeof(int64_t));
  return s.ndofs;
}

// Greedy colouring (src/function.rs:281-351): colour_of[c] for each cell; returns the
// number of colours.
int oracle_colouring(const int64_t* cells, int64_t ncells, int64_t npoints, int degree,
                     int continuous, int32_t* colour_of) {
  Mesh m{nullptr, npoints, cells, ncells, {}};
  Space s = make_space(m, degree, continuous != 0);
  auto cols = colouring(m, s);
  for (size_t c = 0; c < cols.size(); ++c)
    for (int64_t x : cols[c]) colour_of[x] = static_cast<int32_t>(c);
  return static_cast<int>(cols.size());
}

// Duffy rule of configuration `config` (0..27 in the reference's order) with 1-D order
// `order`; returns the number of points and fills the arrays when they are non-null.
int oracle_duffy_rule(int config, int order, double* test_pts, double* trial_pts,
                      double* weights) {
  auto configs = singular_configurations();
  if (config < 0 || config >= static_cast<int>(configs.size())) return -1;
  TestTrialRule r = duffy_rule(configs[config], order);
  if (test_pts) std::memcpy(test_pts, r.test_pts.data(), r.test_pts.size() * sizeof(double));
  if (trial_pts)
    std::memcpy(trial_pts, r.trial_pts.data(), r.trial_pts.size() * sizeof(double));
  if (weights) std::memcpy(weights, r.wts.data(), r.wts.size() * sizeof(double));
  return r.n();
}

// Symmetric triangle rule by point count; returns the count or -1.
int oracle_simplex_rule(int npoints, double* pts, double* wts) {
  try {
    SimplexRule r = simplex_rule(npoints);
    if (pts) std::memcpy(pts, r.pts.data(), r.pts.size() * sizeof(double));
    if (wts) std::memcpy(wts, r.wts.data(), r.wts.size() * sizeof(double));
    return npoints;
  } catch (...) {
    return -1;
  }
}

}  // extern "C"
