// Near field of a (test grid, trial grid) pair for the mixed-precision regular kernels.
//
// The mixed path integrates far pairs in FP32 and near pairs (centroid distance below
// twice the larger cell diameter) in FP64.  Rather than testing every pair inside the FP32
// kernel, the near pairs are found here once per grid pair: tiles of 32 consecutive cells
// get a bounding sphere, only tile pairs whose spheres come within twice the largest cell
// diameter are examined cell by cell, and each such tile pair gets a 32 x 32 bit mask
// (one word per test cell) of its near and vertex-sharing pairs.  The FP32 kernel skips
// the marked pairs; a second launch integrates the list of near pairs that share no
// vertex in FP64, one thread per pair (vertex-sharing pairs belong to the singular
// kernel).
#include <algorithm>
#include <cmath>

#include "core.h"

namespace bempp_b200 {

namespace {

constexpr int kTileCells = 32;

struct CellBall {
  double c[3];
  double diam;
};

std::vector<CellBall> cell_balls(const GridT& g) {
  std::vector<CellBall> out(static_cast<size_t>(g.ncells));
  for (int64_t c = 0; c < g.ncells; ++c) {
    const double* v[3] = {&g.points[3 * g.cells[3 * c]], &g.points[3 * g.cells[3 * c + 1]],
                          &g.points[3 * g.cells[3 * c + 2]]};
    CellBall& b = out[c];
    for (int d = 0; d < 3; ++d) b.c[d] = (v[0][d] + v[1][d] + v[2][d]) / 3.0;
    auto dist = [](const double* p, const double* q) {
      const double x = p[0] - q[0], y = p[1] - q[1], z = p[2] - q[2];
      return std::sqrt(x * x + y * y + z * z);
    };
    b.diam = std::max(dist(v[0], v[1]), std::max(dist(v[0], v[2]), dist(v[1], v[2])));
  }
  return out;
}

struct TileBall {
  double c[3];
  double rad;   // largest centroid distance from c
  double diam;  // largest cell diameter
};

std::vector<TileBall> tile_balls(const std::vector<CellBall>& cells) {
  const size_t n = cells.size(), nt = (n + kTileCells - 1) / kTileCells;
  std::vector<TileBall> out(nt);
  for (size_t t = 0; t < nt; ++t) {
    const size_t c0 = t * kTileCells, c1 = std::min(n, c0 + kTileCells);
    TileBall& b = out[t];
    b.c[0] = b.c[1] = b.c[2] = 0.0;
    b.diam = 0.0;
    for (size_t c = c0; c < c1; ++c) {
      for (int d = 0; d < 3; ++d) b.c[d] += cells[c].c[d];
      b.diam = std::max(b.diam, cells[c].diam);
    }
    for (int d = 0; d < 3; ++d) b.c[d] /= static_cast<double>(c1 - c0);
    b.rad = 0.0;
    for (size_t c = c0; c < c1; ++c) {
      const double x = cells[c].c[0] - b.c[0], y = cells[c].c[1] - b.c[1], z = cells[c].c[2] - b.c[2];
      b.rad = std::max(b.rad, std::sqrt(x * x + y * y + z * z));
    }
  }
  return out;
}

bool share_vertex(const GridT& a, int64_t i, const GridT& b, int64_t j) {
  for (int u = 0; u < 3; ++u)
    for (int v = 0; v < 3; ++v)
      if (a.vtx()[3 * i + u] == b.vtx()[3 * j + v]) return true;
  return false;
}

}  // namespace

const NearField& near_field(GridT& test, GridT& trial) {
  std::lock_guard<std::mutex> lock(test.mu);
  auto& slot = test.near_fields[trial.uid];
  if (slot) return *slot;
  const bool same = &test == &trial;
  const std::vector<CellBall> tc = cell_balls(test);
  const std::vector<CellBall> sc = same ? tc : cell_balls(trial);
  const std::vector<TileBall> tt = tile_balls(tc), st = tile_balls(sc);
  const int ntt = static_cast<int>(tt.size()), nst = static_cast<int>(st.size());

  std::vector<int> tile_mask(static_cast<size_t>(ntt) * nst, -1);
  std::vector<unsigned> masks;
  std::vector<int2> pairs;
  size_t marked = 0;
  int nmasks = 0;
  for (int a = 0; a < ntt; ++a)
    for (int b = 0; b < nst; ++b) {
      const TileBall &A = tt[a], &B = st[b];
      const double dx = A.c[0] - B.c[0], dy = A.c[1] - B.c[1], dz = A.c[2] - B.c[2];
      const double reach = (A.rad + B.rad + 2.0 * std::max(A.diam, B.diam)) * (1.0 + 1e-9) + 1e-300;
      if (dx * dx + dy * dy + dz * dz >= reach * reach) continue;
      unsigned words[kTileCells] = {};
      bool any = false;
      const int64_t i0 = static_cast<int64_t>(a) * kTileCells, j0 = static_cast<int64_t>(b) * kTileCells;
      const int64_t ni = std::min<int64_t>(kTileCells, test.ncells - i0);
      const int64_t nj = std::min<int64_t>(kTileCells, trial.ncells - j0);
      for (int64_t i = 0; i < ni; ++i)
        for (int64_t j = 0; j < nj; ++j) {
          const CellBall &x = tc[i0 + i], &y = sc[j0 + j];
          const double ex = x.c[0] - y.c[0], ey = x.c[1] - y.c[1], ez = x.c[2] - y.c[2];
          const double lim = 2.0 * std::max(x.diam, y.diam);
          const bool adjacent = same && share_vertex(test, i0 + i, trial, j0 + j);
          const bool near = ex * ex + ey * ey + ez * ez < lim * lim;
          if (near || adjacent) {
            words[i] |= 1u << j;
            any = true;
            ++marked;
            if (!adjacent)
              pairs.push_back(make_int2(static_cast<int>(i0 + i), static_cast<int>(j0 + j)));
          }
        }
      if (!any) continue;
      tile_mask[static_cast<size_t>(a) * nst + b] = nmasks++;
      masks.insert(masks.end(), words, words + kTileCells);
    }

  auto nf = std::make_unique<NearField>();
  nf->test_tiles = ntt;
  nf->trial_tiles = nst;
  nf->npairs = static_cast<int>(pairs.size());
  nf->marked = marked;
  nf->tile_mask.upload(tile_mask);
  if (!masks.empty()) nf->masks.upload(masks);
  if (!pairs.empty()) nf->pairs.upload(pairs);
  slot = std::move(nf);
  return *slot;
}

}  // namespace bempp_b200
