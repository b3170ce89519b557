// Grid topology, DOF maps and the host-side layouts the kernels consume.
//
//   make_space:      DOF numbering of Lagrange degree 0/1 spaces exactly as bempp-rs
//                    assign_dofs (src/function.rs:365-445): cells in order, sub-entities
//                    of each dimension in local order, the first visit allocates DOFs.
//   cell_colouring:  greedy colouring of src/function.rs:281-351 (kept for API parity
//                    and tests; the GPU kernels do not need it).
//   singular pairs:  make_cell_blocks + get_pairs_if_smallest
//                    (src/boundary_assemblers.rs:564-606,775-792): each ordered pair of
//                    cells sharing a vertex, once, with its (test_local, trial_local)
//                    vertex pairing mapped to one of the 28 configurations.
//   tiles:           the DOFs touched by each run of 32 consecutive cells, for the
//                    tile-scatter kernel.
#include <algorithm>
#include <cmath>
#include <cstring>

#include <functional>
#include <thread>
#include <string>
#include "core.h"

void GridT::build_topology() {
  if (!vertex_cells.empty() || ncells == 0) return;
  const int* vx = vtx();
  const int n = nv();
  // counts, offsets, then the cells in increasing order
  auto& off = vertex_cells.off;
  off.assign(static_cast<size_t>(nverts()) + 1, 0);
  for (int64_t i = 0; i < n * ncells; ++i) ++off[vx[i] + 1];
  for (size_t v = 1; v < off.size(); ++v) off[v] += off[v - 1];
  vertex_cells.items.resize(static_cast<size_t>(n * ncells));
  std::vector<int64_t> next(off.begin(), off.end() - 1);
  for (int64_t c = 0; c < ncells; ++c)
    for (int i = 0; i < n; ++i) vertex_cells.items[next[vx[n * c + i]]++] = static_cast<int>(c);
}

// Edges of a triangle grid, built for the spaces with edge DOFs (degree 2) only; the
// quadrilateral spaces (degree <= 1) have none.
void GridT::build_edges() {
  if (!cell_edges.empty() || ncells == 0 || quads()) return;
  const int* vx = vtx();
  if (!given_cell_edges.empty()) {
    // ndgrid's own edge numbering (validated when the grid was created)
    const int64_t ne = static_cast<int64_t>(given_edge_vertices.size() / 2);
    edges.resize(ne);
    for (int64_t e = 0; e < ne; ++e) {
      const int a = given_edge_vertices[2 * e], b = given_edge_vertices[2 * e + 1];
      edges[e] = {std::min(a, b), std::max(a, b)};
    }
    cell_edges.resize(ncells);
    for (int64_t c = 0; c < ncells; ++c)
      for (int i = 0; i < 3; ++i) cell_edges[c][i] = given_cell_edges[3 * c + i];
    return;
  }
  // edges: numbered in first-visit order over cells and local edges [1,2], [0,2], [0,1]
  // (an open-addressing hash table of the packed vertex pairs)
  cell_edges.resize(ncells);
  const int local[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  size_t cap = 16;
  while (cap < static_cast<size_t>(6 * ncells)) cap <<= 1;
  std::vector<uint64_t> keys(cap, ~uint64_t(0));
  std::vector<int> vals(cap, -1);
  for (int64_t c = 0; c < ncells; ++c)
    for (int e = 0; e < 3; ++e) {
      const int a = vx[3 * c + local[e][0]], b = vx[3 * c + local[e][1]];
      const uint64_t key = (static_cast<uint64_t>(std::min(a, b)) << 32) | static_cast<uint32_t>(std::max(a, b));
      size_t h = static_cast<size_t>((key * 0x9E3779B97F4A7C15ull) >> 17) & (cap - 1);
      while (keys[h] != key && keys[h] != ~uint64_t(0)) h = (h + 1) & (cap - 1);
      if (keys[h] != key) {
        keys[h] = key;
        vals[h] = static_cast<int>(edges.size());
        edges.push_back({std::min(a, b), std::max(a, b)});
      }
      cell_edges[c][e] = vals[h];
    }
}

namespace bempp_b200 {

SpaceT* make_space(GridT* grid, const ElementFamilyT& fam) {
  if (fam.degree > 2)
    throw Error(kUnsupported, "only Lagrange degree 0, 1 and 2 spaces are supported");
  std::lock_guard<std::mutex> lock(grid->mu);
  if (grid->quads() && fam.degree > 1)
    throw Error(kUnsupported, "quadrilateral grids: Lagrange degree 0 and 1 spaces only");
  grid->build_topology();
  if (fam.degree == 2) grid->build_edges();
  auto* s = new SpaceT();
  s->grid = grid;
  s->degree = fam.degree;
  s->continuous = fam.continuity == 0 && fam.degree >= 1;
  s->dtype = fam.dtype;
  const int64_t nc = grid->ncells;
  // DOF of each vertex and edge (-1: none yet); a cell's interior DOFs are
  // [per_cell * c, per_cell * (c + 1))
  std::vector<int64_t> vdof(static_cast<size_t>(grid->nverts()), -1),
      edof(grid->edges.size(), -1);
  int per_cell = 0;
  if (grid->quads() && fam.degree == 1) {
    // Q1 (one DOF per vertex, first visit) or DQ1 (four interior DOFs per cell)
    s->nbasis = 4;
    s->cell_dofs.resize(4 * nc);
    int64_t size = 0;
    for (int64_t c = 0; c < nc; ++c)
      for (int i = 0; i < 4; ++i) {
        if (s->continuous) {
          int64_t& d = vdof[grid->vtx()[4 * c + i]];
          if (d < 0) d = size++;
          s->cell_dofs[4 * c + i] = d;
        } else {
          s->cell_dofs[4 * c + i] = size++;
        }
      }
    if (!s->continuous) per_cell = 4;
    s->ndofs = size;
  } else if (fam.degree == 0) {
    // DP0: one DOF on the cell itself (Lagrange degree 0 is discontinuous)
    s->nbasis = 1;
    s->cell_dofs.resize(nc);
    for (int64_t c = 0; c < nc; ++c) s->cell_dofs[c] = c;
    per_cell = 1;
    s->ndofs = nc;
  } else if (fam.degree == 1 && s->continuous) {
    s->nbasis = 3;
    s->cell_dofs.resize(3 * nc);
    int64_t size = 0;
    for (int64_t c = 0; c < nc; ++c)
      for (int i = 0; i < 3; ++i) {
        int64_t& d = vdof[grid->vtx()[3 * c + i]];
        if (d < 0) d = size++;
        s->cell_dofs[3 * c + i] = d;
      }
    s->ndofs = size;
  } else if (fam.degree == 2 && s->continuous) {
    // P2: per cell its vertices, then its edges (local edge i opposite vertex i), the
    // first visit of an entity allocating its DOF (src/function.rs:409-440)
    s->nbasis = 6;
    s->cell_dofs.resize(6 * nc);
    int64_t size = 0;
    for (int64_t c = 0; c < nc; ++c) {
      for (int i = 0; i < 3; ++i) {
        int64_t& d = vdof[grid->vtx()[3 * c + i]];
        if (d < 0) d = size++;
        s->cell_dofs[6 * c + i] = d;
      }
      for (int i = 0; i < 3; ++i) {
        int64_t& d = edof[grid->cell_edges[c][i]];
        if (d < 0) d = size++;
        s->cell_dofs[6 * c + 3 + i] = d;
      }
    }
    s->ndofs = size;
  } else {
    // DP1 / DP2: every DOF belongs to the cell interior
    const int nb = fam.degree == 1 ? 3 : 6;
    s->nbasis = nb;
    s->cell_dofs.resize(nb * nc);
    for (int64_t i = 0; i < nb * nc; ++i) s->cell_dofs[i] = i;
    per_cell = nb;
    s->ndofs = nb * nc;
  }
  // entity -> DOFs rows: vertices and edges hold at most one DOF each
  for (int dim = 0; dim < 2; ++dim) {
    const std::vector<int64_t>& one = dim == 0 ? vdof : edof;
    auto& r = s->entity_dofs[dim];
    r.off.assign(one.size() + 1, 0);
    for (size_t e = 0; e < one.size(); ++e) r.off[e + 1] = r.off[e] + (one[e] >= 0 ? 1 : 0);
    r.items.reserve(static_cast<size_t>(r.off.back()));
    for (int64_t d : one)
      if (d >= 0) r.items.push_back(d);
  }
  auto& rc = s->entity_dofs[2];
  rc.off.resize(static_cast<size_t>(nc) + 1);
  for (int64_t c = 0; c <= nc; ++c) rc.off[c] = per_cell * c;
  rc.items.resize(static_cast<size_t>(per_cell * nc));
  for (int64_t i = 0; i < per_cell * nc; ++i) rc.items[i] = i;
  return s;
}

std::vector<std::vector<int64_t>> cell_colouring(const SpaceT& s) {
  const GridT& g = *s.grid;
  const bool vertex_based = s.continuous;
  std::vector<std::vector<int64_t>> colours;
  std::vector<std::vector<int>> entity_colours(vertex_based ? g.nverts() : g.ncells);
  const int nv = g.nv();
  for (int64_t c = 0; c < g.ncells; ++c) {
    int ents[4];
    int ne = 0;
    if (vertex_based)
      for (int i = 0; i < nv; ++i) ents[ne++] = g.vtx()[nv * c + i];
    else
      ents[ne++] = static_cast<int>(c);
    int col = 0;
    for (; col < static_cast<int>(colours.size()); ++col) {
      bool used = false;
      for (int e = 0; e < ne && !used; ++e)
        used = std::find(entity_colours[ents[e]].begin(), entity_colours[ents[e]].end(), col) !=
               entity_colours[ents[e]].end();
      if (!used) break;
    }
    if (col == static_cast<int>(colours.size())) colours.emplace_back();
    colours[col].push_back(c);
    for (int e = 0; e < ne; ++e) entity_colours[ents[e]].push_back(col);
  }
  return colours;
}

namespace {

// Index in quad_singular_configurations() of the shared-vertex pairing (ts[i], ss[i]),
// i < n, trial local ascending: 16 vertex pairings (test * 4 + trial), 32 edge pairings
// (16 + (test edge * 4 + trial edge) * 2 + orientation, edges [0,1], [0,2], [1,3],
// [2,3]), the identical cell 48; -1 for anything else.
int quad_configuration(const int* ts, const int* ss, int n) {
  auto edge = [](int a, int b) {
    const int lo = std::min(a, b), hi = std::max(a, b);
    if (lo == 0 && hi == 1) return 0;
    if (lo == 0 && hi == 2) return 1;
    if (lo == 1 && hi == 3) return 2;
    if (lo == 2 && hi == 3) return 3;
    return -1;
  };
  if (n == 1) return ts[0] * 4 + ss[0];
  if (n == 2) {
    const int et = edge(ts[0], ts[1]), es = edge(ss[0], ss[1]);
    if (et < 0 || es < 0) return -1;
    // orientation 0: the trial edge's first vertex meets the test edge's first vertex
    return 16 + (et * 4 + es) * 2 + (ts[0] < ts[1] ? 0 : 1);
  }
  if (n == 4 && ts[0] == 0 && ts[1] == 1 && ts[2] == 2 && ts[3] == 3) return 48;
  return -1;
}

}  // namespace

// Singular pair enumeration; pairs grouped by configuration (as cell_pairs[config] in
// make_cell_blocks), vertices visited in increasing order.
void build_singular_pairs(GridT& g, SingularPairList& out) {
  // Candidate pairs are enumerated vertex by vertex, each kept by its smallest shared
  // vertex.  Contiguous vertex ranges go to host threads; concatenating their per-
  // configuration lists in range order gives exactly the serial order (configuration,
  // then vertex, then test cell, then trial cell).
  const bool quads = g.quads();
  const int cv = g.nv();  // vertices per cell
  const int ncfg = static_cast<int>(quads ? quad_singular_configurations().size()
                                          : singular_configurations().size());
  const int64_t nv = g.nverts();
  const int nthreads = static_cast<int>(std::max<int64_t>(
      1, std::min<int64_t>({static_cast<int64_t>(std::thread::hardware_concurrency()), 16,
                            nv / 1024})));
  std::vector<std::vector<std::vector<std::pair<int, int>>>> parts(
      nthreads, std::vector<std::vector<std::pair<int, int>>>(ncfg));
  const int* cells = g.vtx();  // topology vertices
  std::vector<std::string> errors(nthreads);
  auto work = [&](int t) {
    auto& by_cfg = parts[t];
    const int64_t v0 = nv * t / nthreads, v1 = nv * (t + 1) / nthreads;
    for (auto& b : by_cfg) b.reserve(static_cast<size_t>((v1 - v0) * 2) + 16);
    for (int64_t v = v0; v < v1; ++v)
      for (int tc : g.vertex_cells[v])
        for (int sc : g.vertex_cells[v]) {
          // shared vertices as (test local, trial local), trial local ascending; the pair
          // belongs to its smallest shared vertex
          int ts[4], ss[4], n = 0;
          bool smallest = true;
          for (int si = 0; si < cv && smallest; ++si)
            for (int ti = 0; ti < cv; ++ti)
              if (cells[cv * tc + ti] == cells[cv * sc + si]) {
                if (cells[cv * tc + ti] < v) {
                  smallest = false;
                  break;
                }
                ts[n] = ti;
                ss[n] = si;
                ++n;
              }
          if (!smallest) continue;
          // configuration index in the order of singular_configurations(): 9 vertex
          // pairings (test * 3 + trial), 18 edge pairings (edges opposite et / es, two
          // orientations), identical cells last
          int cfg = -1;
          if (quads) {
            cfg = quad_configuration(ts, ss, n);
          } else if (n == 1) {
            cfg = ts[0] * 3 + ss[0];
          } else if (n == 2) {
            const int et = 3 - ts[0] - ts[1], es = 3 - ss[0] - ss[1];
            cfg = 9 + (et * 3 + es) * 2 + (ts[0] < ts[1] ? 0 : 1);
          } else if (n == 3 && ts[0] == 0 && ts[1] == 1 && ts[2] == 2) {
            cfg = 27;
          }
          if (cfg < 0 || cfg >= ncfg) {
            errors[t] = "unknown adjacency configuration";
            return;
          }
          by_cfg[cfg].push_back({tc, sc});
        }
  };
  auto run = [&](const std::function<void(int)>& fn) {
    if (nthreads == 1) {
      fn(0);
      return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) pool.emplace_back(fn, t);
    for (auto& th : pool) th.join();
  };
  run(work);
  for (const auto& e : errors)
    if (!e.empty()) throw Error(kInternal, e);
  // slice of (configuration c, thread t) in the output: configuration-major, then threads
  std::vector<size_t> start(static_cast<size_t>(ncfg) * nthreads + 1, 0);
  for (int c = 0; c < ncfg; ++c)
    for (int t = 0; t < nthreads; ++t)
      start[c * nthreads + t + 1] = start[c * nthreads + t] + parts[t][c].size();
  const size_t total = start.back();
  out.test_cell.resize(total);
  out.trial_cell.resize(total);
  out.config.resize(total);
  run([&](int t) {
    for (int c = 0; c < ncfg; ++c) {
      size_t o = start[c * nthreads + t];
      for (const auto& p : parts[t][c]) {
        out.test_cell[o] = p.first;
        out.trial_cell[o] = p.second;
        out.config[o] = c;
        ++o;
      }
    }
  });
}

// Tile layout for the scatter kernel: tiles of `tile` consecutive cells, their sorted
// unique DOFs, and each cell's DOFs as indices into its tile's list.
// Also the incidence of each tile's local DOFs: for local DOF d of tile t, the entries
// inc_ent[t * 3 * tile + k], k in [inc_off[t * (3 * tile + 1) + d], ... + d + 1), each
// b * tile + c for the cell c of the tile whose local basis function b is DOF d (cells
// ascending, then b).
void build_tiles(const SpaceT& s, int tile, std::vector<int>& off, std::vector<int>& dofs,
                 std::vector<uint8_t>& ldof, int& max_dofs, std::vector<uint8_t>& inc_off,
                 std::vector<uint8_t>& inc_ent) {
  const int64_t nc = s.grid->ncells;
  const int nb = s.nbasis;
  const int ntiles = static_cast<int>((nc + tile - 1) / tile);
  off.assign(ntiles + 1, 0);
  dofs.clear();
  ldof.assign(nc * nb, 0);
  max_dofs = 0;
  // the DOF incidence serves the P1 / DP1 gather of the tiled kernels only (degree-2
  // spaces use the generic pair kernel)
  const bool incidence = nb <= 3;
  inc_off.assign(incidence ? static_cast<size_t>(ntiles) * (3 * tile + 1) : 0, 0);
  inc_ent.assign(incidence ? static_cast<size_t>(ntiles) * 3 * tile : 0, 0);
  std::vector<int> local, count;
  for (int t = 0; t < ntiles; ++t) {
    const int64_t c0 = static_cast<int64_t>(t) * tile, c1 = std::min<int64_t>(c0 + tile, nc);
    local.clear();
    for (int64_t c = c0; c < c1; ++c)
      for (int b = 0; b < nb; ++b) local.push_back(static_cast<int>(s.cell_dofs[c * nb + b]));
    std::sort(local.begin(), local.end());
    local.erase(std::unique(local.begin(), local.end()), local.end());
    for (int64_t c = c0; c < c1; ++c)
      for (int b = 0; b < nb; ++b) {
        int d = static_cast<int>(s.cell_dofs[c * nb + b]);
        ldof[c * nb + b] =
            static_cast<uint8_t>(std::lower_bound(local.begin(), local.end(), d) - local.begin());
      }
    dofs.insert(dofs.end(), local.begin(), local.end());
    off[t + 1] = static_cast<int>(dofs.size());
    max_dofs = std::max<int>(max_dofs, static_cast<int>(local.size()));
    if (!incidence) continue;
    // incidence (counting sort of the tile's (cell, basis) entries by local DOF)
    const int nd = static_cast<int>(local.size());
    uint8_t* io = &inc_off[static_cast<size_t>(t) * (3 * tile + 1)];
    uint8_t* ie = &inc_ent[static_cast<size_t>(t) * 3 * tile];
    count.assign(nd + 1, 0);
    for (int64_t c = c0; c < c1; ++c)
      for (int b = 0; b < nb; ++b) ++count[ldof[c * nb + b] + 1];
    for (int d = 0; d < nd; ++d) count[d + 1] += count[d];
    for (int d = 0; d <= nd; ++d) io[d] = static_cast<uint8_t>(count[d]);
    for (int64_t c = c0; c < c1; ++c)
      for (int b = 0; b < nb; ++b)
        ie[count[ldof[c * nb + b]]++] = static_cast<uint8_t>(b * tile + (c - c0));
  }
}

}  // namespace bempp_b200

// Largest distance from a cell's centroid to its vertices: bounds |x - c_x| for every
// point of the cell (the mixed-precision kernels' phase bound k (rad_x + rad_y)).
double GridT::max_circumradius() {
  std::lock_guard<std::mutex> lock(mu);
  if (max_rad >= 0.0) return max_rad;
  double m = 0.0;
  const int n = nv();
  for (int64_t c = 0; c < ncells; ++c) {
    const double* v[4];
    for (int i = 0; i < n; ++i) v[i] = &points[3 * cells[n * c + i]];
    double cen[3];
    for (int d = 0; d < 3; ++d) {
      cen[d] = 0.0;
      for (int i = 0; i < n; ++i) cen[d] += v[i][d];
      cen[d] /= n;
    }
    for (int i = 0; i < n; ++i) {
      const double x = v[i][0] - cen[0], y = v[i][1] - cen[1], z = v[i][2] - cen[2];
      m = std::max(m, std::sqrt(x * x + y * y + z * z));
    }
  }
  max_rad = m;
  return m;
}

