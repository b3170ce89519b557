// Assembly driver: device-resident caches and the kernel sequence of one dense assembly.
//
// bempp-rs BoundaryAssembler::assemble_into_memory (src/boundary_assemblers.rs:176-214)
// runs the regular part over coloured 128x128 cell blocks with rayon, then the singular
// part into COO triplets, then adds the triplets serially.  Here one assembly is a short
// stream-ordered kernel sequence on the caller's stream:
//   1. geometry (once per grid and regular rule, cached on the device),
//   2. regular part: DP0 x DP0 -> direct-store kernel (writes every entry);
//      otherwise memset + tile-scatter kernel,
//   3. singular part: one warp per adjacent cell pair, added into the dense output,
//   4. F32 / C32 outputs: one conversion pass from the FP64 staging buffer.
// Vertex-sharing pairs are skipped by the regular kernels exactly when test and trial
// spaces live on the same grid object (pointer equality, as equal_grids at
// src/boundary_assemblers/helpers.rs:59-64).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>

#include "core.h"

namespace bempp_b200 {

void build_singular_pairs(GridT& g, SingularPairList& out);
void build_tiles(const SpaceT& s, int tile, std::vector<int>& off, std::vector<int>& dofs,
                 std::vector<uint8_t>& ldof, int& max_dofs, std::vector<uint8_t>& inc_off,
                 std::vector<uint8_t>& inc_ent);
int scatter_tile_cells();
cudaError_t launch_convert_to_single(const double* src, void* dst, size_t n_reals,
                                     cudaStream_t stream);

size_t dtype_size(uint8_t dtype) {
  switch (dtype) {
    case 0: return 4;
    case 1: return 8;
    case 2: return 8;
    case 3: return 16;
    default: throw Error(kInvalidArgument, "unknown dtype");
  }
}

namespace {

int current_device() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw Error(kNoDevice, std::string("no CUDA device: ") + cudaGetErrorString(e));
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    throw Error(kNoDevice, "no CUDA device");
  return dev;
}

// Duffy rules per (device, order), shared by all assemblers.
struct DeviceRules {
  DeviceBuffer offset, test_xi, trial_xi, w;
  int total = 0;
};
std::mutex g_rules_mu;
std::map<std::tuple<int, int, bool>, std::unique_ptr<DeviceRules>> g_rules;

// the 28 triangle configurations, or the 49 quadrilateral ones
const DeviceRules& device_rules(int device, int order, bool quads = false) {
  std::lock_guard<std::mutex> lock(g_rules_mu);
  auto& slot = g_rules[std::make_tuple(device, order, quads)];
  if (!slot) {
    auto r = std::make_unique<DeviceRules>();
    std::vector<int> off{0};
    std::vector<double> txi, sxi, w;
    const size_t ncfg =
        quads ? quad_singular_configurations().size() : singular_configurations().size();
    for (size_t c = 0; c < ncfg; ++c) {
      DuffyRule d = quads ? quad_duffy_rule(static_cast<int>(c), order)
                          : duffy_rule(static_cast<int>(c), order);
      txi.insert(txi.end(), d.test_xi.begin(), d.test_xi.end());
      sxi.insert(sxi.end(), d.trial_xi.begin(), d.trial_xi.end());
      w.insert(w.end(), d.w.begin(), d.w.end());
      off.push_back(static_cast<int>(w.size()));
    }
    r->offset.upload(off);
    r->test_xi.upload(txi);
    r->trial_xi.upload(sxi);
    r->w.upload(w);
    r->total = static_cast<int>(w.size());
    slot = std::move(r);
  }
  return *slot;
}

void ensure_grid_device(GridT& g, int device) {
  if (g.device == device && g.d_points.ptr) return;
  if (g.device != -1 && g.device != device)
    throw Error(kUnsupported, "a grid is bound to the device it was first assembled on");
  if (g.ncells > INT32_MAX / 3 || g.npoints > INT32_MAX)
    throw Error(kUnsupported, "grid too large for 32-bit cell indices");
  g.d_points.upload(g.points);
  g.d_cells.upload(g.cells);
  if (!g.topo.empty()) g.d_topo.upload(g.topo);
  g.device = device;
}

const GridGeometry& grid_geometry(GridT& g, int device, const RegularRule& rule,
                                  cudaStream_t stream, size_t& launches) {
  std::lock_guard<std::mutex> lock(g.mu);
  ensure_grid_device(g, device);
  auto& slot = g.geometry[rule.npts];
  if (!slot) {
    auto geo = std::make_unique<GridGeometry>();
    const size_t n = g.ncells;
    geo->npts = rule.npts;
    const size_t S = static_cast<size_t>(cell_stride(static_cast<int>(n)));  // padded rows
    geo->geom.alloc(sizeof(double) * kNumGeomFields * S);
    geo->qpts.alloc(sizeof(double) * 3 * rule.npts * S);
    geo->qrel.alloc(sizeof(float4) * qrel_rows(rule.npts) * S);
    geo->vids.alloc(sizeof(int) * 3 * S);
    BEMPP_CUDA(launch_geometry(g.d_points.as<double>(), g.d_cells.as<int>(),
                               g.topo.empty() ? nullptr : g.d_topo.as<int>(),
                               static_cast<int>(n), rule, geo->geom.as<double>(),
                               geo->qpts.as<double>(), geo->qrel.as<float4>(),
                               geo->vids.as<int>(), stream));
    ++launches;
    // the cache is shared by every stream that assembles on this grid: finish it now
    // (unless the stream is being captured, where later nodes of the graph order after it)
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    BEMPP_CUDA(cudaStreamIsCapturing(stream, &cap));
    if (cap == cudaStreamCaptureStatusNone) BEMPP_CUDA(cudaStreamSynchronize(stream));
    slot = std::move(geo);
  }
  return *slot;
}

SingularPairList& grid_pairs(GridT& g, int device) {
  std::lock_guard<std::mutex> lock(g.mu);
  ensure_grid_device(g, device);
  if (!g.pairs) {
    g.build_topology();
    auto p = std::make_unique<SingularPairList>();
    build_singular_pairs(g, *p);
    p->d_test.upload(p->test_cell);
    p->d_trial.upload(p->trial_cell);
    p->d_config.upload(p->config);
    p->uploaded = true;
    g.pairs = std::move(p);
  }
  return *g.pairs;
}

void ensure_space_device(SpaceT& s, int device) {
  std::lock_guard<std::mutex> lock(s.mu);
  if (s.device == device && s.d_dofs.ptr) return;
  if (s.device != -1 && s.device != device)
    throw Error(kUnsupported, "a space is bound to the device it was first assembled on");
  if (s.ndofs > INT32_MAX) throw Error(kUnsupported, "too many DOFs for 32-bit indices");
  std::vector<int> dofs(s.cell_dofs.begin(), s.cell_dofs.end());
  s.d_dofs.upload(dofs);
  std::vector<int> off, tdofs;
  std::vector<uint8_t> ldof;
  s.tile_cells = scatter_tile_cells();
  std::vector<uint8_t> inc_off, inc_ent;
  build_tiles(s, s.tile_cells, off, tdofs, ldof, s.max_tile_dofs, inc_off, inc_ent);
  s.d_tile_inc_off.upload(inc_off);
  s.d_tile_inc_ent.upload(inc_ent);
  s.ntiles = static_cast<int>(off.size()) - 1;
  s.d_tile_off.upload(off);
  s.d_tile_dofs.upload(tdofs);
  s.d_cell_ldof.upload(ldof);
  s.device = device;
}

CellSet cell_set(const GridT& g, const GridGeometry& geo) {
  CellSet c;
  c.ncells = static_cast<int>(g.ncells);
  c.stride = cell_stride(c.ncells);
  c.geom = geo.geom.as<double>();
  c.qpts = geo.qpts.as<double>();
  c.qrel = geo.qrel.as<float4>();
  c.vids = geo.vids.as<int>();
  return c;
}

SpaceTiles space_tiles(const SpaceT& s) {
  SpaceTiles t;
  t.nbasis = s.nbasis;
  t.tile_cells = s.tile_cells;
  t.ntiles = s.ntiles;
  t.max_tile_dofs = s.max_tile_dofs;
  t.tile_dof_off = s.d_tile_off.as<int>();
  t.tile_dofs = s.d_tile_dofs.as<int>();
  t.cell_ldof = s.d_cell_ldof.as<uint8_t>();
  t.inc_off = s.d_tile_inc_off.as<uint8_t>();
  t.inc_ent = s.d_tile_inc_ent.as<uint8_t>();
  t.cell_dofs = s.d_dofs.as<int>();
  return t;
}

void check_spaces(const BoundaryAssemblerT& a, const SpaceT& trial, const SpaceT& test) {
  if (!trial.grid || !test.grid) throw Error(kInvalidArgument, "space without grid");
  if (trial.grid->quads() != test.grid->quads())
    throw Error(kUnsupported, "a triangle grid and a quadrilateral grid cannot be paired");
  (void)a;
}

QuadCells quad_cells(const GridT& g) {
  QuadCells q;
  q.ncells = static_cast<int>(g.ncells);
  q.points = g.d_points.as<double>();
  q.cells = g.d_cells.as<int>();
  q.vids = g.topo.empty() ? g.d_cells.as<int>() : g.d_topo.as<int>();
  return q;
}

// Device data of a quadrilateral grid, with its geometry at the rule's n x n points
// (computed on first use and cached in the grid, as grid_geometry does for triangles).
QuadCells quad_cells(GridT& g, int device, const QuadGaussRule& rule, cudaStream_t stream,
                     size_t& launches) {
  std::lock_guard<std::mutex> lock(g.mu);
  ensure_grid_device(g, device);
  QuadCells q = quad_cells(g);
  auto& slot = g.quad_geometry[rule.n];
  if (!slot) {
    auto buf = std::make_unique<DeviceBuffer>();
    buf->alloc(sizeof(double) * kQuadGeomFields * static_cast<size_t>(g.ncells) * rule.n * rule.n);
    BEMPP_CUDA(launch_quad_geometry(q, rule, buf->as<double>(), stream));
    ++launches;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    BEMPP_CUDA(cudaStreamIsCapturing(stream, &cap));
    if (cap == cudaStreamCaptureStatusNone) BEMPP_CUDA(cudaStreamSynchronize(stream));
    slot = std::move(buf);
  }
  q.qgeom = slot->as<double>();
  return q;
}

// Regular rule and Duffy order of quadrilateral pairs from the options.
void quad_rules(const Options& o, QuadGaussRule& rule, int& order) {
  const auto qit = o.regular.find(kQuadrilateral);
  if (qit == o.regular.end())
    throw Error(kInvalidArgument, "no regular quadrature degree for quadrilaterals");
  const auto sit = o.singular.find({kQuadrilateral, kQuadrilateral});
  if (sit == o.singular.end())
    throw Error(kInvalidArgument, "no singular quadrature degree for quadrilateral pairs");
  if (sit->second < 1 || sit->second > 16)
    throw Error(kUnsupported, "quadrilateral Duffy rules of order 1..16 only");
  rule = quad_gauss_rule(qit->second);
  order = static_cast<int>(sit->second);
}

struct Timer {
  BoundaryAssemblerT& a;
  cudaStream_t stream;
  int next = 0;
  bool on;
  Timer(BoundaryAssemblerT& asmb, cudaStream_t s, bool enable = true)
      : a(asmb), stream(s), on(asmb.timing && enable) {
    if (!on) return;
    for (auto& e : a.events)
      if (!e) BEMPP_CUDA(cudaEventCreate(&e));
    mark();
  }
  void mark() {
    if (on && next < 5) BEMPP_CUDA(cudaEventRecord(a.events[next++], stream));
  }
  // Durations are read lazily (boundary_assembler_phase_times) so that timing adds no
  // host synchronisation to the assembly itself.
  void finish() { a.events_recorded = on ? next : 0; }
};

// The side stream (and its fork / join events) of the assembler on `device`.
void ensure_side_stream(BoundaryAssemblerT& a, int device) {
  if (a.side && a.side_device == device) return;
  if (a.side) {
    cudaStreamDestroy(a.side);
    cudaEventDestroy(a.fork_ev);
    cudaEventDestroy(a.join_ev);
    a.side = nullptr;
  }
  BEMPP_CUDA(cudaStreamCreateWithFlags(&a.side, cudaStreamNonBlocking));
  BEMPP_CUDA(cudaEventCreateWithFlags(&a.fork_ev, cudaEventDisableTiming));
  BEMPP_CUDA(cudaEventCreateWithFlags(&a.join_ev, cudaEventDisableTiming));
  a.side_device = device;
}

}  // namespace

int effective_chunks(const SpaceT& trial, int want) {
  if (trial.grid->quads()) return 1;  // one launch per part
  const int tiles = static_cast<int>((trial.grid->ncells + 31) / 32);
  return std::max(1, std::min(want, tiles));
}

const ColumnRuns& chunk_columns(SpaceT& trial, int nchunks) {
  std::lock_guard<std::mutex> lock(trial.mu);
  auto& slot = trial.chunk_runs[nchunks];
  if (slot.empty()) {
    const int64_t nc = trial.grid->ncells;
    const int tiles = static_cast<int>((nc + 31) / 32);
    // chunk c holds trial tiles [c * tiles / nchunks, (c + 1) * tiles / nchunks)
    std::vector<int> last(static_cast<size_t>(trial.ndofs), -1);
    for (int64_t c = 0; c < nc; ++c) {
      const int tile = static_cast<int>(c / 32);
      const int chunk = static_cast<int>((static_cast<int64_t>(tile + 1) * nchunks - 1) / tiles);
      for (int b = 0; b < trial.nbasis; ++b) {
        int& l = last[trial.cell_dofs[c * trial.nbasis + b]];
        l = std::max(l, chunk);
      }
    }
    slot.assign(nchunks, {});
    for (int64_t d = 0; d < trial.ndofs;) {
      const int c = std::max(last[d], 0);  // a DOF on no cell: an all-zero column
      int64_t e = d + 1;
      while (e < trial.ndofs && std::max(last[e], 0) == c) ++e;
      slot[c].push_back({d, e - d});
      d = e;
    }
  }
  return slot;
}

namespace {

// Quadrilateral grids: the regular part (every pair that shares no vertex, Gauss tensor
// rule on both cells) and the singular part (the 49 Duffy configurations), FP64 whatever
// the precision option, added into the zeroed output in one chunk.
void assemble_quad_device(BoundaryAssemblerT& a, SpaceT& trial, SpaceT& test, void* d_out,
                          cudaStream_t stream, const std::function<void(int)>& chunk_done) {
  const int device = current_device();
  QuadGaussRule rule;
  int order;
  quad_rules(a.options, rule, order);
  const bool same_grid = trial.grid == test.grid;
  const int64_t nt = test.ndofs, ns = trial.ndofs;
  const bool single = a.dtype == 0 || a.dtype == 2;
  const bool cplx = a.kernel == kHelmholtz;
  a.launches = 0;
  ensure_space_device(test, device);
  ensure_space_device(trial, device);
  Timer timer(a, stream);
  const QuadCells tq = quad_cells(*test.grid, device, rule, stream, a.launches);
  const QuadCells sq = quad_cells(*trial.grid, device, rule, stream, a.launches);
  timer.mark();
  void* out = d_out;
  const size_t esize = cplx ? 16 : 8;
  if (single) {
    a.convert.alloc(static_cast<size_t>(nt) * ns * esize);
    out = a.convert.ptr;
  }
  const bool empty = nt == 0 || ns == 0;
  if (!empty) BEMPP_CUDA(cudaMemsetAsync(out, 0, static_cast<size_t>(nt) * ns * esize, stream));
  timer.mark();
  QuadPairArgs g{};
  g.kernel = a.kernel;
  g.op = a.op;
  g.k = a.k;
  g.nbt = test.nbasis;
  g.nbs = trial.nbasis;
  g.test = tq;
  g.trial = sq;
  g.test_dofs = test.d_dofs.as<int>();
  g.trial_dofs = trial.d_dofs.as<int>();
  g.rule = rule;
  g.same_grid = same_grid ? 1 : 0;
  // one space and a symmetric operator: half of the regular pairs, mirrored
  g.symmetric = (&trial == &test && same_grid && (a.op == kSL || a.op == kHS)) ? 1 : 0;
  g.out = out;
  g.ld = nt;
  if (!empty) {
    g.singular = false;
    BEMPP_CUDA(launch_quad_pairs(g, stream));
    ++a.launches;
  }
  timer.mark();
  if (!empty && same_grid) {
    SingularPairList& pl = grid_pairs(*test.grid, device);
    const DeviceRules& dr = device_rules(device, order, true);
    g.rules = SingularRules{dr.offset.as<int>(), dr.test_xi.as<double>(), dr.trial_xi.as<double>(),
                            dr.w.as<double>()};
    g.pairs = SingularPairs{static_cast<int>(pl.test_cell.size()), pl.d_test.as<int>(),
                            pl.d_trial.as<int>(), pl.d_config.as<int>()};
    g.singular = true;
    BEMPP_CUDA(launch_quad_pairs(g, stream));
    ++a.launches;
  }
  if (single && !empty) {
    BEMPP_CUDA(launch_convert_to_single(static_cast<const double*>(out), d_out,
                                        static_cast<size_t>(nt) * ns * (cplx ? 2 : 1), stream));
    ++a.launches;
  }
  if (chunk_done) chunk_done(0);
  timer.mark();
  timer.finish();
}

}  // namespace

void assemble_device(BoundaryAssemblerT& a, SpaceT& trial, SpaceT& test, void* d_out,
                     cudaStream_t stream, int nchunks, const std::function<void(int)>& chunk_done) {
  check_spaces(a, trial, test);
  if (trial.grid->quads()) {
    a.tx_ge_sy = false;  // one chunk
    assemble_quad_device(a, trial, test, d_out, stream, chunk_done);
    return;
  }
  const int device = current_device();
  const auto qit = a.options.regular.find(kTriangle);
  if (qit == a.options.regular.end())
    throw Error(kInvalidArgument, "no regular quadrature degree for triangles");
  const auto sit = a.options.singular.find({kTriangle, kTriangle});
  if (sit == a.options.singular.end())
    throw Error(kInvalidArgument, "no singular quadrature degree for triangle pairs");
  const RegularRule rule = simplex_rule(static_cast<int>(qit->second));
  const int order = static_cast<int>(sit->second);
  const bool same_grid = trial.grid == test.grid;
  const int64_t nt = test.ndofs, ns = trial.ndofs;
  const bool single = a.dtype == 0 || a.dtype == 2;
  const bool cplx = a.kernel == kHelmholtz;
  const bool dp0 = test.nbasis == 1 && trial.nbasis == 1 && a.op != kHS;
  nchunks = effective_chunks(trial, nchunks);
  if (single && !dp0) nchunks = 1;
  a.launches = 0;

  ensure_space_device(test, device);
  ensure_space_device(trial, device);
  Timer timer(a, stream, nchunks == 1);
  const GridGeometry& tgeo = grid_geometry(*test.grid, device, rule, stream, a.launches);
  const GridGeometry& sgeo = grid_geometry(*trial.grid, device, rule, stream, a.launches);
  timer.mark();

  void* out = d_out;
  const size_t esize = cplx ? 16 : 8;
  if (single) {
    a.convert.alloc(static_cast<size_t>(nt) * ns * esize);
    out = a.convert.ptr;
  }
  RegularArgs ra;
  ra.kernel = a.kernel;
  ra.op = a.op;
  ra.k = a.k;
  ra.same_grid = same_grid ? 1 : 0;
  // one space on both sides and a symmetric kernel: lower-triangle tile pairs, mirrored
  ra.symmetric = (&trial == &test && same_grid && (a.op == kSL || a.op == kHS)) ? 1 : 0;
  ra.precision = a.options.precision == 1 ? kRegularMixed : kRegularFP64;
  ra.out_type = cplx ? kOutC128 : kOutF64;
  ra.ld = nt;
  ra.out = out;
  // bound of |k (r - r0)| over every far pair (r0 the centroid distance); a margin of 1e-6
  // relative covers the device's own rounding of the radii
  const double phase_bound = std::fabs(a.k) *
                             (test.grid->max_circumradius() + trial.grid->max_circumradius()) *
                             (1.0 + 1e-6);
  ra.small_phase = phase_bound <= 0.8 ? 1 : 0;
  // one P1 / DP1 space, double layer or its adjoint, 6-point rule (Helmholtz: with the
  // phases referenced to the pair): the pair (i, j) and the pair (j, i) share their
  // kernel values, so both blocks of a tile pair come from one pass (one-launch assemblies
  // only: a chunked host-memory assembly keeps the full tile grid, whose columns finish
  // evenly through the chunks and go out by DMA meanwhile, where the tx >= sy half
  // finishes most columns only in its last chunks; measured on the 20,480-triangle
  // sphere, 16 chunks: 28.5 against 27.1 ms for the double layer)
  if (&trial == &test && same_grid && (a.kernel == kLaplace || ra.small_phase) &&
      (a.op == kDL || a.op == kADL) && test.nbasis == 3 && rule.npts == 6 && nchunks == 1)
    ra.symmetric = 2;
  a.tx_ge_sy = ra.symmetric != 0;
  if (ra.precision == kRegularMixed && nt > 0 && ns > 0) {
    const NearField& nf = near_field(*test.grid, *trial.grid);
    ra.near.tile_mask = nf.tile_mask.as<int>();
    ra.near.masks = nf.masks.as<unsigned>();
    ra.near.pairs = nf.pairs.as<int2>();
    ra.near.npairs = nf.npairs;
    ra.near.trial_tiles = nf.trial_tiles;
    ra.near.test_dofs = test.d_dofs.as<int>();
    ra.near.trial_dofs = trial.d_dofs.as<int>();
  }
  const CellSet tcs = cell_set(*test.grid, tgeo), scs = cell_set(*trial.grid, sgeo);
  // mixed: the FP32 far-pair launch and the FP64 near-pair launch
  const size_t regular_launches = ra.near.npairs > 0 ? 2 : 1;

  const bool empty = nt == 0 || ns == 0;
  const bool singular = same_grid && !empty;
  SingularArgs sa;
  SingularRules rules{};
  SingularPairs pairs{};
  // the pair list and the Duffy rules are built at the first singular launch, so that on
  // a fresh grid the host builds them while the first regular kernel runs
  bool pairs_ready = false;
  auto ensure_pairs = [&] {
    if (pairs_ready) return;
    SingularPairList& pl = grid_pairs(*test.grid, device);
    const DeviceRules& dr = device_rules(device, order);
    rules = SingularRules{dr.offset.as<int>(), dr.test_xi.as<double>(), dr.trial_xi.as<double>(),
                          dr.w.as<double>()};
    pairs = SingularPairs{static_cast<int>(pl.test_cell.size()), pl.d_test.as<int>(),
                          pl.d_trial.as<int>(), pl.d_config.as<int>()};
    pairs_ready = true;
  };
  if (singular) {
    sa.kernel = a.kernel;
    sa.op = a.op;
    sa.k = a.k;
    sa.out_type = ra.out_type;
    sa.ld = nt;
    sa.out = out;
    sa.unique_entries = dp0 ? 1 : 0;
    sa.pair_values = nullptr;
  }
  auto run_singular = [&](int lo, int hi, cudaStream_t s) {
    ensure_pairs();
    sa.trial_lo = lo;
    sa.trial_hi = hi;
    BEMPP_CUDA(launch_singular(tcs, test.d_dofs.as<int>(), test.nbasis, scs,
                               trial.d_dofs.as<int>(), trial.nbasis, rules, pairs, sa, s));
    ++a.launches;
  };
  const int tiles = static_cast<int>((trial.grid->ncells + 31) / 32);
  auto tile_range = [&](int c, int& t0, int& t1) {
    t0 = static_cast<int>(static_cast<int64_t>(c) * tiles / nchunks);
    t1 = static_cast<int>(static_cast<int64_t>(c + 1) * tiles / nchunks);
  };

  if (dp0) {
    // the direct kernels write every entry once, so each chunk is its regular launches
    // followed by the singular pairs of its trial cells.  Mixed precision: the regular
    // kernels leave the vertex-sharing entries alone, and the singular kernel of a
    // one-chunk assembly runs on a side stream beside them (fork / join events).
    timer.mark();  // no memset phase
    const bool fork = singular && nchunks == 1 && ra.precision == kRegularMixed;
    if (fork) {
      ensure_side_stream(a, device);
      BEMPP_CUDA(cudaEventRecord(a.fork_ev, stream));
      BEMPP_CUDA(cudaStreamWaitEvent(a.side, a.fork_ev, 0));
      run_singular(0, 0x7fffffff, a.side);
      BEMPP_CUDA(cudaEventRecord(a.join_ev, a.side));
    }
    for (int c = 0; c < nchunks; ++c) {
      int t0, t1;
      tile_range(c, t0, t1);
      if (!empty) {
        ra.trial_tile0 = t0;
        ra.trial_tiles = t1 - t0;
        BEMPP_CUDA(launch_regular_dp0(tcs, scs, rule, ra, stream));
        a.launches += regular_launches;
        if (nchunks == 1) timer.mark();
        if (fork)
          BEMPP_CUDA(cudaStreamWaitEvent(stream, a.join_ev, 0));
        else if (singular)
          run_singular(nchunks == 1 ? 0 : 32 * t0, nchunks == 1 ? 0x7fffffff : 32 * t1, stream);
        if (single) {
          const std::vector<std::pair<int64_t, int64_t>> all{{0, ns}};
          for (const auto& run : nchunks == 1 ? all : chunk_columns(trial, nchunks)[c]) {
            const size_t off = static_cast<size_t>(run.first) * nt * (cplx ? 2 : 1);
            BEMPP_CUDA(launch_convert_to_single(static_cast<const double*>(out) + off,
                                                static_cast<char*>(d_out) + off * 4,
                                                static_cast<size_t>(run.second) * nt * (cplx ? 2 : 1),
                                                stream));
            ++a.launches;
          }
        }
      } else if (nchunks == 1) {
        timer.mark();
      }
      if (chunk_done) chunk_done(c);
    }
  } else {
    if (!empty) BEMPP_CUDA(cudaMemsetAsync(out, 0, static_cast<size_t>(nt) * ns * esize, stream));
    timer.mark();
    // Chunked: the full tile grid (columns finish evenly through the chunks) runs the
    // whole singular part on a side stream; its launch is enqueued after the first two
    // chunks' regular launches, so that on a fresh grid the host builds the pair list while
    // they run, and the completion of those chunks is reported after it.  The tx >= sy
    // launches (which finish most columns late) add each chunk's singular pairs after its
    // regular pairs instead, so that its first columns go out as early as they can.
    const bool side_singular = singular && nchunks > 1 && !ra.symmetric;
    const int fork_after = side_singular ? std::min(1, nchunks - 1) : -1;
    if (side_singular) {
      ensure_side_stream(a, device);
      BEMPP_CUDA(cudaEventRecord(a.fork_ev, stream));
      BEMPP_CUDA(cudaStreamWaitEvent(a.side, a.fork_ev, 0));
    }
    int done = 0;  // chunks whose completion has been reported
    for (int c = 0; c < nchunks; ++c) {
      int t0, t1;
      tile_range(c, t0, t1);
      if (!empty) {
        ra.trial_tile0 = t0;
        ra.trial_tiles = t1 - t0;
        BEMPP_CUDA(launch_regular_scatter(tcs, space_tiles(test), scs, space_tiles(trial), rule,
                                          ra, stream));
        a.launches += regular_launches;
        if (singular && nchunks > 1 && !side_singular)
          run_singular(32 * t0, c + 1 == nchunks ? 0x7fffffff : 32 * t1, stream);
      }
      if (c == fork_after) {
        run_singular(0, 0x7fffffff, a.side);
        BEMPP_CUDA(cudaEventRecord(a.join_ev, a.side));
        BEMPP_CUDA(cudaStreamWaitEvent(stream, a.join_ev, 0));
      }
      if (nchunks == 1) {
        timer.mark();
        if (singular) run_singular(0, 0x7fffffff, stream);
        if (single && !empty) {
          BEMPP_CUDA(launch_convert_to_single(static_cast<const double*>(out), d_out,
                                              static_cast<size_t>(nt) * ns * (cplx ? 2 : 1), stream));
          ++a.launches;
        }
      }
      if (c >= fork_after)
        for (; done <= c; ++done)
          if (chunk_done) chunk_done(done);
    }
  }
  timer.mark();
  timer.finish();
}

const GridGeometry& sweep_geometry(GridT& g, int device, const RegularRule& rule) {
  size_t launches = 0;
  return grid_geometry(g, device, rule, nullptr, launches);
}

namespace {
void check_potential(const BoundaryAssemblerT& a, const SpaceT& space, int64_t npoints) {
  if (a.op != kSL && a.op != kDL)
    throw Error(kUnsupported, "potential operators: single and double layer only");
  if (npoints < 0 || npoints > 0x7fffffff) throw Error(kInvalidArgument, "point count");
  if (space.grid->quads())
    throw Error(kUnsupported, "potential operators on quadrilateral grids are not supported");
  if (space.nbasis != 1 && space.nbasis != 3 && space.nbasis != 6)
    throw Error(kUnsupported, "potential operators: Lagrange spaces of degree 0, 1 or 2");
}
}  // namespace

void assemble_potential_device(BoundaryAssemblerT& a, SpaceT& space, const double* d_points,
                               int64_t npoints, void* d_out, cudaStream_t stream) {
  check_potential(a, space, npoints);
  const int device = current_device();
  const auto qit = a.options.regular.find(kTriangle);
  if (qit == a.options.regular.end())
    throw Error(kInvalidArgument, "no regular quadrature degree for triangles");
  const RegularRule rule = simplex_rule(static_cast<int>(qit->second));
  a.launches = 0;
  ensure_space_device(space, device);
  const GridGeometry& geo = grid_geometry(*space.grid, device, rule, stream, a.launches);
  const bool single = a.dtype == 0 || a.dtype == 2;
  const bool cplx = a.kernel == kHelmholtz;
  const size_t reals = static_cast<size_t>(npoints) * space.ndofs * (cplx ? 2 : 1);
  if (reals == 0) return;
  void* out = d_out;
  if (single) {
    a.convert.alloc(sizeof(double) * reals);
    out = a.convert.ptr;
  }
  if (space.nbasis > 1) {  // P1 / P2 DOF columns are sums over the cells of the DOF
    BEMPP_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * reals, stream));
    ++a.launches;
  }
  BEMPP_CUDA(launch_potential(a.kernel, a.op, d_points, static_cast<int>(npoints),
                              cell_set(*space.grid, geo), space.d_dofs.as<int>(), space.nbasis,
                              rule, a.k, static_cast<double*>(out), npoints, stream));
  ++a.launches;
  if (single) {
    BEMPP_CUDA(launch_convert_to_single(static_cast<const double*>(out), d_out, reals, stream));
    ++a.launches;
  }
}

void assemble_potential_host(BoundaryAssemblerT& a, SpaceT& space, const double* points,
                             int64_t npoints, void* data) {
  check_potential(a, space, npoints);
  const bool cplx = a.kernel == kHelmholtz;
  const size_t esize = (a.dtype == 0 || a.dtype == 2) ? (cplx ? 8 : 4) : (cplx ? 16 : 8);
  const size_t bytes = static_cast<size_t>(npoints) * space.ndofs * esize;
  if (bytes == 0) return;
  if (!a.stream) BEMPP_CUDA(cudaStreamCreateWithFlags(&a.stream, cudaStreamNonBlocking));
  DeviceBuffer d_points, d_out;
  d_points.alloc(sizeof(double) * 3 * static_cast<size_t>(npoints));
  d_out.alloc(bytes);
  BEMPP_CUDA(cudaMemcpyAsync(d_points.ptr, points, sizeof(double) * 3 * npoints,
                             cudaMemcpyHostToDevice, a.stream));
  assemble_potential_device(a, space, d_points.as<double>(), npoints, d_out.ptr, a.stream);
  BEMPP_CUDA(cudaMemcpyAsync(data, d_out.ptr, bytes, cudaMemcpyDeviceToHost, a.stream));
  BEMPP_CUDA(cudaStreamSynchronize(a.stream));
}

SingularPairList& sweep_pairs(GridT& g, int device) { return grid_pairs(g, device); }

SingularRules sweep_rules(int device, int order) {
  const DeviceRules& dr = device_rules(device, order);
  return SingularRules{dr.offset.as<int>(), dr.test_xi.as<double>(), dr.trial_xi.as<double>(),
                       dr.w.as<double>()};
}

void helmholtz_sl_gradient_device(GridT& g, const Options& opts, double k, const double* d_lam,
                                  const double* d_mu, double* d_totals, double* d_grad_points,
                                  cudaStream_t stream) {
  if (g.quads()) throw Error(kUnsupported, "the adjoint gradient needs a triangle grid");
  const int device = current_device();
  const auto qit = opts.regular.find(kTriangle);
  const auto sit = opts.singular.find({kTriangle, kTriangle});
  if (qit == opts.regular.end() || sit == opts.singular.end())
    throw Error(kInvalidArgument, "options lack triangle quadrature degrees");
  const RegularRule rule = simplex_rule(static_cast<int>(qit->second));
  size_t launches = 0;
  const GridGeometry& geo = grid_geometry(g, device, rule, stream, launches);
  SingularPairList& pl = grid_pairs(g, device);
  const DeviceRules& dr = device_rules(device, static_cast<int>(sit->second));
  SingularRules rules{dr.offset.as<int>(), dr.test_xi.as<double>(), dr.trial_xi.as<double>(),
                      dr.w.as<double>()};
  SingularPairs pairs{static_cast<int>(pl.test_cell.size()), pl.d_test.as<int>(),
                      pl.d_trial.as<int>(), pl.d_config.as<int>()};
  {
    std::lock_guard<std::mutex> lock(g.mu);
    g.adjoint_scratch.alloc(sizeof(double) * 9 * static_cast<size_t>(std::max<int64_t>(1, g.ncells)));
  }
  BEMPP_CUDA(launch_adjoint_sl(cell_set(g, geo), rule, rules, pairs, k, d_lam, d_mu,
                               g.adjoint_scratch.as<double>(), d_grad_points,
                               static_cast<int>(g.npoints), d_totals, opts.precision == 1,
                               stream));
}

MatrixT* assemble_singular_csr(BoundaryAssemblerT& a, SpaceT& trial, SpaceT& test) {
  check_spaces(a, trial, test);
  const int device = current_device();
  const bool cplx = a.kernel == kHelmholtz;
  const bool single = a.dtype == 0 || a.dtype == 2;
  const size_t es = dtype_size(a.dtype);
  auto* m = new MatrixT();
  m->csr = true;
  m->dtype = a.dtype;
  m->rows = test.ndofs;
  m->cols = trial.ndofs;
  std::vector<int64_t> rows, cols;
  std::vector<double> vals;  // FP64 (interleaved complex)
  const int nvals = test.nbasis * trial.nbasis * (cplx ? 2 : 1);
  int np = 0;
  const SingularPairList* pl_used = nullptr;
  if (trial.grid == test.grid && test.ndofs > 0 && trial.ndofs > 0 && test.grid->quads()) {
    QuadGaussRule qrule;
    int order;
    quad_rules(a.options, qrule, order);
    ensure_space_device(test, device);
    ensure_space_device(trial, device);
    SingularPairList& pl = grid_pairs(*test.grid, device);
    const DeviceRules& dr = device_rules(device, order, true);
    np = static_cast<int>(pl.test_cell.size());
    a.pair_values.alloc(sizeof(double) * std::max(1, np * nvals));
    QuadPairArgs g{};
    g.kernel = a.kernel;
    g.op = a.op;
    g.k = a.k;
    g.nbt = test.nbasis;
    g.nbs = trial.nbasis;
    g.test = g.trial = quad_cells(*test.grid);
    g.test_dofs = test.d_dofs.as<int>();
    g.trial_dofs = trial.d_dofs.as<int>();
    g.rule = qrule;
    g.rules = SingularRules{dr.offset.as<int>(), dr.test_xi.as<double>(), dr.trial_xi.as<double>(),
                            dr.w.as<double>()};
    g.pairs = SingularPairs{np, pl.d_test.as<int>(), pl.d_trial.as<int>(), pl.d_config.as<int>()};
    g.singular = true;
    g.same_grid = 1;
    g.out = nullptr;
    g.pair_values = a.pair_values.as<double>();
    BEMPP_CUDA(launch_quad_pairs(g, nullptr));
    pl_used = &pl;
  } else if (trial.grid == test.grid && test.ndofs > 0 && trial.ndofs > 0) {
    const auto sit = a.options.singular.find({kTriangle, kTriangle});
    if (sit == a.options.singular.end())
      throw Error(kInvalidArgument, "no singular quadrature degree for triangle pairs");
    const auto qit = a.options.regular.find(kTriangle);
    const RegularRule rule = simplex_rule(qit == a.options.regular.end() ? 6 : static_cast<int>(qit->second));
    ensure_space_device(test, device);
    ensure_space_device(trial, device);
    size_t launches = 0;
    const GridGeometry& geo = grid_geometry(*test.grid, device, rule, nullptr, launches);
    SingularPairList& pl = grid_pairs(*test.grid, device);
    const DeviceRules& dr = device_rules(device, static_cast<int>(sit->second));
    np = static_cast<int>(pl.test_cell.size());
    a.pair_values.alloc(sizeof(double) * std::max(1, np * nvals));
    SingularRules rules{dr.offset.as<int>(), dr.test_xi.as<double>(), dr.trial_xi.as<double>(),
                        dr.w.as<double>()};
    SingularPairs pairs{np, pl.d_test.as<int>(), pl.d_trial.as<int>(), pl.d_config.as<int>()};
    SingularArgs sa{a.kernel, a.op, a.k, cplx ? kOutC128 : kOutF64, 0, nullptr, 0,
                    a.pair_values.as<double>()};
    const CellSet cs = cell_set(*test.grid, geo);
    BEMPP_CUDA(launch_singular(cs, test.d_dofs.as<int>(), test.nbasis, cs, trial.d_dofs.as<int>(),
                               trial.nbasis, rules, pairs, sa, nullptr));
    pl_used = &pl;
  }
  if (pl_used) {
    const SingularPairList& pl = *pl_used;
    std::vector<double> pv(static_cast<size_t>(np) * nvals);
    BEMPP_CUDA(cudaMemcpy(pv.data(), a.pair_values.ptr, pv.size() * sizeof(double),
                          cudaMemcpyDeviceToHost));
    // COO triplets in the reference's order: per pair, trial basis outer, test inner
    // (src/boundary_assemblers.rs:675-681)
    for (int p = 0; p < np; ++p)
      for (int b = 0; b < trial.nbasis; ++b)
        for (int aa = 0; aa < test.nbasis; ++aa) {
          const int e = aa + test.nbasis * b;
          rows.push_back(test.cell_dofs[static_cast<int64_t>(pl.test_cell[p]) * test.nbasis + aa]);
          cols.push_back(trial.cell_dofs[static_cast<int64_t>(pl.trial_cell[p]) * trial.nbasis + b]);
          if (cplx) {
            vals.push_back(pv[static_cast<size_t>(p) * nvals + 2 * e]);
            vals.push_back(pv[static_cast<size_t>(p) * nvals + 2 * e + 1]);
          } else {
            vals.push_back(pv[static_cast<size_t>(p) * nvals + e]);
          }
        }
  }
  // src/boundary_assemblers.rs:130-145: an all-(near-)zero singular part is an empty CSR
  const double tiny = 1e-10;
  bool any = false;
  const size_t nnz_in = rows.size();
  for (size_t i = 0; i < nnz_in && !any; ++i) {
    double mag = cplx ? std::hypot(vals[2 * i], vals[2 * i + 1]) : std::fabs(vals[i]);
    any = mag > tiny;
  }
  m->indptr.assign(m->rows + 1, 0);
  if (!any) return m;
  // from_aij: sort by (row, col), sum duplicates
  std::vector<size_t> order(nnz_in);
  for (size_t i = 0; i < nnz_in; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
    return rows[x] != rows[y] ? rows[x] < rows[y] : cols[x] < cols[y];
  });
  std::vector<double> merged;
  std::vector<int64_t> mrow;
  for (size_t k = 0; k < nnz_in; ++k) {
    const size_t i = order[k];
    if (!m->indices.empty() && mrow.back() == rows[i] &&
        static_cast<int64_t>(m->indices.back()) == cols[i]) {
      if (cplx) {
        merged[merged.size() - 2] += vals[2 * i];
        merged[merged.size() - 1] += vals[2 * i + 1];
      } else {
        merged.back() += vals[i];
      }
      continue;
    }
    mrow.push_back(rows[i]);
    m->indices.push_back(static_cast<uintptr_t>(cols[i]));
    if (cplx) {
      merged.push_back(vals[2 * i]);
      merged.push_back(vals[2 * i + 1]);
    } else {
      merged.push_back(vals[i]);
    }
  }
  for (int64_t r : mrow) m->indptr[r + 1]++;
  for (size_t r = 0; r < m->rows; ++r) m->indptr[r + 1] += m->indptr[r];
  const size_t nnz = m->indices.size();
  m->data.resize(nnz * es);
  if (single) {
    float* d = reinterpret_cast<float*>(m->data.data());
    for (size_t i = 0; i < merged.size(); ++i) d[i] = static_cast<float>(merged[i]);
  } else {
    std::memcpy(m->data.data(), merged.data(), merged.size() * sizeof(double));
  }
  return m;
}

}  // namespace bempp_b200

BoundaryAssemblerT::~BoundaryAssemblerT() {
  for (auto& e : events)
    if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  for (auto e : chunk_ev) cudaEventDestroy(e);
  for (auto e : copy_timing)
    if (e) cudaEventDestroy(e);
  if (side) {
    cudaStreamDestroy(side);
    cudaEventDestroy(fork_ev);
    cudaEventDestroy(join_ev);
  }
}
