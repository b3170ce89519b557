// Internal host-side objects behind the opaque C-ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../kernels/launch.h"

namespace bempp_b200 {

// Status codes (BemppStatus in include/bempp_b200.h).
enum Status : int32_t {
  kOk = 0,
  kInvalidArgument = 1,
  kUnsupported = 2,
  kOutOfMemory = 3,
  kCudaError = 4,
  kNoDevice = 5,
  kInternal = 6,
  kIncomplete = 7
};

struct Error : std::runtime_error {
  Status status;
  Error(Status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string& msg);
void clear_last_error();

#define BEMPP_CUDA(call)                                                               \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      throw ::bempp_b200::Error(e_ == cudaErrorMemoryAllocation ? kOutOfMemory           \
                                                                : kCudaError,            \
                                std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)

// Process-wide cache of device blocks behind every DeviceBuffer (device_cache.cpp): a
// freed block is kept for the next request of a similar size on its device, so that
// building and freeing grids and spaces again and again makes no cudaMalloc / cudaFree
// calls (driver calls that can stall behind other processes' allocations).  Returning a
// block waits for the device to finish its work, as cudaFree does.
cudaError_t device_cache_alloc(void** ptr, size_t bytes);
void device_cache_free(void* ptr);
size_t device_cache_trim();  // releases every cached free block; returns the bytes

// Owning device buffer.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { reset(); }
  void reset() {
    if (ptr) device_cache_free(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  void alloc(size_t n) {
    if (n <= bytes && ptr) return;
    reset();
    if (n == 0) return;
    BEMPP_CUDA(device_cache_alloc(&ptr, n));
    bytes = n;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
  // A copy from pageable host memory may return once the data is staged, before the DMA
  // into the buffer has finished, and the legacy default stream it runs on does not order
  // the library's non-blocking streams: wait for it, so that no kernel reads the buffer
  // (possibly a recycled cache block holding older data) before the copy has landed.
  template <typename T>
  void upload(const std::vector<T>& v) {
    alloc(v.size() * sizeof(T));
    if (v.empty()) return;
    BEMPP_CUDA(cudaMemcpy(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    BEMPP_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
  }
};

// ------------------------------------------------------------------------ options ---
enum CellType : uint8_t { kPoint = 0, kInterval = 1, kTriangle = 2, kQuadrilateral = 3 };

struct Options {
  // src/boundary_assemblers.rs:43-57 defaults
  std::map<uint8_t, size_t> regular{{kTriangle, 37}, {kQuadrilateral, 37}};
  std::map<std::pair<uint8_t, uint8_t>, size_t> singular{{{kTriangle, kTriangle}, 4},
                                                         {{kQuadrilateral, kQuadrilateral}, 4},
                                                         {{kQuadrilateral, kTriangle}, 4},
                                                         {{kTriangle, kQuadrilateral}, 4}};
  size_t batch_size = 128;
  uint8_t precision = 0;  // Precision_FP64
};

// --------------------------------------------------------------------------- rules ---
void gauss_legendre_01(int n, std::vector<double>& x, std::vector<double>& w);
// Symmetric triangle rule by number of points; throws if no rule has that count.
RegularRule simplex_rule(int npoints);
bool has_simplex_rule(int npoints);
// The 28 (test_local, trial_local) vertex pairings of the reference
// (src/boundary_assemblers.rs:267-288) and their Duffy rules of 1-D order n.
const std::vector<std::vector<std::pair<int, int>>>& singular_configurations();
struct DuffyRule {
  std::vector<double> test_xi, trial_xi, w;
};
DuffyRule duffy_rule(int config, int order);
// Quadrilaterals: the n x n Gauss tensor rule for a request of `npoints` (n the smallest
// with n^2 >= npoints), the 49 vertex pairings of two quadrilaterals that share a vertex
// (16 vertex, 32 edge, 1 identical) and their Duffy rules of 1-D order n.
int quad_gauss_order(size_t npoints);
QuadGaussRule quad_gauss_rule(size_t npoints);
const std::vector<std::vector<std::pair<int, int>>>& quad_singular_configurations();
DuffyRule quad_duffy_rule(int config, int order);

// --------------------------------------------------------------------- grid/space ---
struct GridGeometry {  // device geometry for one regular rule
  int npts = 0;
  DeviceBuffer geom, qpts, qrel, vids;
};

// Near field of a (test grid, trial grid) pair for the mixed-precision kernels (near.cpp):
// the device arrays behind NearArgs.
struct NearField {
  int test_tiles = 0, trial_tiles = 0, npairs = 0;
  DeviceBuffer tile_mask, masks, pairs;
  size_t marked = 0;  // marked pairs (near or vertex-sharing)
};

// Per chunk of a chunked assembly: runs (first column, number of columns).
using ColumnRuns = std::vector<std::vector<std::pair<int64_t, int64_t>>>;

struct SingularPairList {
  std::vector<int> test_cell, trial_cell, config;
  DeviceBuffer d_test, d_trial, d_config;
  bool uploaded = false;
};

// Rows of varying length in two flat arrays: row r is items[off[r] .. off[r + 1]).
template <typename T>
struct Rows {
  std::vector<int64_t> off{0};
  std::vector<T> items;
  struct View {
    const T* b;
    const T* e;
    const T* begin() const { return b; }
    const T* end() const { return e; }
    size_t size() const { return static_cast<size_t>(e - b); }
  };
  size_t size() const { return off.size() - 1; }
  View operator[](size_t r) const { return {items.data() + off[r], items.data() + off[r + 1]}; }
  bool empty() const { return off.size() == 1; }
};

}  // namespace bempp_b200

// Handle types of the C-ABI (declared opaque in include/bempp_b200.h).
using bempp_b200::DeviceBuffer;

struct GridT {
  uint64_t uid = 0;            // unique per grid object (plans keyed by it)
  std::vector<double> points;  // npoints x 3
  // ncells x nv (nv = 3 for triangles, 4 for quadrilaterals; cell vertices as point
  // indices: geometry)
  std::vector<int> cells;
  int64_t npoints = 0, ncells = 0;
  uint8_t cell_type = bempp_b200::kTriangle;  // kTriangle or kQuadrilateral
  int nv() const { return cell_type == bempp_b200::kQuadrilateral ? 4 : 3; }
  bool quads() const { return cell_type == bempp_b200::kQuadrilateral; }
  // Topology vertex of each cell corner (ncells x nv), when the grid came with ndgrid's
  // cell -> vertex connectivity; empty: the point indices of `cells` are the vertices.
  // Adjacency (singular pairs, near-field vertex tests) and vertex DOFs use these ids.
  std::vector<int> topo;
  int64_t nvertices = 0;
  // ndgrid's cell -> edge connectivity (local edge i opposite local vertex i) and edge ->
  // vertex connectivity, when given; build_edges then keeps ndgrid's edge numbering
  // (triangles; quadrilateral grids keep no edges, their spaces have no edge DOFs).
  std::vector<int> given_cell_edges;    // ncells x 3
  std::vector<int> given_edge_vertices; // nedges x 2
  const int* vtx() const { return topo.empty() ? cells.data() : topo.data(); }
  int64_t nverts() const { return topo.empty() ? npoints : nvertices; }
  uint8_t dtype = 1;
  bempp_b200::Rows<int> vertex_cells;  // upward connectivity, increasing cell index
  std::vector<std::pair<int, int>> edges;      // unique edges (v0 < v1)
  std::vector<std::array<int, 3>> cell_edges;  // local edge i opposite local vertex i
  int device = -1;
  DeviceBuffer d_points, d_cells, d_topo;
  std::map<int, std::unique_ptr<bempp_b200::GridGeometry>> geometry;  // keyed by regular npts
  // quadrilateral grids: geometry at the n x n regular points, keyed by n
  std::map<int, std::unique_ptr<DeviceBuffer>> quad_geometry;
  std::unique_ptr<bempp_b200::SingularPairList> pairs;
  DeviceBuffer adjoint_scratch;  // per-cell vertex gradients of the adjoint kernel
  double max_rad = -1.0;         // largest centroid-to-vertex distance (computed on demand)
  // near fields with other grids (and itself), keyed by the trial grid's uid
  std::map<uint64_t, std::unique_ptr<bempp_b200::NearField>> near_fields;
  std::mutex mu;
  void build_topology();  // vertex_cells
  void build_edges();     // edges and cell_edges (triangles)
  double max_circumradius();
};

struct ElementFamilyT {
  size_t degree;
  uint8_t continuity;  // 0 standard, 1 discontinuous
  uint8_t dtype;
};

struct SpaceT {
  GridT* grid = nullptr;
  size_t degree = 0;
  bool continuous = false;
  uint8_t dtype = 1;
  int nbasis = 1;
  int64_t ndofs = 0;
  std::vector<int64_t> cell_dofs;                  // ncells x nbasis
  bempp_b200::Rows<int64_t> entity_dofs[3];  // [dim][entity] -> dofs
  // device mirrors
  int device = -1;
  DeviceBuffer d_dofs;                                   // int32 ncells x nbasis
  DeviceBuffer d_tile_off, d_tile_dofs, d_cell_ldof;     // tile-scatter layout
  DeviceBuffer d_tile_inc_off, d_tile_inc_ent;           // and its DOF incidence
  int ntiles = 0, max_tile_dofs = 0, tile_cells = 0;
  std::map<int, bempp_b200::ColumnRuns> chunk_runs;  // by number of chunks
  std::mutex mu;
};

// ----------------------------------------------------------------------- matrices ---
struct MatrixT {
  bool csr = false;
  uint8_t dtype = 1;
  size_t rows = 0, cols = 0;
  std::vector<unsigned char> data;
  std::vector<uintptr_t> indices, indptr;
};

// --------------------------------------------------------------------- assemblers ---
struct BoundaryAssemblerT {
  int kernel = bempp_b200::kLaplace;
  int op = bempp_b200::kSL;
  double k = 0.0;
  uint8_t dtype = 1;
  bempp_b200::Options options;
  bool timing = false;
  std::vector<double> phase_ms;
  size_t launches = 0;
  cudaEvent_t events[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int events_recorded = 0;
  DeviceBuffer work;     // device output for host-memory assembly
  cudaStream_t stream = nullptr;  // host-memory assembly stream (created on first use)
  cudaStream_t copy_stream = nullptr;     // page-locked destinations: direct DMA stream
  std::vector<cudaEvent_t> chunk_ev;      // and its per-chunk events
  // side stream and fork / join events: the singular kernel of a one-chunk mixed-precision
  // DP0 assembly, and of a chunked non-DP0 one, runs beside the regular kernels (created on
  // first use, on side_device)
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  int side_device = -1;
  // last host-memory assembly: ms waiting for DMA, ms of host copy, copy groups, chunks,
  // host copy threads, ms of destination page prefaulting, device ms to the end of the
  // last chunk's kernels and to the end of the last DMA (page-locked destinations)
  std::array<double, 8> host_copy_stats{};
  // the last assembly's regular launches covered the tile pairs tx >= sy only (a chunk's
  // work then falls with its index)
  bool tx_ge_sy = false;
  cudaEvent_t copy_timing[3] = {nullptr, nullptr, nullptr};  // start, compute end, DMA end
  DeviceBuffer convert;  // FP64 staging for F32 / C32 outputs
  DeviceBuffer pair_values;
  std::mutex mu;
  ~BoundaryAssemblerT();
};


namespace bempp_b200 {

SpaceT* make_space(GridT* grid, const ElementFamilyT& fam);
// greedy colouring as src/function.rs:281-351 (exposed for tests of the host logic)
std::vector<std::vector<int64_t>> cell_colouring(const SpaceT& s);

size_t dtype_size(uint8_t dtype);

// Dense assembly into device memory (column-major, assembler dtype) on `stream`.
//
// With nchunks > 1 the regular part is launched over nchunks consecutive ranges of trial
// tiles and chunk_done(c) is called (host side, after chunk c's launches are enqueued);
// the trial DOFs whose columns are final after chunk c are chunk_columns(trial, nchunks)[c].
// F32 / C32 outputs of non-DP0 spaces are assembled in one chunk.
void assemble_device(BoundaryAssemblerT& a, SpaceT& trial, SpaceT& test, void* d_out,
                     cudaStream_t stream, int nchunks = 1,
                     const std::function<void(int)>& chunk_done = {});
// Maximal runs [first, first + count) of trial DOFs completed by each chunk of a chunked
// assembly: a column is complete after the last chunk holding one of its cells.
const ColumnRuns& chunk_columns(SpaceT& trial, int nchunks);
// Number of chunks assemble_device uses for a request of `want` (at most one per tile).
int effective_chunks(const SpaceT& trial, int want);
// Near field of (test, trial) on the current device, built on first use and cached in
// the test grid.
const NearField& near_field(GridT& test, GridT& trial);
// Dense assembly into host memory: chunked device assembly with the device-to-host copy
// of finished columns (pinned staging ring, parallel host copy) overlapped (host_copy.cpp).
void assemble_host(BoundaryAssemblerT& a, SpaceT& trial, SpaceT& test, void* data);
// Adjoint gradient of Re(lambda^H A mu), Helmholtz single layer, DP0 x DP0 on one grid;
// device inputs (complex128 lambda, mu per cell) and outputs ({J, dJ/dk}, npoints x 3).
void helmholtz_sl_gradient_device(GridT& g, const Options& opts, double k, const double* d_lam,
                                  const double* d_mu, double* d_totals, double* d_grad_points,
                                  cudaStream_t stream);
// Batched Helmholtz single-layer DP0 sweep (sweep.cpp): outs[i] holds nk complex64
// column-major ncells_i^2 matrices, wavenumber-major.
void helmholtz_sl_sweep_device(GridT* const* grids, size_t ngrids, const double* ks, size_t nk,
                               const Options& opts, void* const* outs, cudaStream_t stream);
// Launch parameters the sweep's autotuner chose (sweep.cpp).
struct SweepTuning {
  int kchunk = 8;         // wavenumbers per work item
  int blocks_per_sm = 4;  // CTAs per SM of the persistent grid
  int tile_shape = 1;     // a work item covers tile_shape x tile_shape 32-cell tile pairs
  double probe_ms = 0.0;  // probe milliseconds per (tile pair, wavenumber)
};
SweepTuning last_sweep_tuning();
// Fixes the sweep's launch parameters (kchunk <= 0: autotune again).
void set_sweep_tuning(int kchunk, int blocks_per_sm, int tile_shape);
// Singular part as CSR (host).
MatrixT* assemble_singular_csr(BoundaryAssemblerT& a, SpaceT& trial, SpaceT& test);
// Off-surface potential operator (single or double layer of the assembler's kernel) of
// `space` at npoints device points (npoints x 3, row-major): column-major npoints x ndofs
// device output in the assembler's dtype (potential.cu).
void assemble_potential_device(BoundaryAssemblerT& a, SpaceT& space, const double* d_points,
                               int64_t npoints, void* d_out, cudaStream_t stream);
// The same from host points into host memory.
void assemble_potential_host(BoundaryAssemblerT& a, SpaceT& space, const double* points,
                             int64_t npoints, void* data);

}  // namespace bempp_b200
