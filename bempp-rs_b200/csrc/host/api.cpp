// extern "C" entry points declared in include/bempp_b200.h.
//
// Every function keeps the name, argument order and meaning of the bempp-rs C interface
// (the src/bindings/ tree).  Where the reference panics (and so aborts across the FFI) these
// record a message for bempp_last_error() and return a neutral value; the *_ex and
// device variants return a status code.
#include <atomic>
#include <cstring>
#include <string>

#include "../../../include/bempp_b200.h"
#include "core.h"

using namespace bempp_b200;

namespace bempp_b200 {
void build_singular_pairs(GridT& g, SingularPairList& out);
}

struct BoundaryAssemblerOptionsT {
  Options options;
};

namespace {
thread_local std::string t_last_error;
std::atomic<uint64_t> g_grid_uid{1};
}

namespace bempp_b200 {
void set_last_error(const std::string& msg) { t_last_error = msg; }
void clear_last_error() { t_last_error.clear(); }
}  // namespace bempp_b200

namespace {

template <typename F>
BemppStatus guarded(F&& f) {
  try {
    clear_last_error();
    f();
    return BemppStatus_Ok;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_last_error("host out of memory");
    return BemppStatus_OutOfMemory;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return BemppStatus_Internal;
  }
}

template <typename T>
T* require(T* p, const char* what) {
  if (!p) throw Error(kInvalidArgument, std::string("null ") + what);
  return p;
}

}  // namespace

extern "C" {

const char* bempp_last_error(void) { return t_last_error.c_str(); }

// ----------------------------------------------------------------------- options ---
BoundaryAssemblerOptionsT* boundary_assembler_options_new(void) {
  return new BoundaryAssemblerOptionsT();
}

void boundary_assembler_options_t_free(BoundaryAssemblerOptionsT* ptr) { delete ptr; }

void boundary_assembler_options_set_regular_quadrature_degree(BoundaryAssemblerOptionsT* o,
                                                              ReferenceCellType cell_type,
                                                              size_t npoints) {
  guarded([&] {
    require(o, "options");
    // HashMap::entry(..).and_modify(..): only an existing key changes
    auto it = o->options.regular.find(cell_type);
    if (it != o->options.regular.end()) it->second = npoints;
  });
}

size_t boundary_assembler_options_get_regular_quadrature_degree(BoundaryAssemblerOptionsT* o,
                                                                ReferenceCellType cell_type) {
  size_t v = 0;
  guarded([&] {
    require(o, "options");
    auto it = o->options.regular.find(cell_type);
    if (it == o->options.regular.end())
      throw Error(kInvalidArgument, "no regular quadrature degree for this cell type");
    v = it->second;
  });
  return v;
}

bool boundary_assembler_options_has_regular_quadrature_degree(BoundaryAssemblerOptionsT* o,
                                                              ReferenceCellType cell_type) {
  return o && o->options.regular.count(cell_type) > 0;
}

void boundary_assembler_options_set_singular_quadrature_degree(BoundaryAssemblerOptionsT* o,
                                                               ReferenceCellType c0,
                                                               ReferenceCellType c1,
                                                               size_t npoints) {
  guarded([&] {
    require(o, "options");
    auto it = o->options.singular.find({c0, c1});
    if (it != o->options.singular.end()) it->second = npoints;
  });
}

size_t boundary_assembler_options_get_singular_quadrature_degree(BoundaryAssemblerOptionsT* o,
                                                                 ReferenceCellType c0,
                                                                 ReferenceCellType c1) {
  size_t v = 0;
  guarded([&] {
    require(o, "options");
    auto it = o->options.singular.find({c0, c1});
    if (it == o->options.singular.end())
      throw Error(kInvalidArgument, "no singular quadrature degree for this cell pair");
    v = it->second;
  });
  return v;
}

bool boundary_assembler_options_has_singular_quadrature_degree(BoundaryAssemblerOptionsT* o,
                                                               ReferenceCellType c0,
                                                               ReferenceCellType c1) {
  return o && o->options.singular.count({c0, c1}) > 0;
}

void boundary_assembler_options_set_batch_size(BoundaryAssemblerOptionsT* o, size_t batch_size) {
  if (o) o->options.batch_size = batch_size;
}

size_t boundary_assembler_options_get_batch_size(BoundaryAssemblerOptionsT* o) {
  return o ? o->options.batch_size : 0;
}

void boundary_assembler_options_set_precision(BoundaryAssemblerOptionsT* o, Precision p) {
  guarded([&] {
    require(o, "options");
    if (p > Precision_Mixed) throw Error(kInvalidArgument, "unknown precision");
    o->options.precision = p;
  });
}

Precision boundary_assembler_options_get_precision(BoundaryAssemblerOptionsT* o) {
  return o ? o->options.precision : Precision_FP64;
}

// -------------------------------------------------------------------- assemblers ---
static BoundaryAssemblerT* new_assembler(const BoundaryAssemblerOptionsT* o, int kernel,
                                         OperatorType op, DType dtype, double k) {
  BoundaryAssemblerT* out = nullptr;
  guarded([&] {
    require(o, "options");
    if (op > OperatorType_Hypersingular)
      throw Error(kUnsupported, std::string("invalid operator for ") +
                                    (kernel == kLaplace ? "Laplace" : "Helmholtz"));
    if (kernel == kLaplace && dtype != DType_F32 && dtype != DType_F64)
      throw Error(kInvalidArgument, "invalid dtype for Laplace");
    if (kernel == kHelmholtz && dtype != DType_C32 && dtype != DType_C64)
      throw Error(kInvalidArgument, "invalid dtype for Helmholtz");
    auto* a = new BoundaryAssemblerT();
    a->kernel = kernel;
    a->op = op;
    a->dtype = dtype;
    a->k = k;
    a->options = o->options;
    out = a;
  });
  return out;
}

BoundaryAssemblerT* laplace_boundary_assembler_new(const BoundaryAssemblerOptionsT* options,
                                                   OperatorType operator_type, DType dtype) {
  return new_assembler(options, kLaplace, operator_type, dtype, 0.0);
}

BoundaryAssemblerT* helmholtz_boundary_assembler_new(const void* k,
                                                     const BoundaryAssemblerOptionsT* options,
                                                     OperatorType operator_type, DType dtype) {
  if (!k) {
    set_last_error("null wavenumber");
    return nullptr;
  }
  double kv = dtype == DType_C32 ? static_cast<double>(*static_cast<const float*>(k))
                                 : *static_cast<const double*>(k);
  return new_assembler(options, kHelmholtz, operator_type, dtype, kv);
}

void boundary_assembler_t_free(BoundaryAssemblerT* ptr) { delete ptr; }

DType boundary_assembler_dtype(BoundaryAssemblerT* a) { return a ? a->dtype : DType_F64; }

BemppStatus boundary_assembler_assemble_into_device(BoundaryAssemblerT* a, SpaceT* trial,
                                                    SpaceT* test, void* device_data,
                                                    void* stream) {
  return guarded([&] {
    require(a, "assembler");
    require(trial, "trial space");
    require(test, "test space");
    if (test->ndofs > 0 && trial->ndofs > 0) require(device_data, "output");
    std::lock_guard<std::mutex> lock(a->mu);
    assemble_device(*a, *trial, *test, device_data, static_cast<cudaStream_t>(stream));
  });
}

BemppStatus bempp_device_status(void* stream) {
  return guarded([&] {
    BEMPP_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    unsigned n = 0;
    BEMPP_CUDA(take_stage_timeouts(&n));
    if (n)
      throw Error(kIncomplete, std::to_string(n) +
                                   " tile blocks timed out staging their input; their entries "
                                   "were not written");
  });
}

BemppStatus bempp_set_stage_wait_limit(int32_t polls) {
  return guarded([&] {
    if (polls < 0) throw Error(kInvalidArgument, "the poll count must be >= 0");
    BEMPP_CUDA(set_stage_poll_limit(polls));
  });
}

BemppStatus boundary_assembler_assemble_into_memory_ex(BoundaryAssemblerT* a, SpaceT* trial,
                                                       SpaceT* test, void* data) {
  return guarded([&] {
    require(a, "assembler");
    require(trial, "trial space");
    require(test, "test space");
    const size_t n = static_cast<size_t>(test->ndofs) * trial->ndofs;
    if (n == 0) return;
    require(data, "output");
    std::lock_guard<std::mutex> lock(a->mu);
    assemble_host(*a, *trial, *test, data);
  });
}

BemppStatus potential_assemble_into_memory(BoundaryAssemblerT* a, SpaceT* space,
                                           const double* points, size_t npoints, void* data) {
  return guarded([&] {
    require(a, "assembler");
    require(space, "space");
    if (npoints == 0 || space->ndofs == 0) return;
    require(points, "points");
    require(data, "output");
    std::lock_guard<std::mutex> lock(a->mu);
    assemble_potential_host(*a, *space, points, static_cast<int64_t>(npoints), data);
  });
}

BemppStatus potential_assemble_into_device(BoundaryAssemblerT* a, SpaceT* space,
                                           const double* device_points, size_t npoints,
                                           void* device_data, void* stream) {
  return guarded([&] {
    require(a, "assembler");
    require(space, "space");
    if (npoints == 0 || space->ndofs == 0) return;
    require(device_points, "points");
    require(device_data, "output");
    std::lock_guard<std::mutex> lock(a->mu);
    assemble_potential_device(*a, *space, device_points, static_cast<int64_t>(npoints),
                              device_data, static_cast<cudaStream_t>(stream));
  });
}

void boundary_assembler_assemble_into_memory(BoundaryAssemblerT* a, SpaceT* trial,
                                             SpaceT* test, void* data) {
  boundary_assembler_assemble_into_memory_ex(a, trial, test, data);
}

MatrixT* boundary_assembler_assemble(BoundaryAssemblerT* a, SpaceT* trial, SpaceT* test) {
  MatrixT* out = nullptr;
  guarded([&] {
    require(a, "assembler");
    require(trial, "trial space");
    require(test, "test space");
    auto* m = new MatrixT();
    m->csr = false;
    m->dtype = a->dtype;
    m->rows = test->ndofs;
    m->cols = trial->ndofs;
    m->data.resize(m->rows * m->cols * dtype_size(a->dtype));
    BemppStatus s = boundary_assembler_assemble_into_memory_ex(a, trial, test, m->data.data());
    if (s != BemppStatus_Ok) {
      std::string msg = bempp_last_error();
      delete m;
      throw Error(static_cast<Status>(s), msg);
    }
    out = m;
  });
  return out;
}

MatrixT* boundary_assembler_assemble_singular(BoundaryAssemblerT* a, SpaceT* trial,
                                              SpaceT* test) {
  MatrixT* out = nullptr;
  guarded([&] {
    require(a, "assembler");
    require(trial, "trial space");
    require(test, "test space");
    std::lock_guard<std::mutex> lock(a->mu);
    out = assemble_singular_csr(*a, *trial, *test);
  });
  return out;
}

void boundary_assembler_set_timing(BoundaryAssemblerT* a, bool enabled) {
  if (a) a->timing = enabled;
}

size_t boundary_assembler_host_copy_stats(BoundaryAssemblerT* a, double* out, size_t n) {
  if (!a || !out) return 0;
  std::lock_guard<std::mutex> lock(a->mu);
  const size_t m = std::min(n, a->host_copy_stats.size());
  for (size_t i = 0; i < m; ++i) out[i] = a->host_copy_stats[i];
  return m;
}

size_t boundary_assembler_phase_times(BoundaryAssemblerT* a, double* ms, size_t n) {
  size_t written = 0;
  guarded([&] {
    require(a, "assembler");
    if (a->events_recorded < 2) return;
    BEMPP_CUDA(cudaEventSynchronize(a->events[a->events_recorded - 1]));
    for (int i = 1; i < a->events_recorded && written < n; ++i) {
      float t = 0.f;
      BEMPP_CUDA(cudaEventElapsedTime(&t, a->events[i - 1], a->events[i]));
      if (ms) ms[written] = t;
      ++written;
    }
  });
  return written;
}

size_t boundary_assembler_last_launch_count(BoundaryAssemblerT* a) { return a ? a->launches : 0; }

BemppStatus bempp_measure_fma_peak(int fp64, int iters, int reps, double* tflops) {
  return guarded([&] {
    require(tflops, "output");
    if (iters <= 0 || reps <= 0) throw Error(kInvalidArgument, "iters and reps must be positive");
    BEMPP_CUDA(measure_fma_peak(fp64, iters, reps, tflops));
  });
}

long long bempp_lower_tile_pairs(int ntt, int ty0, int ty1, int* tx, int* sy,
                                 long long capacity) {
  if (ntt < 0 || ty0 < 0 || ty1 < ty0 || ty1 > ntt) return -1;
  const long long n = lower_tile_pair_count(ntt, ty0, ty1);
  for (long long b = 0; b < n && b < capacity; ++b) lower_tile_pair(b, ntt, ty0, ty1, tx[b], sy[b]);
  return n;
}

// ------------------------------------------------------------ page-locked outputs ---
// A cache of page-locked blocks: cudaHostAlloc'ing a gigabyte takes hundreds of
// milliseconds, so freed blocks are kept for the next result of a similar size (a block
// is reused for requests between half its size and its size).  Free blocks beyond
// kHostCacheBytes are released.
namespace {
constexpr size_t kHostCacheBytes = size_t(16) << 30;
std::mutex g_host_mu;
std::map<void*, size_t> g_host_used;
std::multimap<size_t, void*> g_host_free;  // by size
size_t g_host_free_bytes = 0;
}  // namespace

void* bempp_host_alloc(size_t bytes) {
  void* out = nullptr;
  guarded([&] {
    if (bytes == 0) throw Error(kInvalidArgument, "zero-byte block");
    std::lock_guard<std::mutex> lock(g_host_mu);
    auto it = g_host_free.lower_bound(bytes);
    if (it != g_host_free.end() && it->first / 2 <= bytes) {
      out = it->second;
      g_host_used[out] = it->first;
      g_host_free_bytes -= it->first;
      g_host_free.erase(it);
      return;
    }
    const size_t size = (bytes + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    BEMPP_CUDA(cudaHostAlloc(&out, size, cudaHostAllocDefault));
    g_host_used[out] = size;
  });
  return out;
}

void bempp_host_free(void* ptr) {
  if (!ptr) return;
  std::lock_guard<std::mutex> lock(g_host_mu);
  auto it = g_host_used.find(ptr);
  if (it == g_host_used.end()) return;
  g_host_free.emplace(it->second, ptr);
  g_host_free_bytes += it->second;
  g_host_used.erase(it);
  while (g_host_free_bytes > kHostCacheBytes && !g_host_free.empty()) {
    auto big = std::prev(g_host_free.end());
    cudaFreeHost(big->second);
    g_host_free_bytes -= big->first;
    g_host_free.erase(big);
  }
}

size_t bempp_host_trim(void) {
  std::lock_guard<std::mutex> lock(g_host_mu);
  size_t released = 0;
  for (auto& e : g_host_free) {
    cudaFreeHost(e.second);
    released += e.first;
  }
  g_host_free.clear();
  g_host_free_bytes = 0;
  return released;
}

size_t bempp_device_trim(void) { return device_cache_trim(); }

// ---------------------------------------------------------------------- matrices ---
size_t matrix_shape0(MatrixT* m) { return m ? m->rows : 0; }
size_t matrix_shape1(MatrixT* m) { return m ? m->cols : 0; }
DType matrix_dtype(MatrixT* m) { return m ? m->dtype : DType_F64; }
bool matrix_is_csr(MatrixT* m) { return m && m->csr; }

const void* matrix_dense_data(MatrixT* m) {
  if (!m || m->csr) {
    set_last_error("not a dense matrix");
    return nullptr;
  }
  return m->data.data();
}

void matrix_dense_data_copy(MatrixT* m, void* data) {
  if (!m || m->csr || !data) {
    set_last_error("not a dense matrix or null output");
    return;
  }
  std::memcpy(data, m->data.data(), m->data.size());
}

size_t matrix_csr_data_size(MatrixT* m) {
  return (m && m->csr) ? m->indices.size() : 0;
}
const void* matrix_csr_data(MatrixT* m) { return (m && m->csr) ? m->data.data() : nullptr; }
void matrix_csr_data_copy(MatrixT* m, void* data) {
  if (m && m->csr && data) std::memcpy(data, m->data.data(), m->data.size());
}
size_t matrix_csr_indices_size(MatrixT* m) { return (m && m->csr) ? m->indices.size() : 0; }
const uintptr_t* matrix_csr_indices(MatrixT* m) {
  return (m && m->csr) ? m->indices.data() : nullptr;
}
void matrix_csr_indices_copy(MatrixT* m, uintptr_t* indices) {
  if (m && m->csr && indices)
    std::memcpy(indices, m->indices.data(), m->indices.size() * sizeof(uintptr_t));
}
size_t matrix_csr_indptr_size(MatrixT* m) { return (m && m->csr) ? m->indptr.size() : 0; }
const uintptr_t* matrix_csr_indptr(MatrixT* m) {
  return (m && m->csr) ? m->indptr.data() : nullptr;
}
void matrix_csr_indptr_copy(MatrixT* m, uintptr_t* indptr) {
  if (m && m->csr && indptr)
    std::memcpy(indptr, m->indptr.data(), m->indptr.size() * sizeof(uintptr_t));
}
void matrix_t_free(MatrixT* ptr) { delete ptr; }

// ------------------------------------------------------------------------ spaces ---
SpaceT* function_space(GridT* grid, ElementFamilyT* e_family) {
  SpaceT* out = nullptr;
  guarded([&] {
    require(grid, "grid");
    require(e_family, "element family");
    out = make_space(grid, *e_family);
  });
  return out;
}

void space_t_free(SpaceT* ptr) { delete ptr; }

SpaceT* space_local_space(SpaceT* s) {
  SpaceT* out = nullptr;
  guarded([&] {
    require(s, "space");
    ElementFamilyT fam{s->degree, static_cast<uint8_t>(s->continuous ? 0 : 1), s->dtype};
    out = make_space(s->grid, fam);
  });
  return out;
}

bool space_is_serial(SpaceT* s) { return s != nullptr; }

size_t space_get_local_dof_numbers_size(SpaceT* s, size_t dim, size_t entity) {
  if (!s || dim > 2 || entity >= s->entity_dofs[dim].size()) return 0;
  return s->entity_dofs[dim][entity].size();
}

void space_get_local_dof_numbers(SpaceT* s, size_t dim, size_t entity, uintptr_t* dofs) {
  if (!s || !dofs || dim > 2 || entity >= s->entity_dofs[dim].size()) return;
  for (int64_t d : s->entity_dofs[dim][entity]) *dofs++ = static_cast<uintptr_t>(d);
}

size_t space_local_size(SpaceT* s) { return s ? static_cast<size_t>(s->ndofs) : 0; }
size_t space_global_size(SpaceT* s) { return s ? static_cast<size_t>(s->ndofs) : 0; }

bool space_has_cell_dofs(SpaceT* s, size_t cell) {
  return s && cell < static_cast<size_t>(s->grid->ncells);
}

size_t space_cell_dofs_size(SpaceT* s, size_t cell) {
  return space_has_cell_dofs(s, cell) ? static_cast<size_t>(s->nbasis) : 0;
}

void space_cell_dofs(SpaceT* s, size_t cell, uintptr_t* dofs) {
  if (!space_has_cell_dofs(s, cell) || !dofs) return;
  for (int b = 0; b < s->nbasis; ++b)
    dofs[b] = static_cast<uintptr_t>(s->cell_dofs[cell * s->nbasis + b]);
}

size_t space_cell_colouring(SpaceT* s, size_t* colours) {
  size_t n = 0;
  guarded([&] {
    require(s, "space");
    std::vector<std::vector<int64_t>> groups;
    {
      std::lock_guard<std::mutex> lock(s->grid->mu);
      s->grid->build_topology();
      groups = cell_colouring(*s);
    }
    n = groups.size();
    if (colours)
      for (size_t c = 0; c < groups.size(); ++c)
        for (int64_t cell : groups[c]) colours[cell] = c;
  });
  return n;
}

size_t space_global_dof_index(SpaceT* s, size_t local_dof_index) {
  (void)s;
  return local_dof_index;  // serial space: global numbering = local numbering
}

bool space_is_owned(SpaceT* s, size_t local_dof_index) {
  return s && local_dof_index < static_cast<size_t>(s->ndofs);
}

size_t space_ownership_process(SpaceT* s, size_t local_dof_index) {
  (void)s;
  (void)local_dof_index;
  return 0;
}

size_t space_ownership_index(SpaceT* s, size_t local_dof_index) {
  (void)s;
  return local_dof_index;
}

DType space_dtype(SpaceT* s) { return s ? s->dtype : DType_F64; }

// ------------------------------------------------------------- grids, elements ---
static GridT* make_grid(const void* points, size_t npoints, size_t gdim, DType dtype,
                        const size_t* cells, size_t ncells, size_t points_per_cell,
                        uint8_t cell_type = kTriangle) {
  GridT* out = nullptr;
  guarded([&] {
    if (npoints > 0) require(points, "points");
    if (ncells > 0) require(cells, "cells");
    if (gdim != 3) throw Error(kUnsupported, "only surface grids in 3D are supported");
    const int nv = cell_type == kQuadrilateral ? 4 : 3;
    if (points_per_cell < static_cast<size_t>(nv))
      throw Error(kInvalidArgument, nv == 4 ? "quadrilateral cells need four vertices"
                                            : "cells need three vertices");
    if (dtype != DType_F32 && dtype != DType_F64)
      throw Error(kInvalidArgument, "grid points must be F32 or F64");
    auto* g = new GridT();
    g->uid = g_grid_uid.fetch_add(1);
    g->dtype = dtype;
    g->npoints = static_cast<int64_t>(npoints);
    g->ncells = static_cast<int64_t>(ncells);
    g->cell_type = cell_type;
    g->points.resize(3 * npoints);
    for (size_t i = 0; i < 3 * npoints; ++i)
      g->points[i] = dtype == DType_F64 ? static_cast<const double*>(points)[i]
                                        : static_cast<const float*>(points)[i];
    g->cells.resize(nv * ncells);
    for (size_t c = 0; c < ncells; ++c)
      for (int i = 0; i < nv; ++i) {
        size_t v = cells[c * points_per_cell + i];
        if (v >= npoints) {
          delete g;
          throw Error(kInvalidArgument, "cell vertex index out of range");
        }
        g->cells[nv * c + i] = static_cast<int>(v);
      }
    out = g;
  });
  return out;
}

// ndgrid's single-element grid arrays (src/bindings/ndgrid.rs:18-56).  Layout as ndgrid's
// SingleElementGrid exposes it: per dimension d = 0..tdim, entity_counts[d] entities;
// downward_connectivity[d][sd] (sd = 0..d) holds, for each entity of dimension d, its
// downward_connectivity_shape0[d][sd] sub-entities of dimension sd contiguously (a
// column-major shape0 x count array).  Used here: cell -> vertex ([2][0], 3 per triangle,
// 4 per quadrilateral), and for triangles cell -> edge ([2][1], 3 per cell, local edge i
// opposite local vertex i) and edge -> vertex ([1][0], 2 per edge).  The topology's
// vertex ids decide adjacency and vertex DOFs (they may differ from the point indices of
// `cells`, e.g. when two points at one position are one vertex); the edge numbering is
// kept.  entity_types[2] (Triangle or Quadrilateral) is the cell type; a quadrilateral's
// vertices are in the reference square's order (0,0), (1,0), (0,1), (1,1).  Entity ids
// and the upward connectivity carry nothing the assembly needs.
GridT* single_element_grid_borrowed_create_bempp(
    size_t tdim, const size_t* id_sizes, const size_t* const* id_pointers,
    const ReferenceCellType* entity_types, const size_t* entity_counts,
    const size_t* const* const* downward_connectivity,
    const size_t* const* downward_connectivity_shape0,
    const size_t* const* const* const* upward_connectivity,
    const size_t* const* const* upward_connectivity_lens, const void* points, size_t gdim,
    size_t npoints, DType dtype, const size_t* cells, size_t points_per_cell, size_t ncells,
    size_t geometry_degree) {
  (void)id_sizes;
  (void)id_pointers;
  (void)upward_connectivity;
  (void)upward_connectivity_lens;
  const bool quads = entity_types && entity_types[2] == ReferenceCellType_Quadrilateral;
  if (tdim != 2 || (entity_types && entity_types[2] != ReferenceCellType_Triangle && !quads)) {
    set_last_error("only triangle and quadrilateral surface grids are supported");
    return nullptr;
  }
  if (geometry_degree != 1) {
    set_last_error("only degree-1 (flat triangle, bilinear quadrilateral) cells are supported");
    return nullptr;
  }
  const size_t nvc = quads ? 4 : 3;  // vertices per cell
  GridT* g = make_grid(points, npoints, gdim, dtype, cells, ncells, points_per_cell,
                       quads ? kQuadrilateral : kTriangle);
  if (!g || !downward_connectivity) return g;
  const BemppStatus st = guarded([&] {
    require(entity_counts, "entity_counts");
    require(downward_connectivity_shape0, "downward_connectivity_shape0");
    const size_t nv = entity_counts[0], ne = entity_counts[1];
    if (entity_counts[2] != ncells)
      throw Error(kInvalidArgument, "entity_counts[2] differs from the number of cells");
    if (nv > static_cast<size_t>(INT32_MAX) || ne > static_cast<size_t>(INT32_MAX))
      throw Error(kUnsupported, "too many topological entities for 32-bit ids");
    auto conn = [&](int d, int sd, size_t per) -> const size_t* {
      if (!downward_connectivity[d] || !downward_connectivity_shape0[d])
        throw Error(kInvalidArgument, "missing downward connectivity of dimension " + std::to_string(d));
      if (downward_connectivity_shape0[d][sd] != per)
        throw Error(kInvalidArgument, "downward connectivity [" + std::to_string(d) + "][" +
                                          std::to_string(sd) + "] must have " +
                                          std::to_string(per) + " entries per entity");
      return require(downward_connectivity[d][sd], "downward connectivity array");
    };
    const size_t* cv = conn(2, 0, nvc);
    g->topo.resize(nvc * ncells);
    for (size_t i = 0; i < nvc * ncells; ++i) {
      if (cv[i] >= nv) throw Error(kInvalidArgument, "cell -> vertex index out of range");
      g->topo[i] = static_cast<int>(cv[i]);
    }
    g->nvertices = static_cast<int64_t>(nv);
    if (!quads && ne > 0 && downward_connectivity[2][1] && downward_connectivity[1]) {
      const size_t* ce = conn(2, 1, 3);
      const size_t* ev = conn(1, 0, 2);
      g->given_edge_vertices.resize(2 * ne);
      for (size_t i = 0; i < 2 * ne; ++i) {
        if (ev[i] >= nv) throw Error(kInvalidArgument, "edge -> vertex index out of range");
        g->given_edge_vertices[i] = static_cast<int>(ev[i]);
      }
      g->given_cell_edges.resize(3 * ncells);
      for (size_t c = 0; c < ncells; ++c)
        for (int i = 0; i < 3; ++i) {
          const size_t e = ce[3 * c + i];
          if (e >= ne) throw Error(kInvalidArgument, "cell -> edge index out of range");
          // local edge i joins the cell's two vertices other than vertex i
          const int a = g->topo[3 * c + (i + 1) % 3], b = g->topo[3 * c + (i + 2) % 3];
          const int u = g->given_edge_vertices[2 * e], v = g->given_edge_vertices[2 * e + 1];
          if (!((u == a && v == b) || (u == b && v == a)))
            throw Error(kInvalidArgument, "cell -> edge connectivity disagrees with the "
                                          "cell -> vertex connectivity");
          g->given_cell_edges[3 * c + i] = static_cast<int>(e);
        }
    }
  });
  if (st != BemppStatus_Ok) {
    delete g;
    return nullptr;
  }
  return g;
}

GridT* bempp_grid_from_points_cells(const void* points, size_t npoints, DType dtype,
                                    const size_t* cells, size_t ncells) {
  return make_grid(points, npoints, 3, dtype, cells, ncells, 3);
}

void grid_t_free_bempp(GridT* ptr) { delete ptr; }

ElementFamilyT* create_lagrange_family_bempp(size_t degree, Continuity continuity, DType dtype) {
  if (degree > 2) {
    set_last_error("only Lagrange degree 0, 1 and 2 are supported");
    return nullptr;
  }
  if (continuity > Continuity_Discontinuous || dtype > DType_C64) {
    set_last_error("invalid continuity or dtype");
    return nullptr;
  }
  // degree 0 is always discontinuous
  return new ElementFamilyT{degree, static_cast<uint8_t>(degree == 0 ? 1 : continuity), dtype};
}

ElementFamilyT* create_raviart_thomas_family_bempp(size_t, Continuity, DType) {
  set_last_error("Raviart-Thomas spaces are not supported");
  return nullptr;
}

ElementFamilyT* create_nedelec_family_bempp(size_t, Continuity, DType) {
  set_last_error("Nedelec spaces are not supported");
  return nullptr;
}

void element_family_t_free_bempp(ElementFamilyT* ptr) { delete ptr; }

// ---------------------------------------------------------------- adjoint gradient ---
BemppStatus bempp_helmholtz_single_layer_dp0_gradient_device(
    GridT* grid, const BoundaryAssemblerOptionsT* options, double k, const void* lambda,
    const void* mu, double* value_and_grad_k, double* grad_points, void* stream) {
  return guarded([&] {
    require(grid, "grid");
    require(options, "options");
    if (grid->ncells == 0) return;
    require(lambda, "lambda");
    require(mu, "mu");
    require(value_and_grad_k, "value");
    require(grad_points, "grad_points");
    helmholtz_sl_gradient_device(*grid, options->options, k, static_cast<const double*>(lambda),
                                 static_cast<const double*>(mu), value_and_grad_k, grad_points,
                                 static_cast<cudaStream_t>(stream));
  });
}

BemppStatus bempp_helmholtz_single_layer_dp0_gradient(GridT* grid,
                                                      const BoundaryAssemblerOptionsT* options,
                                                      double k, const void* lambda,
                                                      const void* mu, double* value,
                                                      double* grad_k, double* grad_points) {
  return guarded([&] {
    require(grid, "grid");
    require(options, "options");
    require(value, "value");
    require(grad_k, "grad_k");
    require(grad_points, "grad_points");
    const size_t nc = static_cast<size_t>(grid->ncells), np = static_cast<size_t>(grid->npoints);
    if (nc == 0) {
      *value = *grad_k = 0.0;
      std::memset(grad_points, 0, sizeof(double) * 3 * np);
      return;
    }
    require(lambda, "lambda");
    require(mu, "mu");
    DeviceBuffer d_lam, d_mu, d_out, d_grad;
    d_lam.alloc(16 * nc);
    d_mu.alloc(16 * nc);
    d_out.alloc(16);
    d_grad.alloc(sizeof(double) * 3 * np);
    BEMPP_CUDA(cudaMemcpy(d_lam.ptr, lambda, 16 * nc, cudaMemcpyHostToDevice));
    BEMPP_CUDA(cudaMemcpy(d_mu.ptr, mu, 16 * nc, cudaMemcpyHostToDevice));
    BEMPP_CUDA(cudaStreamSynchronize(cudaStreamLegacy));  // the pageable copies have landed
    helmholtz_sl_gradient_device(*grid, options->options, k, d_lam.as<double>(),
                                 d_mu.as<double>(), d_out.as<double>(), d_grad.as<double>(),
                                 nullptr);
    double tot[2];
    BEMPP_CUDA(cudaMemcpy(tot, d_out.ptr, sizeof(tot), cudaMemcpyDeviceToHost));
    BEMPP_CUDA(cudaMemcpy(grad_points, d_grad.ptr, sizeof(double) * 3 * np,
                          cudaMemcpyDeviceToHost));
    unsigned n = 0;
    BEMPP_CUDA(take_stage_timeouts(&n));
    if (n)
      throw Error(kIncomplete, std::to_string(n) +
                                   " tile blocks timed out staging their input; the gradient "
                                   "misses their pairs");
    *value = tot[0];
    *grad_k = tot[1];
  });
}

// ------------------------------------------------------------------------- sweep ---
BemppStatus bempp_helmholtz_single_layer_dp0_sweep_device(GridT* const* grids, size_t ngrids,
                                                          const double* wavenumbers, size_t nk,
                                                          const BoundaryAssemblerOptionsT* options,
                                                          void* const* outputs, void* stream) {
  return guarded([&] {
    require(options, "options");
    if (ngrids == 0 || nk == 0) return;
    require(grids, "grids");
    require(wavenumbers, "wavenumbers");
    require(outputs, "outputs");
    for (size_t i = 0; i < ngrids; ++i) require(grids[i], "grid");
    helmholtz_sl_sweep_device(grids, ngrids, wavenumbers, nk, options->options, outputs,
                              static_cast<cudaStream_t>(stream));
  });
}

BemppStatus bempp_sweep_set_tuning(int32_t kchunk, int32_t blocks_per_sm, int32_t tile_shape) {
  return guarded([&] { set_sweep_tuning(kchunk, blocks_per_sm, tile_shape); });
}

BemppStatus bempp_sweep_last_tuning(int32_t* kchunk, int32_t* blocks_per_sm, int32_t* tile_shape,
                                    double* probe_ms) {
  return guarded([&] {
    const SweepTuning t = last_sweep_tuning();
    if (kchunk) *kchunk = t.kchunk;
    if (blocks_per_sm) *blocks_per_sm = t.blocks_per_sm;
    if (tile_shape) *tile_shape = t.tile_shape;
    if (probe_ms) *probe_ms = t.probe_ms;
  });
}

// ------------------------------------------------------- allocation-free assembly ---
BemppStatus bempp_assemble_regular_dp0_noalloc(
    int32_t kernel, OperatorType operator_type, double k, Precision precision,
    size_t regular_points, const double* test_points, size_t test_npoints,
    const int32_t* test_cells, size_t test_ncells, const double* trial_points,
    size_t trial_npoints, const int32_t* trial_cells, size_t trial_ncells, void* out,
    void* stream) {
  return guarded([&] {
    if (kernel != kLaplace && kernel != kHelmholtz) throw Error(kInvalidArgument, "kernel must be 0 or 1");
    if (operator_type > OperatorType_AdjointDoubleLayer)
      throw Error(kInvalidArgument, "operator must be single, double or adjoint double layer");
    if (precision > Precision_Mixed) throw Error(kInvalidArgument, "unknown precision");
    const size_t maxc = static_cast<size_t>(noalloc_max_cells());
    if (test_ncells > maxc || trial_ncells > maxc)
      throw Error(kInvalidArgument, "more than " + std::to_string(maxc) +
                                        " cells in a mesh (the scratch array's limit)");
    if (regular_points > static_cast<size_t>(noalloc_max_points()) ||
        !has_simplex_rule(static_cast<int>(regular_points)))
      throw Error(kInvalidArgument, "regular rule must have at most " +
                                        std::to_string(noalloc_max_points()) +
                                        " points and exist (1, 3, 6, 7 or 12)");
    if (test_ncells == 0 || trial_ncells == 0) return;
    require(test_points, "test points");
    require(test_cells, "test cells");
    require(trial_points, "trial points");
    require(trial_cells, "trial cells");
    require(out, "output");
    if (test_npoints == 0 || trial_npoints == 0) throw Error(kInvalidArgument, "empty point set");
    const RegularRule rule = simplex_rule(static_cast<int>(regular_points));
    RegularArgs ra;
    ra.kernel = kernel;
    ra.op = operator_type;
    ra.k = k;
    ra.same_grid = 0;
    ra.precision = precision == Precision_Mixed ? kRegularMixed : kRegularFP64;
    ra.out_type = kernel == kHelmholtz ? kOutC128 : kOutF64;
    ra.ld = static_cast<int64_t>(test_ncells);
    ra.out = out;
    if (test_npoints > static_cast<size_t>(INT32_MAX) || trial_npoints > static_cast<size_t>(INT32_MAX))
      throw Error(kInvalidArgument, "more points than int32 vertex indices can address");
    unsigned bad = 0;
    BEMPP_CUDA(assemble_regular_dp0_noalloc(
        ra, rule, test_points, static_cast<int>(test_npoints), test_cells,
        static_cast<int>(test_ncells), trial_points, static_cast<int>(trial_npoints), trial_cells,
        static_cast<int>(trial_ncells), &bad, static_cast<cudaStream_t>(stream)));
    if (bad != 0)
      throw Error(kInvalidArgument, std::to_string(bad) +
                                        " cell vertex index(es) outside [0, npoints); nothing "
                                        "was assembled");
  });
}

// -------------------------------------------------------------------- inspection ---
size_t bempp_regular_rule(size_t npoints, double* points, double* weights) {
  size_t n = 0;
  guarded([&] {
    if (!has_simplex_rule(static_cast<int>(npoints))) return;
    RegularRule r = simplex_rule(static_cast<int>(npoints));
    for (int i = 0; i < r.npts; ++i) {
      if (points) {
        points[2 * i] = r.xi[2 * i];
        points[2 * i + 1] = r.xi[2 * i + 1];
      }
      if (weights) weights[i] = r.w[i];
    }
    n = static_cast<size_t>(r.npts);
  });
  return n;
}

size_t bempp_singular_rule(size_t config, size_t order, double* test_points,
                           double* trial_points, double* weights) {
  size_t n = 0;
  guarded([&] {
    DuffyRule r = duffy_rule(static_cast<int>(config), static_cast<int>(order));
    n = r.w.size();
    if (test_points) std::memcpy(test_points, r.test_xi.data(), r.test_xi.size() * sizeof(double));
    if (trial_points)
      std::memcpy(trial_points, r.trial_xi.data(), r.trial_xi.size() * sizeof(double));
    if (weights) std::memcpy(weights, r.w.data(), r.w.size() * sizeof(double));
  });
  return n;
}

size_t bempp_quadrilateral_regular_rule(size_t npoints, double* points, double* weights) {
  size_t n = 0;
  guarded([&] {
    const QuadGaussRule r = quad_gauss_rule(npoints);
    for (int i = 0; i < r.n; ++i)
      for (int j = 0; j < r.n; ++j) {
        const int p = i * r.n + j;
        if (points) {
          points[2 * p] = r.x[i];
          points[2 * p + 1] = r.x[j];
        }
        if (weights) weights[p] = r.w[i] * r.w[j];
      }
    n = static_cast<size_t>(r.n) * r.n;
  });
  return n;
}

size_t bempp_quadrilateral_singular_rule(size_t config, size_t order, double* test_points,
                                         double* trial_points, double* weights) {
  size_t n = 0;
  guarded([&] {
    DuffyRule r = quad_duffy_rule(static_cast<int>(config), static_cast<int>(order));
    n = r.w.size();
    if (test_points) std::memcpy(test_points, r.test_xi.data(), r.test_xi.size() * sizeof(double));
    if (trial_points)
      std::memcpy(trial_points, r.trial_xi.data(), r.trial_xi.size() * sizeof(double));
    if (weights) std::memcpy(weights, r.w.data(), r.w.size() * sizeof(double));
  });
  return n;
}

size_t bempp_grid_singular_pairs(GridT* grid, size_t* test_cells, size_t* trial_cells,
                                 size_t* configs) {
  size_t n = 0;
  guarded([&] {
    require(grid, "grid");
    SingularPairList pl;
    {
      std::lock_guard<std::mutex> lock(grid->mu);
      grid->build_topology();
      build_singular_pairs(*grid, pl);
    }
    n = pl.test_cell.size();
    for (size_t i = 0; i < n; ++i) {
      if (test_cells) test_cells[i] = static_cast<size_t>(pl.test_cell[i]);
      if (trial_cells) trial_cells[i] = static_cast<size_t>(pl.trial_cell[i]);
      if (configs) configs[i] = static_cast<size_t>(pl.config[i]);
    }
  });
  return n;
}

}  // extern "C"
