// Allocation-free variant of the regular DP0 assembly, for callers that cannot allocate
// GPU memory.
//
// Some callers own every byte of device memory they hand to a library and cannot let it
// call cudaMalloc: embedders that run under a fixed memory budget or a custom pool, code
// that must not allocate after start-up, and processes that only pass in buffers they
// already hold.  The regular DP0 kernel needs scratch beyond its inputs and outputs (the
// per-cell geometry and the physical quadrature points of both meshes, which the
// geometry kernel writes).  This file keeps that scratch in one file-scope
// `static __device__` array of fixed size, so bempp_assemble_regular_dp0_noalloc
// allocates nothing on the device (and makes no allocating library call): every GPU that
// loads the library holds the array (10.6 MB) until the process exits.
//
// The entry point assembles the regular-quadrature matrix between two distinct meshes:
// every (test cell, trial cell) pair with the regular rule and no singular part, which
// is exactly what the dense assembler computes when test and trial spaces live on
// different grid objects.  Limits: at most kNoAllocMaxCells cells per mesh and
// kNoAllocMaxPoints regular points.  Calls share the array: two calls whose work overlaps
// on the GPU (different streams, or different host threads) race on it and must be
// serialised by the caller.  Each call overwrites all the scratch it reads, so nothing
// has to be cleared between calls except the word that counts invalid vertex indices,
// which each call zeroes before its check.
//
// Vertex indices are validated on the device before the geometry pass reads any point:
// a small kernel counts the indices outside [0, npoints) of both meshes, the host reads
// that count back (one 4-byte copy and a wait for the caller's stream), and the call is
// rejected before any geometry or output is written when it is non-zero.
//
// The device address of the array is looked up once per device and kept for the life of
// the process; the entry point must not be used on a device after cudaDeviceReset (the
// array is re-created in the new context at another address).
#include <mutex>

#include "launch.h"

namespace bempp_b200 {
namespace {

constexpr int kNoAllocMaxCells = 8192;
constexpr int kNoAllocMaxPoints = 12;
constexpr int kMaxDevices = 64;

// Scratch of one mesh, in doubles: geometry fields, FP64 quadrature points, FP32 offsets
// (float4 per point: two doubles) and int32 vertex ids (two per double), with rows of
// kNoAllocMaxCells cells (a multiple of 32, so every sub-array keeps 256-byte alignment).
constexpr size_t kGeomDoubles = static_cast<size_t>(kNumGeomFields) * kNoAllocMaxCells;
constexpr size_t kQptsDoubles = static_cast<size_t>(3) * kNoAllocMaxPoints * kNoAllocMaxCells;
constexpr size_t kQrelDoubles = static_cast<size_t>(2) * kNoAllocMaxPoints * kNoAllocMaxCells;
constexpr size_t kVidsDoubles = static_cast<size_t>(3) * kNoAllocMaxCells / 2;
constexpr size_t kMeshDoubles = kGeomDoubles + kQptsDoubles + kQrelDoubles + kVidsDoubles;

static __device__ __align__(256) double g_noalloc_scratch[2 * kMeshDoubles];
// Invalid vertex indices found by the last call's check.
static __device__ unsigned g_noalloc_bad_indices;

// Device address of g_noalloc_scratch per device, looked up once per device with that
// device current.  The name of the array in host code is only a host-side stand-in.
std::mutex g_addr_mu;
double* g_addr[kMaxDevices] = {};
unsigned* g_bad_addr[kMaxDevices] = {};

cudaError_t scratch_address(int device, double** out, unsigned** bad) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_addr_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    void* q = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    e = cudaGetSymbolAddress(&q, g_noalloc_bad_indices);
    if (e != cudaSuccess) return e;
    g_addr[device] = static_cast<double*>(p);
    g_bad_addr[device] = static_cast<unsigned*>(q);
  }
  *out = g_addr[device];
  *bad = g_bad_addr[device];
  return cudaSuccess;
}

// Counts the entries of cells[0 .. n) outside [0, npoints) (grid-stride loop).
__global__ void count_bad_indices(const int* __restrict__ cells, int n, int npoints,
                                  unsigned* __restrict__ bad) {
  unsigned local = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int v = __ldg(cells + i);
    local += (v < 0 || v >= npoints) ? 1u : 0u;
  }
  if (local) atomicAdd(bad, local);
}

CellSet mesh_scratch(double* base, int ncells, int npts) {
  // field-major layouts with the padded stride of common.cuh
  CellSet cs;
  cs.ncells = ncells;
  cs.stride = cell_stride(ncells);
  double* geom = base;
  double* qpts = geom + kGeomDoubles;
  float4* qrel = reinterpret_cast<float4*>(qpts + kQptsDoubles);
  int* vids = reinterpret_cast<int*>(qpts + kQptsDoubles + kQrelDoubles);
  (void)npts;
  cs.geom = geom;
  cs.qpts = qpts;
  cs.qrel = qrel;
  cs.vids = vids;
  return cs;
}

}  // namespace

int noalloc_max_cells() { return kNoAllocMaxCells; }
int noalloc_max_points() { return kNoAllocMaxPoints; }

cudaError_t assemble_regular_dp0_noalloc(const RegularArgs& args, const RegularRule& rule,
                                         const double* test_points, int test_npoints,
                                         const int* test_cells, int test_ncells,
                                         const double* trial_points, int trial_npoints,
                                         const int* trial_cells, int trial_ncells,
                                         unsigned* bad_indices, cudaStream_t stream) {
  *bad_indices = 0;
  if (test_ncells > kNoAllocMaxCells || trial_ncells > kNoAllocMaxCells ||
      rule.npts > kNoAllocMaxPoints)
    return cudaErrorInvalidValue;
  int device = -1;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  double* base = nullptr;
  unsigned* bad = nullptr;
  e = scratch_address(device, &base, &bad);
  if (e != cudaSuccess) return e;
  // vertex indices first: nothing below reads a point before they are known to be valid
  e = cudaMemsetAsync(bad, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  count_bad_indices<<<64, 256, 0, stream>>>(test_cells, 3 * test_ncells, test_npoints, bad);
  count_bad_indices<<<64, 256, 0, stream>>>(trial_cells, 3 * trial_ncells, trial_npoints, bad);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  unsigned nbad = 0;
  e = cudaMemcpyAsync(&nbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, stream);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return e;
  if (nbad != 0) {
    *bad_indices = nbad;
    return cudaSuccess;
  }
  CellSet test = mesh_scratch(base, test_ncells, rule.npts);
  CellSet trial = mesh_scratch(base + kMeshDoubles, trial_ncells, rule.npts);
  e = launch_geometry(test_points, test_cells, nullptr, test_ncells, rule,
                      const_cast<double*>(test.geom),
                      const_cast<double*>(test.qpts), const_cast<float4*>(test.qrel),
                      const_cast<int*>(test.vids), stream);
  if (e != cudaSuccess) return e;
  e = launch_geometry(trial_points, trial_cells, nullptr, trial_ncells, rule,
                      const_cast<double*>(trial.geom), const_cast<double*>(trial.qpts),
                      const_cast<float4*>(trial.qrel), const_cast<int*>(trial.vids), stream);
  if (e != cudaSuccess) return e;
  return launch_regular_dp0(test, trial, rule, args, stream);
}

}  // namespace bempp_b200
