// Host-side launchers of the assembly kernels (implemented in the .cu files of this
// directory).  All launches are asynchronous on `stream`; each returns the CUDA error of
// its launch.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "tile_order.h"

namespace bempp_b200 {

// Number of regular-kernel blocks since the last call whose shared-memory tile copies
// did not complete within their bounded wait (and that wrote nothing); resets it.
cudaError_t take_stage_timeouts(unsigned* count);
// Polls of the regular kernels' first wait for their tile copies on the current device
// (default kStagePolls; a test hook: 0 makes every block give up and write nothing).
cudaError_t set_stage_poll_limit(int polls);
// Device address of the timeout counter and the current first-wait poll limit, for kernels
// of other files that stage tiles the same way (the adjoint gradient's regular kernel).
cudaError_t stage_wait_state(unsigned** counter, int* polls);

// Per-cell FP64 geometry, regular quadrature points and vertex ids of a flat-triangle
// grid (points: npoints x 3 FP64; cells: ncells x 3 int32 point indices; topo: ncells x 3
// topology vertex ids for the adjacency tests, or null when they are the point indices).
cudaError_t launch_geometry(const double* points, const int* cells, const int* topo,
                            int ncells, const RegularRule& rule, double* geom, double* qpts,
                            float4* qrel, int* vids, cudaStream_t stream);

// Arithmetic of the regular far-pair quadrature.
enum RegularPrecision : int { kRegularFP64 = 0, kRegularMixed = 1 };

// Output element type of a dense matrix.
enum OutType : int { kOutF64 = 0, kOutC128 = 1, kOutF32 = 2, kOutC64 = 3 };

// Near field of a (test grid, trial grid) pair for the mixed-precision kernels, built on
// the host: per tile pair (test tile * trial tiles + trial tile) the index of its 32-word
// mask or -1; mask word [m * 32 + test lane] has bit j set when the pair (test lane, trial
// cell j) is near (centroid distance < 2 max diameter) or shares a vertex.  `pairs` lists
// the near pairs that share no vertex as (test cell, trial cell).
struct NearArgs {
  const int* tile_mask = nullptr;
  const unsigned* masks = nullptr;
  const int2* pairs = nullptr;
  int npairs = 0;
  int trial_tiles = 0;
  const int* test_dofs = nullptr;   // cell DOFs (scatter outputs)
  const int* trial_dofs = nullptr;
};

struct RegularArgs {
  int kernel;        // KernelKind
  int op;            // OpKind
  double k;          // wavenumber (Helmholtz)
  int same_grid;     // skip vertex-sharing pairs (they belong to the singular part)
  int precision;     // RegularPrecision
  int out_type;      // OutType
  int64_t ld;        // leading dimension = number of test DOFs
  void* out;         // column-major output
  int small_phase = 0;   // Helmholtz, mixed: k (max rad_test + max rad_trial) <= 0.8, so
                         // |k (r - r0)| <= 0.8 for every far pair (no phase reduction)
  NearArgs near{};       // mixed: near field (null: near pairs found per pair in the kernel)
  int symmetric = 0;     // 1: test and trial are one space and the operator is symmetric
                         // (SL, HS): only tile pairs (tx >= sy) are computed, then mirrored;
                         // 2: one P1 / DP1 space, DL or ADL, 6-point rule (Helmholtz:
                         // phases within the polynomial range): tile pairs (tx >= sy),
                         // each integrated in both orders
  int trial_tile0 = 0;   // first trial tile of this launch
  int trial_tiles = 0;   // trial tiles of this launch (0: all from trial_tile0 on)
};

// DP0 test x DP0 trial: every entry is written exactly once (no pre-zeroing needed).
cudaError_t launch_regular_dp0(const CellSet& test, const CellSet& trial,
                               const RegularRule& rule, const RegularArgs& a,
                               cudaStream_t stream);

// DOF layout of a space for the tile-scatter kernel.
struct SpaceTiles {
  int nbasis;               // 1 (DP0), 3 (P1 / DP1) or 6 (P2 / DP2)
  int tile_cells;           // cells per tile
  int ntiles;
  int max_tile_dofs;
  const int* tile_dof_off;  // ntiles + 1
  const int* tile_dofs;     // global DOF numbers of each tile, ascending
  const uint8_t* cell_ldof; // ncells * nbasis local (in-tile) DOF indices
  // incidence of the local DOFs: per tile (3 * tile_cells + 1) offsets and 3 * tile_cells
  // entries b * tile_cells + c, grouped by local DOF
  const uint8_t* inc_off = nullptr;
  const uint8_t* inc_ent = nullptr;
  const int* cell_dofs = nullptr;  // ncells * nbasis global DOF numbers
};

// Any pair of spaces: per-tile shared-memory accumulation, then atomic adds into a
// zero-initialised output.
cudaError_t launch_regular_scatter(const CellSet& test, const SpaceTiles& ttiles,
                                   const CellSet& trial, const SpaceTiles& stiles,
                                   const RegularRule& rule, const RegularArgs& a,
                                   cudaStream_t stream);

// Singular (Duffy) rules of all 28 adjacency configurations, concatenated.
struct SingularRules {
  const int* offset;       // 29 entries: first point of each configuration
  const double* test_xi;   // 2 * total
  const double* trial_xi;  // 2 * total
  const double* w;         // total
};

// Adjacent cell pairs (test cell, trial cell, configuration), grouped by configuration.
struct SingularPairs {
  int npairs;
  const int* test_cell;
  const int* trial_cell;
  const int* config;
};

struct SingularArgs {
  int kernel;
  int op;
  double k;
  int out_type;
  int64_t ld;
  void* out;          // dense column-major output (added into), or null
  int unique_entries; // 1 when every pair owns its entry (DP0 x DP0): plain stores
  double* pair_values;  // if non-null: per-pair local blocks (nbt * nbs [*2 complex])
  int trial_lo = 0;         // only pairs whose trial cell lies in [trial_lo, trial_hi)
  int trial_hi = 0x7fffffff;
};

cudaError_t launch_singular(const CellSet& test, const int* test_dofs, int nbt,
                            const CellSet& trial, const int* trial_dofs, int nbs,
                            const SingularRules& rules, const SingularPairs& pairs,
                            const SingularArgs& a, cudaStream_t stream);

// Cell-pair quadrature for any pairing of Lagrange degrees 0..2 (generic.cu), FP64, one
// warp per pair: the regular part over every (test cell, trial cell in [trial_lo,
// trial_hi)) pair (vertex-sharing pairs skipped on one grid) with the tensor rule, or the
// singular list with its Duffy rules.  Adds into the zero-initialised dense output (or
// stores per-pair blocks, singular only).
struct GenericPairArgs {
  int kernel, op;
  double k;
  int nbt, nbs;
  CellSet test, trial;
  const int* test_dofs;
  const int* trial_dofs;
  RegularRule rule;
  SingularRules rules;
  SingularPairs pairs;
  bool singular;
  int same_grid;
  void* out;
  int64_t ld;
  int trial_lo = 0, trial_hi = 0x7fffffff;
  double* pair_values = nullptr;
  // regular part, test and trial one space, symmetric operator (SL, HS): only the pairs
  // with test cell >= trial cell, each also added at the transposed entries
  int symmetric = 0;
};
cudaError_t launch_generic_pairs(const GenericPairArgs& g, cudaStream_t stream);

// Quadrilateral grids (quad.cu): bilinear cells given by their four vertices in the
// reference square's order (0,0), (1,0), (0,1), (1,1).
constexpr int kMaxQuadGauss = 16;
struct QuadGaussRule {  // n-point Gauss-Legendre rule on [0, 1]; the cell rule is n x n
  int n;
  double x[kMaxQuadGauss];
  double w[kMaxQuadGauss];
};
struct QuadCells {
  int ncells;
  const double* points;  // npoints x 3
  const int* cells;      // ncells x 4 point indices (geometry)
  const int* vids;       // ncells x 4 topology vertex ids (adjacency)
  // geometry at the n x n regular points (launch_quad_geometry), read by the regular part
  const double* qgeom = nullptr;
};
// Geometry of every cell at the rule's n x n points: field f of point p of cell c at
// out[f * ncells * n^2 + c * n^2 + p], fields x (3), jdet, unit normal (3), J0 (3), J1 (3)
// (13 * ncells * n^2 doubles).
constexpr int kQuadGeomFields = 13;
cudaError_t launch_quad_geometry(const QuadCells& cells, const QuadGaussRule& rule, double* out,
                                 cudaStream_t stream);
// Cell-pair quadrature of DP0 / Q1 / DQ1 spaces (nbt, nbs in {1, 4}), FP64, one warp per
// pair, as GenericPairArgs: the regular part over every (test cell, trial cell in
// [trial_lo, trial_hi)) pair (vertex-sharing pairs skipped on one grid) with the n x n
// Gauss rule on both cells, or the singular list with the quadrilateral Duffy rules.
struct QuadPairArgs {
  int kernel, op;
  double k;
  int nbt, nbs;
  QuadCells test, trial;
  const int* test_dofs;
  const int* trial_dofs;
  QuadGaussRule rule;
  SingularRules rules;
  SingularPairs pairs;
  bool singular;
  int same_grid;
  void* out;
  int64_t ld;
  int trial_lo = 0, trial_hi = 0x7fffffff;
  double* pair_values = nullptr;
  int symmetric = 0;  // as GenericPairArgs::symmetric
};
cudaError_t launch_quad_pairs(const QuadPairArgs& g, cudaStream_t stream);

// Allocation-free regular DP0 assembly between two distinct meshes (noalloc.cu); the
// scratch lives in a static device array of noalloc_max_cells() cells per mesh and
// noalloc_max_points() regular points.  The vertex indices are checked on the device
// first (the call waits for that check): *bad_indices receives the number outside
// [0, npoints), and when it is non-zero nothing else is launched.
int noalloc_max_cells();
int noalloc_max_points();
cudaError_t assemble_regular_dp0_noalloc(const RegularArgs& args, const RegularRule& rule,
                                         const double* test_points, int test_npoints,
                                         const int* test_cells, int test_ncells,
                                         const double* trial_points, int trial_npoints,
                                         const int* trial_cells, int trial_ncells,
                                         unsigned* bad_indices, cudaStream_t stream);

// Adjoint gradient of Re(lambda^H A mu) for the Helmholtz single layer on DP0 (adjoint.cu):
// grad_points (npoints x 3) and totals = {J, dJ/dk}; grad_cell is F x 9 scratch.
// Off-surface potential operators (potential.cu): out[i + ld * dof] for the npoints x 3
// row-major FP64 points and the trial space's DOFs; op kSL or kDL; P1 adds into the output
// (zero it first), DP0 stores.
cudaError_t launch_potential(int kernel, int op, const double* points, int npoints,
                             const CellSet& trial, const int* dofs, int nbasis,
                             const RegularRule& rule, double k, double* out, int64_t ld,
                             cudaStream_t stream);

cudaError_t launch_adjoint_sl(const CellSet& cs, const RegularRule& rule,
                              const SingularRules& rules, const SingularPairs& pairs, double k,
                              const double* lam, const double* mu, double* grad_cell,
                              double* grad_points, int npoints, double* totals, bool mixed,
                              cudaStream_t stream);

// Batched Helmholtz single-layer DP0 sweep (regular.cu): one persistent launch over
// every (mesh, test tile, trial tile, wavenumber chunk) item; complex64 outputs.
constexpr int kMaxSweepMeshes = 8;
struct SweepMesh {
  CellSet cells;          // geometry for the 6-point rule, with FP32 offsets
  float2* out;            // nk column-major ncells x ncells matrices, wavenumber-major
  int ntiles;             // ceil(ncells / 32)
  long long item_begin;   // first work item of this mesh
  // near field of the mesh with itself (NearArgs layout): per tile pair the index of its
  // 32-word mask of near or vertex-sharing pairs (or -1); the near pairs that share no
  // vertex, and the vertex-sharing pairs with their adjacency configuration
  const int* tile_mask;
  const unsigned* masks;
  const int2* near_pairs;
  int nnear;
  SingularPairs sing;
};
struct SweepArgs {
  SweepMesh mesh[kMaxSweepMeshes];
  int nmesh;
  const double* ks;       // device array of nk wavenumbers
  int nk;
  int kchunk;             // wavenumbers per work item
  int tile_shape = 1;     // a work item covers tile_shape x tile_shape pairs of 32-cell tiles
  long long nitems;
  unsigned long long* counter;  // work counter, zeroed before each launch
  // prefix sums over the meshes of (near pairs x nk) and (vertex-sharing pairs x nk)
  long long near_begin[kMaxSweepMeshes + 1];
  long long sing_begin[kMaxSweepMeshes + 1];
};
size_t sweep_smem_bytes(int tile_shape);
// The far pairs of every item: persistent launch of blocks_per_sm (at most 6) x sms CTAs
// (FP32, the pairs marked in the meshes' near-field masks left alone).
cudaError_t launch_sweep_sl(const SweepArgs& args, const RegularRule& rule,
                            const SingularRules& rules, int blocks_per_sm, int sms,
                            cudaStream_t stream);
// The near pairs (FP64, one thread per pair and wavenumber) and the vertex-sharing pairs
// (their Duffy rules, FP64, one warp per pair and wavenumber) of every mesh and
// wavenumber: they write the entries the far-pair launch leaves alone, so both may run
// concurrently.
cudaError_t launch_sweep_near_singular(const SweepArgs& args, const RegularRule& rule,
                                       const SingularRules& rules, cudaStream_t stream);

// CUDA-core FMA throughput probe (diag.cu).
cudaError_t measure_fma_peak(int fp64, int iters, int reps, double* tflops);

}  // namespace bempp_b200
