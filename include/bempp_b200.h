/*
 * bempp_b200.h -- C-ABI of the B200 dense boundary-operator assembler.
 *
 * Drop-in for the C interface that bempp-rs generates with cbindgen from
 * the src/bindings/ tree (cbindgen.toml: enums prefixed with their name): every function of
 * that interface on the dense-assembly path keeps its name, argument order, argument
 * meaning and ownership rules.  Each declaration cites the reference function it
 * replaces.  Additions (status-returning variants, device-pointer assembly, precision
 * selection, timing, batched sweep, adjoint gradient) are marked "Addition".
 *
 * Conventions (as in the reference):
 *   - Opaque heap handles, each released by its *_t_free function (null-safe).
 *   - Dense outputs are column-major: entry (test dof i, trial dof j) is at
 *     i + n_test * j (src/boundary_assemblers.rs:766).
 *   - Functions that return nothing in the reference abort on invalid input there; here
 *     they record the error (bempp_last_error) and return without writing.  The *_ex
 *     variants return a status code instead.
 */
#ifndef BEMPP_B200_H
#define BEMPP_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* c-api-tools DType (src/bindings/space.rs:189-198; python/bempp/function_space.py:13-16). */
enum { DType_F32 = 0, DType_F64 = 1, DType_C32 = 2, DType_C64 = 3 };
typedef uint8_t DType;

/* ndelement ReferenceCellType (python/bempp/function_space.py:23-35). */
enum {
  ReferenceCellType_Point = 0,
  ReferenceCellType_Interval = 1,
  ReferenceCellType_Triangle = 2,
  ReferenceCellType_Quadrilateral = 3,
  ReferenceCellType_Tetrahedron = 4,
  ReferenceCellType_Hexahedron = 5,
  ReferenceCellType_Prism = 6,
  ReferenceCellType_Pyramid = 7
};
typedef uint8_t ReferenceCellType;

/* ndelement Continuity (src/bindings/ndelement.rs:19-25). */
enum { Continuity_Standard = 0, Continuity_Discontinuous = 1 };
typedef uint8_t Continuity;

/* src/bindings/boundary_assemblers.rs:15-24 */
enum {
  OperatorType_SingleLayer = 0,
  OperatorType_DoubleLayer = 1,
  OperatorType_AdjointDoubleLayer = 2,
  OperatorType_Hypersingular = 3,
  OperatorType_ElectricField = 4,
  OperatorType_MagneticField = 5
};
typedef uint8_t OperatorType;

/* Addition: arithmetic of the regular far-pair quadrature.  Precision_FP64 computes
 * everything in FP64 (the reference's f64/c64 semantics).  Precision_Mixed computes
 * regular pairs whose centroid distance is at least two element diameters in FP32
 * with compensated accumulation; geometry, near pairs and singular pairs stay FP64. */
enum { Precision_FP64 = 0, Precision_Mixed = 1 };
typedef uint8_t Precision;

/* Addition: status codes of the *_ex functions. */
enum {
  BemppStatus_Ok = 0,
  BemppStatus_InvalidArgument = 1,
  BemppStatus_Unsupported = 2,
  BemppStatus_OutOfMemory = 3,
  BemppStatus_CudaError = 4,
  BemppStatus_NoDevice = 5,
  BemppStatus_Internal = 6,
  BemppStatus_Incomplete = 7
};
typedef int32_t BemppStatus;

typedef struct BoundaryAssemblerOptionsT BoundaryAssemblerOptionsT;
typedef struct BoundaryAssemblerT BoundaryAssemblerT;
typedef struct MatrixT MatrixT;
typedef struct SpaceT SpaceT;
typedef struct GridT GridT;
typedef struct ElementFamilyT ElementFamilyT;

/* Addition: message of the last error on this thread ("" if none). */
const char *bempp_last_error(void);

/* ------------------------------------------------------------------ options ----- */
/* src/bindings/boundary_assemblers.rs:34-40 */
BoundaryAssemblerOptionsT *boundary_assembler_options_new(void);
/* src/bindings/boundary_assemblers.rs:42-50 (null-safe) */
void boundary_assembler_options_t_free(BoundaryAssemblerOptionsT *ptr);
/* src/bindings/boundary_assemblers.rs:52-60 (only changes an existing cell type) */
void boundary_assembler_options_set_regular_quadrature_degree(
    BoundaryAssemblerOptionsT *options, ReferenceCellType cell_type, size_t npoints);
/* src/bindings/boundary_assemblers.rs:61-68 (returns 0 and records an error if absent) */
size_t boundary_assembler_options_get_regular_quadrature_degree(
    BoundaryAssemblerOptionsT *options, ReferenceCellType cell_type);
/* src/bindings/boundary_assemblers.rs:69-76 */
bool boundary_assembler_options_has_regular_quadrature_degree(
    BoundaryAssemblerOptionsT *options, ReferenceCellType cell_type);
/* src/bindings/boundary_assemblers.rs:78-87 */
void boundary_assembler_options_set_singular_quadrature_degree(
    BoundaryAssemblerOptionsT *options, ReferenceCellType cell_type0,
    ReferenceCellType cell_type1, size_t npoints);
/* src/bindings/boundary_assemblers.rs:88-98 */
size_t boundary_assembler_options_get_singular_quadrature_degree(
    BoundaryAssemblerOptionsT *options, ReferenceCellType cell_type0,
    ReferenceCellType cell_type1);
/* src/bindings/boundary_assemblers.rs:99-109 */
bool boundary_assembler_options_has_singular_quadrature_degree(
    BoundaryAssemblerOptionsT *options, ReferenceCellType cell_type0,
    ReferenceCellType cell_type1);
/* src/bindings/boundary_assemblers.rs:111-118 */
void boundary_assembler_options_set_batch_size(BoundaryAssemblerOptionsT *options,
                                               size_t batch_size);
/* src/bindings/boundary_assemblers.rs:119-125 */
size_t boundary_assembler_options_get_batch_size(BoundaryAssemblerOptionsT *options);
/* Addition: precision of the regular far-pair quadrature (default Precision_FP64). */
void boundary_assembler_options_set_precision(BoundaryAssemblerOptionsT *options,
                                              Precision precision);
Precision boundary_assembler_options_get_precision(BoundaryAssemblerOptionsT *options);

/* --------------------------------------------------------------- assemblers ----- */
/* src/bindings/boundary_assemblers.rs:127-166 (F32 or F64) */
BoundaryAssemblerT *laplace_boundary_assembler_new(const BoundaryAssemblerOptionsT *options,
                                                   OperatorType operator_type, DType dtype);
/* src/bindings/boundary_assemblers.rs:168-210 (C32 or C64; k points to a float for C32
 * and a double for C64, as T::Real there) */
BoundaryAssemblerT *helmholtz_boundary_assembler_new(const void *k,
                                                     const BoundaryAssemblerOptionsT *options,
                                                     OperatorType operator_type, DType dtype);
/* src/bindings/boundary_assemblers.rs:26-27 (#[cfuncs(name = "boundary_assembler_t", free)]) */
void boundary_assembler_t_free(BoundaryAssemblerT *ptr);
/* src/bindings/boundary_assemblers.rs:212-233 */
DType boundary_assembler_dtype(BoundaryAssemblerT *assembler);
/* src/bindings/boundary_assemblers.rs:272-307: owned dense MatrixT (column-major) */
MatrixT *boundary_assembler_assemble(BoundaryAssemblerT *assembler, SpaceT *trial_space,
                                     SpaceT *test_space);
/* src/bindings/boundary_assemblers.rs:235-270: singular part as an owned CSR MatrixT */
MatrixT *boundary_assembler_assemble_singular(BoundaryAssemblerT *assembler,
                                              SpaceT *trial_space, SpaceT *test_space);
/* src/bindings/boundary_assemblers.rs:309-348: dense assembly into caller memory holding
 * n_test * n_trial elements of the assembler's dtype, column-major (host memory). */
void boundary_assembler_assemble_into_memory(BoundaryAssemblerT *assembler,
                                             SpaceT *trial_space, SpaceT *test_space,
                                             void *data);
/* Addition: as boundary_assembler_assemble_into_memory, with a status code. */
BemppStatus boundary_assembler_assemble_into_memory_ex(BoundaryAssemblerT *assembler,
                                                       SpaceT *trial_space,
                                                       SpaceT *test_space, void *data);
/* Addition: dense assembly into device memory on the current CUDA device, enqueued on
 * `stream` (a cudaStream_t; NULL = legacy default stream).  Returns after enqueueing;
 * the matrix is complete when the stream reaches that point. */
BemppStatus boundary_assembler_assemble_into_device(BoundaryAssemblerT *assembler,
                                                    SpaceT *trial_space, SpaceT *test_space,
                                                    void *device_data, void *stream);
/* Addition: completion check of device-memory assemblies.  Waits for `stream` (a
 * cudaStream_t; NULL = legacy default stream), then reports whether any block of the
 * regular kernels launched on the current device since the last check gave up waiting for
 * its shared-memory tile copies (a bounded wait; never expected): such a block writes none
 * of its entries, and the call returns BemppStatus_Incomplete with the block count in
 * bempp_last_error().  Resets the count.  The host-memory entry points make this check
 * themselves. */
BemppStatus bempp_device_status(void *stream);
/* Addition, a test hook: the number of polls of the regular kernels' first wait for their
 * tile copies on the current device (default 4194304; 0 makes every block give up at once
 * and write nothing, after a second full-length wait that drains its copies). */
BemppStatus bempp_set_stage_wait_limit(int32_t polls);
/* Addition: record CUDA events around each phase of the next assemblies and read the
 * last durations in milliseconds: [geometry, output clear, regular, singular (+ final
 * conversion)]; returns the number of phases written (at most n).  Reading waits for
 * the last assembly to finish. */
void boundary_assembler_set_timing(BoundaryAssemblerT *assembler, bool enabled);
size_t boundary_assembler_phase_times(BoundaryAssemblerT *assembler, double *ms, size_t n);
/* Addition: number of kernel launches the last assembly enqueued. */
size_t boundary_assembler_last_launch_count(BoundaryAssemblerT *assembler);
/* Addition (no counterpart in the reference): statistics of the last host-memory
 * assembly (boundary_assembler_assemble_into_memory[_ex] / boundary_assembler_assemble):
 * [ms the host waited for device-to-host DMA, ms of host copies into the caller's array,
 * copy groups, assembly chunks, host copy threads, ms spent taking the destination's page
 * faults ahead of the copies, device ms from the first launch to the end of the last
 * chunk's kernels and to the end of the last DMA (page-locked destinations, else 0)];
 * returns the number written (<= n). */
size_t boundary_assembler_host_copy_stats(BoundaryAssemblerT *assembler, double *out, size_t n);
/* Addition: off-surface potential operators, the single and double layer potentials of
 * the assembler's kernel (OperatorType SingleLayer or DoubleLayer; others fail with
 * BemppStatus_Unsupported).  out[i + npoints * j] = sum over the cells of DOF j of
 * jdet int psi_j(y) K(x_i, y) dy by the regular rule of the assembler's options, with
 * K = G(x, y) (single layer) or n_y . grad_y G(x, y) (double layer), G = 1/(4 pi r) or
 * e^{ikr}/(4 pi r); column-major npoints x ndofs in the assembler's dtype.  `points` is
 * npoints x 3, row-major FP64.  Replaces the evaluator the reference declares in
 * src/boundary_evaluators.rs (an empty file; its bempp-cl comparisons are the commented
 * tests at tests/compare_to_bempp_cl.rs:208-320).  The points must lie off the surface. */
BemppStatus potential_assemble_into_memory(BoundaryAssemblerT *assembler, SpaceT *space,
                                           const double *points, size_t npoints, void *data);
/* The same with device points and a device output, enqueued on `stream`. */
BemppStatus potential_assemble_into_device(BoundaryAssemblerT *assembler, SpaceT *space,
                                           const double *device_points, size_t npoints,
                                           void *device_data, void *stream);
/* Addition: measured CUDA-core fused multiply-add throughput of the current device in
 * TFLOP/s (fp64 != 0: FP64, else FP32), the roofline denominator of the regular
 * quadrature kernels. */
BemppStatus bempp_measure_fma_peak(int fp64, int iters, int reps, double *tflops);
/* Addition: the order in which a lower-triangle launch (symmetric operator on one space,
 * adjoint gradient, batched sweep) visits the tile pairs of trial tiles [ty0, ty1) out of
 * ntt 32-cell tiles: writes up to `capacity` (test tile, trial tile) pairs to tx / sy and
 * returns the pair count (host copy of the kernels' decoding, for self-checks). */
long long bempp_lower_tile_pairs(int ntt, int ty0, int ty1, int *tx, int *sy, long long capacity);
/* Addition (no counterpart in the reference): page-locked host blocks for dense outputs.
 * A matrix assembled into page-locked memory is written by DMA as its columns finish,
 * with no staging copy.  bempp_host_alloc returns a block of at least `bytes` (NULL and
 * bempp_last_error() on failure) from a process-wide cache; bempp_host_free returns it
 * to the cache (blocks stay page-locked for reuse); bempp_host_trim releases every
 * cached free block to the system and returns the bytes released. */
void *bempp_host_alloc(size_t bytes);
void bempp_host_free(void *ptr);
size_t bempp_host_trim(void);
/* Addition (no counterpart in the reference): the library keeps the device blocks of
 * freed grids, spaces and assemblers for reuse (building and freeing them again makes no
 * cudaMalloc / cudaFree calls); bempp_device_trim releases every cached free block to the
 * driver and returns the bytes released. */
size_t bempp_device_trim(void);

/* ------------------------------------------------------------------ matrices ----- */
/* src/bindings/matrices.rs:6-20 */
size_t matrix_shape0(MatrixT *matrix);
size_t matrix_shape1(MatrixT *matrix);
/* src/bindings/matrices.rs:29-49 (dense only) */
const void *matrix_dense_data(MatrixT *matrix);
void matrix_dense_data_copy(MatrixT *matrix, void *data);
/* src/bindings/matrices.rs:57-137 (CSR only; indices and indptr are uintptr_t) */
size_t matrix_csr_data_size(MatrixT *matrix);
const void *matrix_csr_data(MatrixT *matrix);
void matrix_csr_data_copy(MatrixT *matrix, void *data);
size_t matrix_csr_indices_size(MatrixT *matrix);
const uintptr_t *matrix_csr_indices(MatrixT *matrix);
void matrix_csr_indices_copy(MatrixT *matrix, uintptr_t *indices);
size_t matrix_csr_indptr_size(MatrixT *matrix);
const uintptr_t *matrix_csr_indptr(MatrixT *matrix);
void matrix_csr_indptr_copy(MatrixT *matrix, uintptr_t *indptr);
/* src/bindings.rs:13-14 (#[cfuncs(name = "matrix_t", free)]) */
void matrix_t_free(MatrixT *ptr);
/* Addition: DType of a matrix, and whether it is CSR (true) or dense (false). */
DType matrix_dtype(MatrixT *matrix);
bool matrix_is_csr(MatrixT *matrix);

/* -------------------------------------------------------------------- spaces ----- */
/* src/bindings/space.rs:20-42 */
SpaceT *function_space(GridT *grid, ElementFamilyT *e_family);
/* src/bindings/space.rs:17-18 (#[cfuncs(name = "space_t", free)]) */
void space_t_free(SpaceT *ptr);
/* src/bindings/space.rs:44-56 (a serial space is its own local space) */
SpaceT *space_local_space(SpaceT *space);
/* src/bindings/space.rs:58-67 */
bool space_is_serial(SpaceT *space);
/* src/bindings/space.rs:69-106 */
size_t space_get_local_dof_numbers_size(SpaceT *space, size_t entity_dim,
                                        size_t entity_number);
void space_get_local_dof_numbers(SpaceT *space, size_t entity_dim, size_t entity_number,
                                 uintptr_t *dofs);
/* src/bindings/space.rs:108-128 */
size_t space_local_size(SpaceT *space);
size_t space_global_size(SpaceT *space);
/* src/bindings/space.rs:130-165 */
bool space_has_cell_dofs(SpaceT *space, size_t cell);
size_t space_cell_dofs_size(SpaceT *space, size_t cell);
void space_cell_dofs(SpaceT *space, size_t cell, uintptr_t *dofs);
/* Addition: the greedy cell colouring of FunctionSpace::cell_colouring
 * (src/function.rs:281-351, which has no C binding in the reference): cells in grid order
 * take the lowest colour not yet used by a cell sharing one of their DOF entities
 * (vertices for continuous spaces, the cell itself otherwise).  Writes each cell's colour
 * to colours[cell] (ncells entries; NULL to query) and returns the number of colours. */
size_t space_cell_colouring(SpaceT *space, size_t *colours);
/* src/bindings/space.rs:167-187 */
size_t space_global_dof_index(SpaceT *space, size_t local_dof_index);
bool space_is_owned(SpaceT *space, size_t local_dof_index);
/* python/bempp/function_space.py:95-102 (ghost owner; serial spaces own every DOF) */
size_t space_ownership_process(SpaceT *space, size_t local_dof_index);
size_t space_ownership_index(SpaceT *space, size_t local_dof_index);
/* src/bindings/space.rs:189-198 */
DType space_dtype(SpaceT *space);

/* ---------------------------------------------------------- grids, elements ----- */
/* src/bindings/ndgrid.rs:18-56: ndgrid's borrowed single-element grid.  The topology
 * arrays are accepted for signature compatibility; the grid is rebuilt from `points`
 * (npoints x gdim, DType_F32 or DType_F64) and `cells` (ncells x points_per_cell point
 * indices, the first three being the triangle's vertices). */
GridT *single_element_grid_borrowed_create_bempp(
    size_t tdim, const size_t *id_sizes, const size_t *const *id_pointers,
    const ReferenceCellType *entity_types, const size_t *entity_counts,
    const size_t *const *const *downward_connectivity,
    const size_t *const *downward_connectivity_shape0,
    const size_t *const *const *const *upward_connectivity,
    const size_t *const *const *upward_connectivity_lens, const void *points, size_t gdim,
    size_t npoints, DType dtype, const size_t *cells, size_t points_per_cell, size_t ncells,
    size_t geometry_degree);
/* Addition: flat-triangle grid from points (npoints x 3) and cells (ncells x 3). */
GridT *bempp_grid_from_points_cells(const void *points, size_t npoints, DType dtype,
                                    const size_t *cells, size_t ncells);
/* src/bindings/ndgrid.rs:6-16 (null-safe) */
void grid_t_free_bempp(GridT *ptr);
/* src/bindings/ndelement.rs:18-25: Lagrange degree 0, 1 or 2 on triangles (degree 2:
 * DOFs at the vertices, then at the midpoints of edges [1,2], [0,2], [0,1], nodal basis;
 * spaces of degree 2 are assembled in FP64 by a warp-per-cell-pair kernel whatever the
 * precision option) */
ElementFamilyT *create_lagrange_family_bempp(size_t degree, Continuity continuity,
                                             DType dtype);
/* src/bindings/ndelement.rs:27-43: not supported (returns NULL, records an error) */
ElementFamilyT *create_raviart_thomas_family_bempp(size_t degree, Continuity continuity,
                                                   DType dtype);
ElementFamilyT *create_nedelec_family_bempp(size_t degree, Continuity continuity,
                                            DType dtype);
/* src/bindings/ndelement.rs:9-19 (null-safe) */
void element_family_t_free_bempp(ElementFamilyT *ptr);

/* Addition: adjoint gradient of J = Re(lambda^H A mu) for the Helmholtz single-layer
 * operator A(x, k) on DP0 x DP0 spaces of `grid` (test = trial), with respect to every
 * point coordinate and to k, without forming dA (FP64; options give the regular rule and
 * the singular order).  lambda, mu: complex128 arrays of ncells; outputs J, dJ/dk and
 * grad_points (npoints x 3).  Host pointers: */
BemppStatus bempp_helmholtz_single_layer_dp0_gradient(GridT *grid,
                                                      const BoundaryAssemblerOptionsT *options,
                                                      double k, const void *lambda,
                                                      const void *mu, double *value,
                                                      double *grad_k, double *grad_points);
/* Addition: the same with device pointers, enqueued on `stream`; value_and_grad_k holds
 * {J, dJ/dk}.  Its tile copies have the bounded wait of the assembly kernels: the host
 * version returns BemppStatus_Incomplete if one gave up, and after this one
 * bempp_device_status(stream) does. */
BemppStatus bempp_helmholtz_single_layer_dp0_gradient_device(
    GridT *grid, const BoundaryAssemblerOptionsT *options, double k, const void *lambda,
    const void *mu, double *value_and_grad_k, double *grad_points, void *stream);

/* Addition: batched Helmholtz single-layer DP0 frequency sweep.  For every grid i and
 * every wavenumber k_j, writes the ncells_i x ncells_i complex64 matrix (column-major) at
 * outputs[i] + j * ncells_i^2 (device memory, nk matrices per grid): regular far pairs in
 * FP32, near and singular pairs in FP64, all in one persistent launch replayed from a
 * captured CUDA graph.  `wavenumbers` is a host array; the options must select the
 * 6-point regular rule.  The launch parameters (wavenumbers per work item, CTAs per SM)
 * are chosen by a timing autotuner on the first call for a set of mesh sizes; calls with
 * the same grids, wavenumbers and outputs replay the same graph.  Enqueued on `stream`. */
BemppStatus bempp_helmholtz_single_layer_dp0_sweep_device(GridT *const *grids, size_t ngrids,
                                                          const double *wavenumbers, size_t nk,
                                                          const BoundaryAssemblerOptionsT *options,
                                                          void *const *outputs, void *stream);
/* Addition: fixes the sweep's launch parameters for the following sweeps instead of
 * autotuning (kchunk wavenumbers per work item, blocks_per_sm 1..6 CTAs per SM,
 * tile_shape 1 or 2); kchunk <= 0 returns to autotuning and forgets earlier results. */
BemppStatus bempp_sweep_set_tuning(int32_t kchunk, int32_t blocks_per_sm, int32_t tile_shape);
/* Addition: parameters the autotuner chose for the last sweep: wavenumbers per work item,
 * CTAs per SM, tile shape (a work item covers tile_shape x tile_shape pairs of 32-cell
 * tiles) and probe_ms, its measured milliseconds per (tile pair, wavenumber) on the probe
 * slice.  Any pointer may be NULL. */
BemppStatus bempp_sweep_last_tuning(int32_t *kchunk, int32_t *blocks_per_sm, int32_t *tile_shape,
                                    double *probe_ms);

/* Addition, with no counterpart in the reference: dense regular-quadrature assembly of a
 * DP0 x DP0 Laplace (kernel 0) or Helmholtz (kernel 1) single-layer, double-layer or
 * adjoint double-layer operator between two distinct meshes, for callers that cannot
 * allocate GPU memory.  It allocates nothing: every input and the output are the
 * caller's device buffers, and the scratch it needs (per-cell geometry and quadrature
 * points) is a fixed static device array held by each GPU that loads the library.
 * Inputs: points (n x 3 FP64) and cells (n x 3 int32) of each mesh, in device memory.
 * Output: n_test_cells x n_trial_cells column-major, FP64 (Laplace) or interleaved
 * complex128 (Helmholtz).  Every pair uses the regular rule of `regular_points` points
 * and there is no singular part (the two meshes are treated as different grids), as in
 * boundary_assembler_assemble_into_device with spaces on two grid objects.  Limits: at
 * most 8192 cells per mesh and 12 regular points; larger sizes are rejected with
 * BemppStatus_InvalidArgument.  Vertex indices are checked on the device against
 * test_npoints / trial_npoints before any point is read: the call waits for that check
 * (and for the work queued before it on `stream`) and returns BemppStatus_InvalidArgument,
 * having written nothing, if an index lies outside [0, npoints); the assembly itself is
 * then enqueued and the call returns.  The first call on a device looks up the array's
 * device address; make that call before any stream capture, and do not call it on a
 * device after cudaDeviceReset.  Calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
BemppStatus bempp_assemble_regular_dp0_noalloc(
    int32_t kernel, OperatorType operator_type, double k, Precision precision,
    size_t regular_points, const double *test_points, size_t test_npoints,
    const int32_t *test_cells, size_t test_ncells, const double *trial_points,
    size_t trial_npoints, const int32_t *trial_cells, size_t trial_ncells, void *out,
    void *stream);

/* ------------------------------------------------------- inspection (host) ----- */
/* Addition: the regular (non-singular) rule with `npoints` points on the reference
 * triangle: points as x0,y0,x1,y1,... and weights summing to 1/2.  Returns npoints, or
 * 0 if no rule has that many points.  Either array may be NULL. */
size_t bempp_regular_rule(size_t npoints, double *points, double *weights);
/* Addition: the Duffy rule of adjacency configuration `config` (0..27 in the order of
 * src/boundary_assemblers.rs:267-288: 9 vertex, 18 edge, 1 identical) with 1-D order
 * `order`.  Returns the number of points (arrays of 2n, 2n, n; NULL to query), or 0. */
size_t bempp_singular_rule(size_t config, size_t order, double *test_points,
                           double *trial_points, double *weights);
/* Addition: the regular rule used on quadrilaterals for a requested count of `npoints`:
 * the n x n Gauss-Legendre tensor rule on [0,1]^2, n the smallest with n^2 >= npoints
 * (at most 16).  Points as x0,y0,x1,y1,... (point i * n + j at (g_i, g_j)), weights
 * summing to 1.  Returns n^2 (0 on error); either array may be NULL. */
size_t bempp_quadrilateral_regular_rule(size_t npoints, double *points, double *weights);
/* Addition: the Duffy rule of quadrilateral configuration `config` (0..48: 16 vertex
 * pairings test * 4 + trial, 32 edge pairings 16 + (test edge * 4 + trial edge) * 2 +
 * orientation with the edges [0,1], [0,2], [1,3], [2,3], the identical cell 48) with 1-D
 * order `order`: 4, 6 or 8 regions of order^4 points.  Returns the number of points. */
size_t bempp_quadrilateral_singular_rule(size_t config, size_t order, double *test_points,
                                         double *trial_points, double *weights);
/* Addition: the ordered cell pairs of a grid that share a vertex (the singular part),
 * grouped by configuration as src/boundary_assemblers.rs:564-606 groups them (the 28
 * triangle or the 49 quadrilateral configurations).  Returns the number of pairs; arrays
 * may be NULL to query. */
size_t bempp_grid_singular_pairs(GridT *grid, size_t *test_cells, size_t *trial_cells,
                                 size_t *configs);

#ifdef __cplusplus
}
#endif

#endif /* BEMPP_B200_H */
