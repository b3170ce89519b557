// Off-surface potential operators of the boundary kernels, FP64:
//   P[i, j] = sum_{cells c with DOF j} jdet_c sum_q w_q psi_b(xi_q) K(x_i, y_c(xi_q)),
// single layer K = G(x, y), double layer K = n_y . grad_y G(x, y), with
//   Laplace     G = 1 / (4 pi r),         n_y . grad_y G = (x - y).n_y / (4 pi r^3),
//   Helmholtz   G = e^{ikr} / (4 pi r),   n_y . grad_y G = e^{ikr} (1 - ikr) (x - y).n_y / (4 pi r^3),
// r = |x - y|, for evaluation points x_i off the surface (regular quadrature only).  The
// reference declares src/boundary_evaluators.rs (empty) and keeps bempp-cl values for these
// four operators in commented tests (tests/compare_to_bempp_cl.rs:208-320); the kernel
// conventions are those of its boundary operators (src/boundary_assemblers/helpers.rs:7-40,
// integrands/single_layer.rs, integrands/double_layer.rs).
//
// Tiles of 32 points (lane = point, coordinates in registers) x 32 trial cells (staged in
// shared memory, warps stride them).  DP0: every (point, cell) pair owns its entry (plain
// stores); P1: three DOFs per cell, added with global atomics into the zeroed output.
#include "launch.h"
#include "tiles.cuh"

namespace bempp_b200 {
namespace {

using namespace tiles;

template <int KER, int OP, int NB>
__global__ void __launch_bounds__(kThreads)
    potential_tiles(const double* __restrict__ points, int npoints, CellSet trial,
                    const int* __restrict__ dofs, RegularRule rule, double k,
                    double* __restrict__ out, int64_t ld) {
  constexpr bool kC = KER == kHelmholtz;
  const int Q = rule.npts;
  const int i0 = blockIdx.x * kTile, c0 = blockIdx.y * kTile;
  const int nc = min(kTile, trial.ncells - c0);
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* cursor = smem;
  const Tile S = carve_tile(cursor, Q, false, 1);
  load_tile(S, trial, c0, nc, Q, false, nullptr, 1);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i = i0 + lane;
  if (i >= npoints) return;  // no barrier follows
  const double x0 = points[3 * static_cast<int64_t>(i)], x1 = points[3 * static_cast<int64_t>(i) + 1],
               x2 = points[3 * static_cast<int64_t>(i) + 2];
  for (int js = warp; js < nc; js += kWarps) {
    const double nx = S.G(fNx, js), ny = S.G(fNy, js), nz = S.G(fNz, js);
    double u_re[NB], u_im[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) u_re[b] = u_im[b] = 0.0;
    for (int q = 0; q < Q; ++q) {
      const double dx = x0 - S.P(q, 0, js), dy = x1 - S.P(q, 1, js), dz = x2 - S.P(q, 2, js);
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double rinv = rsqrt(r2);
      double kre, kim = 0.0;
      if (KER == kLaplace) {
        kre = OP == kSL ? rinv : (dx * nx + dy * ny + dz * nz) * rinv * rinv * rinv;
      } else {
        const double r = r2 * rinv, kr = k * r;
        double sn, cs;
        sincos(kr, &sn, &cs);
        if (OP == kSL) {
          kre = rinv * cs;
          kim = rinv * sn;
        } else {
          // Re, Im of e^{ikr} (1 - ikr) = (cos + kr sin) + i (sin - kr cos)
          const double f = (dx * nx + dy * ny + dz * nz) * rinv * rinv * rinv;
          kre = f * fma(kr, sn, cs);
          kim = f * fma(-kr, cs, sn);
        }
      }
      double bv[NB], bd0[NB], bd1[NB];  // degree 2: the basis at the point (bd* unused)
      if (NB == 6) lagrange_basis<NB>(rule.xi[2 * q], rule.xi[2 * q + 1], bv, bd0, bd1);
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const double wb = NB == 1 ? rule.w[q] : NB == 3 ? rule.wphi[b][q] : rule.w[q] * bv[b];
        u_re[b] = fma(kre, wb, u_re[b]);
        if (kC) u_im[b] = fma(kim, wb, u_im[b]);
      }
    }
    const double sc = S.G(fJdet, js) * kInv4Pi;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int64_t o = i + ld * __ldg(dofs + static_cast<int64_t>(c0 + js) * NB + b);
      if (NB == 1) {
        if (kC)
          reinterpret_cast<double2*>(out)[o] = make_double2(u_re[b] * sc, u_im[b] * sc);
        else
          out[o] = u_re[b] * sc;
      } else {
        atomicAdd(out + (kC ? 2 * o : o), u_re[b] * sc);
        if (kC) atomicAdd(out + 2 * o + 1, u_im[b] * sc);
      }
    }
  }
}

template <int KER, int OP, int NB>
cudaError_t launch_nb(const double* points, int npoints, const CellSet& trial, const int* dofs,
                      const RegularRule& rule, double k, double* out, int64_t ld,
                      cudaStream_t stream) {
  const size_t smem = sizeof(double) * tile_doubles(rule.npts) + sizeof(int) * tile_ints(1) + 32;
  auto fn = potential_tiles<KER, OP, NB>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  const dim3 grid((npoints + kTile - 1) / kTile, (trial.ncells + kTile - 1) / kTile);
  fn<<<grid, kThreads, smem, stream>>>(points, npoints, trial, dofs, rule, k, out, ld);
  return cudaGetLastError();
}

template <int KER, int OP>
cudaError_t launch_op(const double* points, int npoints, const CellSet& trial, const int* dofs,
                      int nbasis, const RegularRule& rule, double k, double* out, int64_t ld,
                      cudaStream_t stream) {
  if (nbasis == 1) return launch_nb<KER, OP, 1>(points, npoints, trial, dofs, rule, k, out, ld, stream);
  if (nbasis == 3) return launch_nb<KER, OP, 3>(points, npoints, trial, dofs, rule, k, out, ld, stream);
  if (nbasis == 6) return launch_nb<KER, OP, 6>(points, npoints, trial, dofs, rule, k, out, ld, stream);
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_potential(int kernel, int op, const double* points, int npoints,
                             const CellSet& trial, const int* dofs, int nbasis,
                             const RegularRule& rule, double k, double* out, int64_t ld,
                             cudaStream_t stream) {
  if (npoints <= 0 || trial.ncells <= 0) return cudaSuccess;
  if (op != kSL && op != kDL) return cudaErrorInvalidValue;
  if (kernel == kLaplace)
    return op == kSL ? launch_op<kLaplace, kSL>(points, npoints, trial, dofs, nbasis, rule, k, out, ld, stream)
                     : launch_op<kLaplace, kDL>(points, npoints, trial, dofs, nbasis, rule, k, out, ld, stream);
  return op == kSL ? launch_op<kHelmholtz, kSL>(points, npoints, trial, dofs, nbasis, rule, k, out, ld, stream)
                   : launch_op<kHelmholtz, kDL>(points, npoints, trial, dofs, nbasis, rule, k, out, ld, stream);
}

}  // namespace bempp_b200
