// Regular (non-singular) quadrature for DP0 test x DP0 trial spaces.
//
// Replaces the hot loop of bempp-rs assemble_batch_nonadjacent
// (src/boundary_assemblers.rs:689-773) with NonsingularCellPairAssemblerWithTestCaching
// (src/boundary_assemblers/cell_pair_assemblers.rs:283-339) for the single-layer,
// double-layer and adjoint double-layer integrands
// (src/boundary_assemblers/integrands/{single_layer,double_layer,adjoint_double_layer}.rs).
// Entry (i, j) = sum_p sum_q w_p w_q jdet_i jdet_j f(x_ip, y_jq); vertex-sharing pairs
// are written as 0 (the singular kernel adds them), as in
// src/boundary_assemblers.rs:754-756.
//
// Mapping: a CTA owns 128 consecutive test cells (one per thread, so a warp stores 32
// consecutive entries of one output column: column-major stores are coalesced) and
// kTrialTile consecutive trial cells, whose quadrature points are staged in shared
// memory and read as warp-wide broadcasts.  Each thread keeps its test cell's points
// in registers.  FP64 throughout; the mixed-precision variant computes far pairs in FP32.
#include "launch.h"

namespace bempp_b200 {
namespace {

constexpr int kThreads = 128;
constexpr int kTrialTile = 32;

struct TrialTileSmem {
  static __host__ __device__ size_t bytes(int q) {
    return sizeof(double) * (3 * q * kTrialTile + 5 * kTrialTile) + sizeof(int) * 3 * kTrialTile;
  }
};

// Coordinates of the test points: registers when Q is a template constant, otherwise
// a bounded local array.
template <int QT>
struct TestPoints {
  static constexpr int kCap = QT > 0 ? QT : kMaxRegularPoints;
  double x[kCap], y[kCap], z[kCap];
};

template <int QT, int KER, int OP>
__global__ void __launch_bounds__(kThreads)
    regular_dp0_fp64(CellSet test, CellSet trial, RegularRule rule, double k, int same_grid,
                     double* __restrict__ out, int64_t ld) {
  const int Q = QT > 0 ? QT : rule.npts;
  extern __shared__ double smem[];
  double* s_pts = smem;                     // [(q*3+d) * kTrialTile + j]
  double* s_jdet = s_pts + 3 * Q * kTrialTile;
  double* s_n = s_jdet + kTrialTile;        // [d * kTrialTile + j]
  double* s_h = s_n + 3 * kTrialTile;       // plane offset v0 . n
  int* s_vid = reinterpret_cast<int*>(s_h + kTrialTile);

  const int nt = test.ncells, ns = trial.ncells;
  const int j0 = blockIdx.y * kTrialTile;
  const int nj = min(kTrialTile, ns - j0);
  for (int idx = threadIdx.x; idx < 3 * Q * kTrialTile; idx += kThreads) {
    int j = idx % kTrialTile, pd = idx / kTrialTile;
    s_pts[idx] = j < nj ? __ldg(trial.qpts + static_cast<int64_t>(pd) * ns + j0 + j) : 0.0;
  }
  for (int j = threadIdx.x; j < kTrialTile; j += kThreads) {
    if (j < nj) {
      int c = j0 + j;
      double nx = g(trial.geom, kNx, ns, c), ny = g(trial.geom, kNy, ns, c),
             nz = g(trial.geom, kNz, ns, c);
      s_jdet[j] = g(trial.geom, kJdet, ns, c);
      s_n[j] = nx;
      s_n[kTrialTile + j] = ny;
      s_n[2 * kTrialTile + j] = nz;
      s_h[j] = g(trial.geom, kV0x, ns, c) * nx + g(trial.geom, kV0y, ns, c) * ny +
               g(trial.geom, kV0z, ns, c) * nz;
      for (int v = 0; v < 3; ++v) s_vid[v * kTrialTile + j] = __ldg(trial.vids + v * ns + c);
    } else {
      s_jdet[j] = 0.0;
      s_n[j] = s_n[kTrialTile + j] = s_n[2 * kTrialTile + j] = 0.0;
      s_h[j] = 0.0;
      for (int v = 0; v < 3; ++v) s_vid[v * kTrialTile + j] = -1;
    }
  }
  __syncthreads();

  const int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= nt) return;

  TestPoints<QT> tp;
#pragma unroll
  for (int p = 0; p < Q; ++p) {
    tp.x[p] = __ldg(test.qpts + static_cast<int64_t>(3 * p) * nt + i);
    tp.y[p] = __ldg(test.qpts + static_cast<int64_t>(3 * p + 1) * nt + i);
    tp.z[p] = __ldg(test.qpts + static_cast<int64_t>(3 * p + 2) * nt + i);
  }
  const double jdet_i = g(test.geom, kJdet, nt, i);
  const double nxi = g(test.geom, kNx, nt, i), nyi = g(test.geom, kNy, nt, i),
               nzi = g(test.geom, kNz, nt, i);
  const double h_i = g(test.geom, kV0x, nt, i) * nxi + g(test.geom, kV0y, nt, i) * nyi +
                     g(test.geom, kV0z, nt, i) * nzi;
  const int a0 = __ldg(test.vids + i), a1 = __ldg(test.vids + nt + i),
            a2 = __ldg(test.vids + 2 * nt + i);

  for (int j = 0; j < nj; ++j) {
    const int64_t o = static_cast<int64_t>(j0 + j) * ld + i;
    const bool adjacent =
        same_grid && share_vertex(a0, a1, a2, s_vid[j], s_vid[kTrialTile + j],
                                  s_vid[2 * kTrialTile + j]);
    const double scale = jdet_i * s_jdet[j] * kInv4Pi;
    double bq[QT > 0 ? QT : kMaxRegularPoints];
    if (OP == kADL) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
        bq[q] = s_pts[(3 * q) * kTrialTile + j] * nxi + s_pts[(3 * q + 1) * kTrialTile + j] * nyi +
                s_pts[(3 * q + 2) * kTrialTile + j] * nzi - h_i;
    }
    double acc_re = 0.0, acc_im = 0.0;
    if (!adjacent) {
#pragma unroll
      for (int p = 0; p < Q; ++p) {
        double ap = 0.0;
        if (OP == kDL)
          ap = tp.x[p] * s_n[j] + tp.y[p] * s_n[kTrialTile + j] +
               tp.z[p] * s_n[2 * kTrialTile + j] - s_h[j];
        double in_re = 0.0, in_im = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const double dx = tp.x[p] - s_pts[(3 * q) * kTrialTile + j];
          const double dy = tp.y[p] - s_pts[(3 * q + 1) * kTrialTile + j];
          const double dz = tp.z[p] - s_pts[(3 * q + 2) * kTrialTile + j];
          const double r2 = dx * dx + dy * dy + dz * dz;
          const double rinv = rsqrt(r2);
          double wq = rule.w[q];
          if (OP == kADL) wq *= bq[q];
          if (KER == kLaplace) {
            if (OP == kSL)
              in_re = fma(wq, rinv, in_re);
            else
              in_re = fma(wq, rinv * rinv * rinv, in_re);
          } else {
            const double r = r2 * rinv;
            double s, c;
            sincos(k * r, &s, &c);
            if (OP == kSL) {
              const double f = wq * rinv;
              in_re = fma(f, c, in_re);
              in_im = fma(f, s, in_im);
            } else {
              const double f = wq * rinv * rinv * rinv;
              const double kr = k * r;
              in_re = fma(f, fma(kr, s, c), in_re);
              in_im = fma(f, fma(-kr, c, s), in_im);
            }
          }
        }
        double wp = rule.w[p];
        if (OP == kDL) wp *= ap;
        acc_re = fma(wp, in_re, acc_re);
        if (KER == kHelmholtz) acc_im = fma(wp, in_im, acc_im);
      }
    }
    if (KER == kLaplace) {
      out[o] = acc_re * scale;
    } else {
      double2 v = make_double2(acc_re * scale, acc_im * scale);
      reinterpret_cast<double2*>(out)[o] = v;
    }
  }
}

template <int QT, int KER>
cudaError_t launch_op(const CellSet& test, const CellSet& trial, const RegularRule& rule,
                      const RegularArgs& a, cudaStream_t stream) {
  dim3 grid((test.ncells + kThreads - 1) / kThreads, (trial.ncells + kTrialTile - 1) / kTrialTile);
  size_t smem = TrialTileSmem::bytes(rule.npts);
  double* out = static_cast<double*>(a.out);
  switch (a.op) {
    case kSL:
      cudaFuncSetAttribute(regular_dp0_fp64<QT, KER, kSL>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      regular_dp0_fp64<QT, KER, kSL><<<grid, kThreads, smem, stream>>>(test, trial, rule, a.k,
                                                                       a.same_grid, out, a.ld);
      break;
    case kDL:
      cudaFuncSetAttribute(regular_dp0_fp64<QT, KER, kDL>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      regular_dp0_fp64<QT, KER, kDL><<<grid, kThreads, smem, stream>>>(test, trial, rule, a.k,
                                                                       a.same_grid, out, a.ld);
      break;
    case kADL:
      cudaFuncSetAttribute(regular_dp0_fp64<QT, KER, kADL>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      regular_dp0_fp64<QT, KER, kADL><<<grid, kThreads, smem, stream>>>(test, trial, rule, a.k,
                                                                        a.same_grid, out, a.ld);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int QT>
cudaError_t launch_q(const CellSet& test, const CellSet& trial, const RegularRule& rule,
                     const RegularArgs& a, cudaStream_t stream) {
  return a.kernel == kLaplace ? launch_op<QT, kLaplace>(test, trial, rule, a, stream)
                              : launch_op<QT, kHelmholtz>(test, trial, rule, a, stream);
}

}  // namespace

cudaError_t launch_regular_dp0_mixed(const CellSet& test, const CellSet& trial,
                                     const RegularRule& rule, const RegularArgs& a,
                                     cudaStream_t stream);

cudaError_t launch_regular_dp0(const CellSet& test, const CellSet& trial,
                               const RegularRule& rule, const RegularArgs& a,
                               cudaStream_t stream) {
  if (test.ncells <= 0 || trial.ncells <= 0) return cudaSuccess;
  if (a.precision == kRegularMixed || a.out_type == kOutF32 || a.out_type == kOutC64)
    return launch_regular_dp0_mixed(test, trial, rule, a, stream);
  if (a.op == kHS) return cudaErrorInvalidValue;
  switch (rule.npts) {
    case 6:
      return launch_q<6>(test, trial, rule, a, stream);
    default:
      return launch_q<0>(test, trial, rule, a, stream);
  }
}

}  // namespace bempp_b200
