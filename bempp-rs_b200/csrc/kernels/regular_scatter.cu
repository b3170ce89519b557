// Regular (non-singular) quadrature for any pair of DP0 / P1 / DP1 spaces.
//
// Replaces bempp-rs assemble_nonsingular_part + assemble_batch_nonadjacent
// (src/boundary_assemblers.rs:396-521,689-773) with the cell-pair assembler
// (src/boundary_assemblers/cell_pair_assemblers.rs:283-339) and all four integrands,
// including the Helmholtz hypersingular sum curl-curl - k^2 normal-normal
// (src/helmholtz.rs:98-104).  The reference avoids write races by colouring cells
// (src/function.rs:281-351) and scattering each 128x128 block serially; here a CTA owns
// a tile of kTile test cells x kTile trial cells, accumulates the local blocks of its
// kTile^2 cell pairs into a shared-memory matrix over the DOFs those cells touch, and
// flushes that matrix once with atomic adds into the zero-initialised output.
//
// Per cell pair the point-pair loop is factorised: U_b(p) = sum_q K(x_p, y_q) psi_b(q)
// w_q, block[a][b] = sum_p phi_a(p) w_p U_b(p), so a P1 x P1 pair costs one kernel
// evaluation and NBS fused multiply-adds per point pair.  The hypersingular curl-curl
// term uses the constant surface curls of flat cells: c_a = t1 d0(phi_a) - t0 d1(phi_a)
// = (t0 - t1, t1, -t0) for the three P1 basis functions.
#include "launch.h"

namespace bempp_b200 {
namespace {

constexpr int kTile = 32;       // cells per tile (test and trial)
constexpr int kThreads = 256;   // 8 warps: lane = test cell, warp = trial cell stride
constexpr int kWarps = kThreads / 32;

// Real or complex accumulator.
template <int KER>
struct Acc;
template <>
struct Acc<kLaplace> {
  double re;
  __device__ void zero() { re = 0.0; }
};
template <>
struct Acc<kHelmholtz> {
  double re, im;
  __device__ void zero() { re = im = 0.0; }
};

struct TrialSmem {
  // layout of the per-CTA trial tile, in doubles then ints
  static __host__ __device__ size_t doubles(int q) { return (3 * q + 16) * kTile; }
  static __host__ __device__ size_t ints(int nbs) { return (3 + nbs) * kTile; }
};

template <int QT>
struct Pts {
  static constexpr int kCap = QT > 0 ? QT : kMaxRegularPoints;
  double x[kCap], y[kCap], z[kCap];
};

template <int QT, int KER, int OP, int NBT, int NBS>
__global__ void __launch_bounds__(kThreads)
    regular_scatter_fp64(CellSet test, SpaceTiles tt, CellSet trial, SpaceTiles st,
                         RegularRule rule, double k, int same_grid, double* __restrict__ out,
                         int64_t ld) {
  constexpr bool kCplx = KER == kHelmholtz;
  const int Q = QT > 0 ? QT : rule.npts;
  const int nt = test.ncells, ns = trial.ncells;
  const int ti0 = blockIdx.x * kTile, sj0 = blockIdx.y * kTile;
  const int nti = min(kTile, nt - ti0), nsj = min(kTile, ns - sj0);

  const int tdof0 = tt.tile_dof_off[blockIdx.x];
  const int ndt = tt.tile_dof_off[blockIdx.x + 1] - tdof0;
  const int sdof0 = st.tile_dof_off[blockIdx.y];
  const int nds = st.tile_dof_off[blockIdx.y + 1] - sdof0;

  extern __shared__ double smem[];
  double* acc_re = smem;                              // ndt * nds
  double* acc_im = acc_re + tt.max_tile_dofs * st.max_tile_dofs;  // complex only
  double* s = acc_re + (kCplx ? 2 : 1) * tt.max_tile_dofs * st.max_tile_dofs;
  double* s_pts = s;                       // [(q*3+d) * kTile + j]
  double* s_geo = s_pts + 3 * Q * kTile;   // 16 fields * kTile
  int* s_int = reinterpret_cast<int*>(s_geo + 16 * kTile);  // vids (3), ldofs (NBS)

  for (int idx = threadIdx.x; idx < ndt * nds; idx += kThreads) {
    acc_re[idx] = 0.0;
    if (kCplx) acc_im[idx] = 0.0;
  }
  for (int idx = threadIdx.x; idx < 3 * Q * kTile; idx += kThreads) {
    int j = idx % kTile, pd = idx / kTile;
    s_pts[idx] = j < nsj ? __ldg(trial.qpts + static_cast<int64_t>(pd) * ns + sj0 + j) : 0.0;
  }
  for (int j = threadIdx.x; j < kTile; j += kThreads) {
    const int c = sj0 + min(j, nsj - 1);
    // 0 jdet, 1-3 n, 4 h, 5-7 t0, 8-10 t1
    double nx = g(trial.geom, kNx, ns, c), ny = g(trial.geom, kNy, ns, c),
           nz = g(trial.geom, kNz, ns, c);
    s_geo[0 * kTile + j] = g(trial.geom, kJdet, ns, c);
    s_geo[1 * kTile + j] = nx;
    s_geo[2 * kTile + j] = ny;
    s_geo[3 * kTile + j] = nz;
    s_geo[4 * kTile + j] = g(trial.geom, kV0x, ns, c) * nx + g(trial.geom, kV0y, ns, c) * ny +
                           g(trial.geom, kV0z, ns, c) * nz;
    for (int f = 0; f < 6; ++f) s_geo[(5 + f) * kTile + j] = g(trial.geom, kT0x + f, ns, c);
    for (int v = 0; v < 3; ++v) s_int[v * kTile + j] = __ldg(trial.vids + v * ns + c);
    for (int b = 0; b < NBS; ++b) s_int[(3 + b) * kTile + j] = st.cell_ldof[c * NBS + b];
  }
  __syncthreads();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i = ti0 + lane;
  if (lane < nti) {
    Pts<QT> tp;
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
    double t0i[3], t1i[3];
    for (int d = 0; d < 3; ++d) {
      t0i[d] = g(test.geom, kT0x + d, nt, i);
      t1i[d] = g(test.geom, kT1x + d, nt, i);
    }
    const int a0 = __ldg(test.vids + i), a1 = __ldg(test.vids + nt + i),
              a2 = __ldg(test.vids + 2 * nt + i);
    int lt[NBT];
    for (int a = 0; a < NBT; ++a) lt[a] = tt.cell_ldof[i * NBT + a];

    for (int j = warp; j < nsj; j += kWarps) {
      if (same_grid && share_vertex(a0, a1, a2, s_int[j], s_int[kTile + j], s_int[2 * kTile + j]))
        continue;
      const double* sn = s_geo + kTile;  // normals at [d * kTile + j]
      double blk_re[NBT][NBS], blk_im[NBT][NBS];
      double S_re = 0.0, S_im = 0.0;  // sum_pq w_p w_q G (hypersingular curl term)
#pragma unroll
      for (int a = 0; a < NBT; ++a)
#pragma unroll
        for (int b = 0; b < NBS; ++b) blk_re[a][b] = blk_im[a][b] = 0.0;

      double bq[QT > 0 ? QT : kMaxRegularPoints];
      if (OP == kADL) {
#pragma unroll
        for (int q = 0; q < Q; ++q)
          bq[q] = s_pts[(3 * q) * kTile + j] * nxi + s_pts[(3 * q + 1) * kTile + j] * nyi +
                  s_pts[(3 * q + 2) * kTile + j] * nzi - h_i;
      }
      // For the hypersingular operator the factorised basis sum is only needed for the
      // Helmholtz normal-normal term.
      constexpr bool kNeedBasis = OP != kHS || KER == kHelmholtz;
#pragma unroll
      for (int p = 0; p < Q; ++p) {
        double ap = 1.0;
        if (OP == kDL)
          ap = tp.x[p] * sn[j] + tp.y[p] * sn[kTile + j] + tp.z[p] * sn[2 * kTile + j] -
               s_geo[4 * kTile + j];
        double u_re[NBS], u_im[NBS];
        double g_re = 0.0, g_im = 0.0;
#pragma unroll
        for (int b = 0; b < NBS; ++b) u_re[b] = u_im[b] = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const double dx = tp.x[p] - s_pts[(3 * q) * kTile + j];
          const double dy = tp.y[p] - s_pts[(3 * q + 1) * kTile + j];
          const double dz = tp.z[p] - s_pts[(3 * q + 2) * kTile + j];
          const double r2 = dx * dx + dy * dy + dz * dz;
          const double rinv = rsqrt(r2);
          double wq = rule.w[q];
          if (OP == kADL) wq *= bq[q];
          double kre, kim = 0.0;
          if (KER == kLaplace) {
            kre = (OP == kSL || OP == kHS) ? wq * rinv : wq * rinv * rinv * rinv;
          } else {
            const double r = r2 * rinv;
            double sn_, cs_;
            sincos(k * r, &sn_, &cs_);
            if (OP == kSL || OP == kHS) {
              const double f = wq * rinv;
              kre = f * cs_;
              kim = f * sn_;
            } else {
              const double f = wq * rinv * rinv * rinv;
              const double kr = k * r;
              kre = f * fma(kr, sn_, cs_);
              kim = f * fma(-kr, cs_, sn_);
            }
          }
          if (OP == kHS) {
            g_re += kre;
            if (kCplx) g_im += kim;
          }
          if (kNeedBasis) {
            if (NBS == 1) {
              u_re[0] += kre;
              if (kCplx) u_im[0] += kim;
            } else {
              const double x0 = rule.xi[2 * q], x1 = rule.xi[2 * q + 1];
              const double psi[3] = {1.0 - x0 - x1, x0, x1};
#pragma unroll
              for (int b = 0; b < NBS; ++b) {
                u_re[b] = fma(kre, psi[b], u_re[b]);
                if (kCplx) u_im[b] = fma(kim, psi[b], u_im[b]);
              }
            }
          }
        }
        const double wp = rule.w[p] * ap;
        if (OP == kHS) {
          S_re = fma(rule.w[p], g_re, S_re);
          if (kCplx) S_im = fma(rule.w[p], g_im, S_im);
        }
        if (kNeedBasis) {
          const double x0 = rule.xi[2 * p], x1 = rule.xi[2 * p + 1];
          const double phi[3] = {1.0 - x0 - x1, x0, x1};
#pragma unroll
          for (int a = 0; a < NBT; ++a) {
            const double f = NBT == 1 ? wp : wp * phi[a];
#pragma unroll
            for (int b = 0; b < NBS; ++b) {
              blk_re[a][b] = fma(f, u_re[b], blk_re[a][b]);
              if (kCplx) blk_im[a][b] = fma(f, u_im[b], blk_im[a][b]);
            }
          }
        }
      }
      const double jdet_j = s_geo[j];
      double out_re[NBT][NBS], out_im[NBT][NBS];
      if (OP != kHS) {
        const double sc = jdet_i * jdet_j * kInv4Pi;
#pragma unroll
        for (int a = 0; a < NBT; ++a)
#pragma unroll
          for (int b = 0; b < NBS; ++b) {
            out_re[a][b] = blk_re[a][b] * sc;
            out_im[a][b] = blk_im[a][b] * sc;
          }
      } else {
        // curls of the test and trial basis functions (zero for DP0)
        double ct[NBT][3], cs[NBS][3];
        const double* t0j = s_geo + 5 * kTile;
        const double* t1j = s_geo + 8 * kTile;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          if (NBT == 3) {
            ct[0][d] = t0i[d] - t1i[d];
            ct[1][d] = t1i[d];
            ct[2][d] = -t0i[d];
          } else {
            ct[0][d] = 0.0;
          }
          const double u0 = t0j[d * kTile + j], u1 = t1j[d * kTile + j];
          if (NBS == 3) {
            cs[0][d] = u0 - u1;
            cs[1][d] = u1;
            cs[2][d] = -u0;
          } else {
            cs[0][d] = 0.0;
          }
        }
        const double nn = nxi * sn[j] + nyi * sn[kTile + j] + nzi * sn[2 * kTile + j];
        const double nnsc = -k * k * nn * jdet_i * jdet_j;
#pragma unroll
        for (int a = 0; a < NBT; ++a)
#pragma unroll
          for (int b = 0; b < NBS; ++b) {
            const double cc = ct[a][0] * cs[b][0] + ct[a][1] * cs[b][1] + ct[a][2] * cs[b][2];
            double re = S_re * cc, im = S_im * cc;
            if (kCplx) {
              re = fma(nnsc, blk_re[a][b], re);
              im = fma(nnsc, blk_im[a][b], im);
            }
            out_re[a][b] = re * kInv4Pi;
            out_im[a][b] = im * kInv4Pi;
          }
      }
#pragma unroll
      for (int b = 0; b < NBS; ++b) {
        const int ls = s_int[(3 + b) * kTile + j];
#pragma unroll
        for (int a = 0; a < NBT; ++a) {
          const int idx = lt[a] + ndt * ls;
          atomicAdd(acc_re + idx, out_re[a][b]);
          if (kCplx) atomicAdd(acc_im + idx, out_im[a][b]);
        }
      }
    }
  }
  __syncthreads();
  const int* tdofs = tt.tile_dofs + tdof0;
  const int* sdofs = st.tile_dofs + sdof0;
  for (int idx = threadIdx.x; idx < ndt * nds; idx += kThreads) {
    const int a = idx % ndt, b = idx / ndt;
    const int64_t o = static_cast<int64_t>(sdofs[b]) * ld + tdofs[a];
    const double re = acc_re[idx];
    if (kCplx) {
      const double im = acc_im[idx];
      if (re != 0.0 || im != 0.0) {
        atomicAdd(out + 2 * o, re);
        atomicAdd(out + 2 * o + 1, im);
      }
    } else if (re != 0.0) {
      atomicAdd(out + o, re);
    }
  }
}

template <int QT, int KER, int OP, int NBT, int NBS>
cudaError_t launch_one(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                       const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                       cudaStream_t stream) {
  const size_t acc = static_cast<size_t>(tt.max_tile_dofs) * st.max_tile_dofs *
                     (KER == kHelmholtz ? 2 : 1) * sizeof(double);
  const size_t smem = acc + TrialSmem::doubles(rule.npts) * sizeof(double) +
                      TrialSmem::ints(NBS) * sizeof(int);
  auto fn = regular_scatter_fp64<QT, KER, OP, NBT, NBS>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  dim3 grid(tt.ntiles, st.ntiles);
  fn<<<grid, kThreads, smem, stream>>>(test, tt, trial, st, rule, a.k, a.same_grid,
                                       static_cast<double*>(a.out), a.ld);
  return cudaGetLastError();
}

template <int QT, int KER, int OP>
cudaError_t launch_nb(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                      const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                      cudaStream_t stream) {
  if (tt.nbasis == 1 && st.nbasis == 1)
    return launch_one<QT, KER, OP, 1, 1>(test, tt, trial, st, rule, a, stream);
  if (tt.nbasis == 1 && st.nbasis == 3)
    return launch_one<QT, KER, OP, 1, 3>(test, tt, trial, st, rule, a, stream);
  if (tt.nbasis == 3 && st.nbasis == 1)
    return launch_one<QT, KER, OP, 3, 1>(test, tt, trial, st, rule, a, stream);
  if (tt.nbasis == 3 && st.nbasis == 3)
    return launch_one<QT, KER, OP, 3, 3>(test, tt, trial, st, rule, a, stream);
  return cudaErrorInvalidValue;
}

template <int QT, int KER>
cudaError_t launch_op(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                      const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                      cudaStream_t stream) {
  switch (a.op) {
    case kSL: return launch_nb<QT, KER, kSL>(test, tt, trial, st, rule, a, stream);
    case kDL: return launch_nb<QT, KER, kDL>(test, tt, trial, st, rule, a, stream);
    case kADL: return launch_nb<QT, KER, kADL>(test, tt, trial, st, rule, a, stream);
    case kHS: return launch_nb<QT, KER, kHS>(test, tt, trial, st, rule, a, stream);
    default: return cudaErrorInvalidValue;
  }
}

template <int QT>
cudaError_t launch_q(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                     const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                     cudaStream_t stream) {
  return a.kernel == kLaplace ? launch_op<QT, kLaplace>(test, tt, trial, st, rule, a, stream)
                              : launch_op<QT, kHelmholtz>(test, tt, trial, st, rule, a, stream);
}

}  // namespace

cudaError_t launch_regular_scatter_mixed(const CellSet& test, const SpaceTiles& tt,
                                         const CellSet& trial, const SpaceTiles& st,
                                         const RegularRule& rule, const RegularArgs& a,
                                         cudaStream_t stream);

int scatter_tile_cells() { return kTile; }

cudaError_t launch_regular_scatter(const CellSet& test, const SpaceTiles& tt,
                                   const CellSet& trial, const SpaceTiles& st,
                                   const RegularRule& rule, const RegularArgs& a,
                                   cudaStream_t stream) {
  if (test.ncells <= 0 || trial.ncells <= 0) return cudaSuccess;
  if (tt.tile_cells != kTile || st.tile_cells != kTile) return cudaErrorInvalidValue;
  if (a.precision == kRegularMixed || a.out_type == kOutF32 || a.out_type == kOutC64)
    return launch_regular_scatter_mixed(test, tt, trial, st, rule, a, stream);
  if (rule.npts == 6) return launch_q<6>(test, tt, trial, st, rule, a, stream);
  return launch_q<0>(test, tt, trial, st, rule, a, stream);
}

}  // namespace bempp_b200
