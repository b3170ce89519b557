// Cell-pair quadrature on single-element quadrilateral grids, FP64: one warp per cell pair,
// lanes over the points of the pair's rule (the n x n Gauss tensor rule on both cells for
// pairs that share no vertex, else the Duffy rule of the pair's configuration), every
// basis pair accumulated per lane and reduced by shuffles, atomic adds into the
// zero-initialised dense output (or per-pair blocks for the CSR singular path).
//
// Degree-1 quadrilaterals are bilinear, x(s, t) = v0 (1-s)(1-t) + v1 s (1-t) + v2 (1-s) t
// + v3 s t (ndelement's vertex order), so the Jacobian columns J0 = dx/ds, J1 = dx/dt, the
// Jacobian determinant |J0 x J1| and the unit normal vary per point (the geometry map that
// bempp-rs takes from ndgrid, cell_pair_assemblers.rs:87-108): they are precomputed for
// every cell at the n x n regular points (quad_geometry_kernel, read back per point pair
// from L1 / L2) and formed at both points of every Duffy point pair.  The
// integrands are those of src/boundary_assemblers/integrands/*.rs; the hypersingular one
// uses the surface curl (J1 d0 phi - J0 d1 phi) / jdet, so that
//   jdet_x jdet_y curl phi_a . curl psi_b = (J1x d0 phi - J0x d1 phi) . (J1y d0 psi - J0y d1 psi),
// and for Helmholtz subtracts k^2 (n_x . n_y) G phi_a psi_b (src/helmholtz.rs:98-104).
// Bases: DP0 (one function) and Q1 (the tensor basis (1-s)(1-t), s(1-t), (1-s)t, st, one
// function per vertex in the vertex order).
#include "launch.h"

namespace bempp_b200 {
namespace {

constexpr int kThreads = 128;
constexpr int kWarpsPerBlock = kThreads / 32;

template <int NB>
__device__ __forceinline__ void quad_basis(double s, double t, double v[NB], double d0[NB],
                                           double d1[NB]) {
  if constexpr (NB == 1) {
    v[0] = 1.0;
    d0[0] = d1[0] = 0.0;
  } else {
    v[0] = (1.0 - s) * (1.0 - t); d0[0] = -(1.0 - t); d1[0] = -(1.0 - s);
    v[1] = s * (1.0 - t);         d0[1] = 1.0 - t;    d1[1] = -s;
    v[2] = (1.0 - s) * t;         d0[2] = -t;         d1[2] = 1.0 - s;
    v[3] = s * t;                 d0[3] = t;          d1[3] = s;
  }
}

struct QuadCell {
  double v[4][3];
};

__device__ __forceinline__ void load_quad(const QuadCells& qc, int c, QuadCell& q) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int p = __ldg(qc.cells + 4 * static_cast<int64_t>(c) + i);
#pragma unroll
    for (int d = 0; d < 3; ++d) q.v[i][d] = __ldg(qc.points + 3 * static_cast<int64_t>(p) + d);
  }
}

// point, Jacobian columns, normal and Jacobian determinant at reference point (s, t)
__device__ __forceinline__ void quad_point(const QuadCell& q, double s, double t, double x[3],
                                           double j0[3], double j1[3], double n[3],
                                           double& jdet) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    x[d] = q.v[0][d] * (1.0 - s) * (1.0 - t) + q.v[1][d] * s * (1.0 - t) +
           q.v[2][d] * (1.0 - s) * t + q.v[3][d] * s * t;
    j0[d] = (q.v[1][d] - q.v[0][d]) * (1.0 - t) + (q.v[3][d] - q.v[2][d]) * t;
    j1[d] = (q.v[2][d] - q.v[0][d]) * (1.0 - s) + (q.v[3][d] - q.v[1][d]) * s;
  }
  const double cx = j0[1] * j1[2] - j0[2] * j1[1], cy = j0[2] * j1[0] - j0[0] * j1[2],
               cz = j0[0] * j1[1] - j0[1] * j1[0];
  jdet = sqrt(cx * cx + cy * cy + cz * cz);
  const double inv = 1.0 / jdet;
  n[0] = cx * inv;
  n[1] = cy * inv;
  n[2] = cz * inv;
}

// Geometry of every cell at the n x n regular points: field f of point p of cell c at
// out[f * ncells * n^2 + c * n^2 + p]; fields x (3), jdet, unit normal (3), J0 (3), J1 (3).
__global__ void __launch_bounds__(256)
    quad_geometry_kernel(QuadCells cells, QuadGaussRule rule, double* __restrict__ out) {
  const int m = rule.n * rule.n;
  const int64_t total = static_cast<int64_t>(cells.ncells) * m;
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int c = static_cast<int>(i / m), p = static_cast<int>(i - static_cast<int64_t>(c) * m);
  QuadCell q;
  load_quad(cells, c, q);
  double x[3], j0[3], j1[3], n[3], jdet;
  quad_point(q, rule.x[p / rule.n], rule.x[p % rule.n], x, j0, j1, n, jdet);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    out[d * total + i] = x[d];
    out[(4 + d) * total + i] = n[d];
    out[(7 + d) * total + i] = j0[d];
    out[(10 + d) * total + i] = j1[d];
  }
  out[3 * total + i] = jdet;
}

template <int KER, int OP, int NBT, int NBS, bool SING>
__global__ void __launch_bounds__(kThreads)
    quad_pairs(QuadCells test, const int* __restrict__ tdofs, QuadCells trial,
               const int* __restrict__ sdofs, QuadGaussRule rule, SingularRules srules,
               SingularPairs pairs, int same_grid, double k, double* __restrict__ out,
               int64_t ld, int trial_lo, int trial_hi, double* __restrict__ pair_values,
               int symmetric) {
  constexpr bool kC = KER == kHelmholtz;
  const int lane = threadIdx.x & 31;
  const int64_t w = static_cast<int64_t>(blockIdx.x) * kWarpsPerBlock + (threadIdx.x >> 5);
  int tc, sc, off = 0, npts;
  if (SING) {
    if (w >= pairs.npairs) return;
    tc = __ldg(pairs.test_cell + w);
    sc = __ldg(pairs.trial_cell + w);
    const int cfg = __ldg(pairs.config + w);
    off = __ldg(srules.offset + cfg);
    npts = __ldg(srules.offset + cfg + 1) - off;
  } else {
    const int64_t span = static_cast<int64_t>(trial_hi - trial_lo);
    if (w >= span * test.ncells) return;
    tc = static_cast<int>(w % test.ncells);
    sc = trial_lo + static_cast<int>(w / test.ncells);
    // one space and a symmetric operator: the pair (tc, sc) also gives (sc, tc)
    if (symmetric && tc < sc) return;
    if (same_grid) {
      bool shared = false;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          shared |= __ldg(test.vids + 4 * static_cast<int64_t>(tc) + i) ==
                    __ldg(trial.vids + 4 * static_cast<int64_t>(sc) + j);
      if (shared) return;  // the singular part's pair
    }
    npts = rule.n * rule.n * rule.n * rule.n;
  }
  if (sc < trial_lo || sc >= trial_hi) return;  // warp-uniform
  QuadCell X, Y;
  if (SING) {
    load_quad(test, tc, X);
    load_quad(trial, sc, Y);
  }

  double acc_re[NBT][NBS], acc_im[NBT][NBS];
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b) acc_re[a][b] = acc_im[a][b] = 0.0;

  // fields of the precomputed regular points each operator reads
  constexpr bool kXN = OP == kADL || (OP == kHS && kC);
  constexpr bool kYN = OP == kDL || (OP == kHS && kC);
  constexpr bool kJ = OP == kHS;
  const int m = rule.n * rule.n;  // regular points per cell
  const int64_t tstride = static_cast<int64_t>(test.ncells) * m;
  const int64_t sstride = static_cast<int64_t>(trial.ncells) * m;
  // regular part: the lane's point pair ii = p * m + q is stepped by 32 without dividing,
  // and a point index splits into its (s, t) Gauss indices by an exact FP32 product
  // (indices below 256, so (i + 0.5) / n never rounds across an integer)
  int p = lane / m, q = lane - (lane / m) * m;
  const int dp = 32 / m, dq = 32 - dp * m;
  const float inv_n = 1.f / static_cast<float>(rule.n);
  for (int ii = lane; ii < npts; ii += 32) {
    double xs, xt, ys, yt, wt;
    double x[3], xj0[3], xj1[3], xn[3], xjd, y[3], yj0[3], yj1[3], yn[3], yjd;
    if (SING) {
      const int i = off + ii;
      xs = __ldg(srules.test_xi + 2 * i);
      xt = __ldg(srules.test_xi + 2 * i + 1);
      ys = __ldg(srules.trial_xi + 2 * i);
      yt = __ldg(srules.trial_xi + 2 * i + 1);
      wt = __ldg(srules.w + i);
      quad_point(X, xs, xt, x, xj0, xj1, xn, xjd);
      quad_point(Y, ys, yt, y, yj0, yj1, yn, yjd);
    } else {
      // ii = test point * m + trial point; point p = (s index) * n + (t index)
      const int n = rule.n;
      const int p0 = static_cast<int>((static_cast<float>(p) + 0.5f) * inv_n), p1 = p - p0 * n;
      const int q0 = static_cast<int>((static_cast<float>(q) + 0.5f) * inv_n), q1 = q - q0 * n;
      xs = rule.x[p0];
      xt = rule.x[p1];
      ys = rule.x[q0];
      yt = rule.x[q1];
      wt = rule.w[p0] * rule.w[p1] * rule.w[q0] * rule.w[q1];
      const double* tg = test.qgeom + static_cast<int64_t>(tc) * m + p;
      const double* sg = trial.qgeom + static_cast<int64_t>(sc) * m + q;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        x[c] = __ldg(tg + c * tstride);
        y[c] = __ldg(sg + c * sstride);
        if (kXN) xn[c] = __ldg(tg + (4 + c) * tstride);
        if (kYN) yn[c] = __ldg(sg + (4 + c) * sstride);
        if (kJ) {
          xj0[c] = __ldg(tg + (7 + c) * tstride);
          xj1[c] = __ldg(tg + (10 + c) * tstride);
          yj0[c] = __ldg(sg + (7 + c) * sstride);
          yj1[c] = __ldg(sg + (10 + c) * sstride);
        }
      }
      xjd = __ldg(tg + 3 * tstride);
      yjd = __ldg(sg + 3 * sstride);
    }
    const double d[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double rinv = rsqrt_refined(r2);
    double cs = 1.0, sn = 0.0, r = 0.0;
    if (kC) {
      r = r2 * rinv;
      sincos_cw(k * r, sn, cs);
    }
    // kernel factor (without 1/(4 pi)) times the weight
    double kre, kim = 0.0;
    if (OP == kSL || OP == kHS) {
      kre = rinv * cs;
      kim = rinv * sn;
    } else {
      const double dn = OP == kDL ? (d[0] * yn[0] + d[1] * yn[1] + d[2] * yn[2])
                                  : -(d[0] * xn[0] + d[1] * xn[1] + d[2] * xn[2]);
      const double f = dn * rinv * rinv * rinv;
      if (kC) {
        const double kr = k * r;
        kre = f * fma(kr, sn, cs);
        kim = f * fma(-kr, cs, sn);
      } else {
        kre = f;
      }
    }
    kre *= wt;
    kim *= wt;
    const double jj = xjd * yjd;
    double pv[NBT], p0[NBT], p1[NBT], sv[NBS], s0[NBS], s1[NBS];
    quad_basis<NBT>(xs, xt, pv, p0, p1);
    quad_basis<NBS>(ys, yt, sv, s0, s1);
    const double nn = xn[0] * yn[0] + xn[1] * yn[1] + xn[2] * yn[2];
#pragma unroll
    for (int a = 0; a < NBT; ++a)
#pragma unroll
      for (int b = 0; b < NBS; ++b) {
        double f;
        if (OP == kHS) {
          f = 0.0;
#pragma unroll
          for (int c = 0; c < 3; ++c)
            f = fma(xj1[c] * p0[a] - xj0[c] * p1[a], yj1[c] * s0[b] - yj0[c] * s1[b], f);
          if (kC) f = fma(-k * k * nn * jj, pv[a] * sv[b], f);
        } else {
          f = pv[a] * sv[b] * jj;
        }
        acc_re[a][b] = fma(kre, f, acc_re[a][b]);
        if (kC) acc_im[a][b] = fma(kim, f, acc_im[a][b]);
      }
    if (!SING) {
      p += dp;
      q += dq;
      if (q >= m) {
        q -= m;
        ++p;
      }
    }
  }
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b)
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) {
        acc_re[a][b] += __shfl_xor_sync(0xffffffffu, acc_re[a][b], s);
        if (kC) acc_im[a][b] += __shfl_xor_sync(0xffffffffu, acc_im[a][b], s);
      }
  if (lane != 0) return;
  if (SING && pair_values) {
    double* pvv = pair_values + w * NBT * NBS * (kC ? 2 : 1);
#pragma unroll
    for (int b = 0; b < NBS; ++b)
#pragma unroll
      for (int a = 0; a < NBT; ++a) {
        const int e = a + NBT * b;
        if (kC) {
          pvv[2 * e] = acc_re[a][b] * kInv4Pi;
          pvv[2 * e + 1] = acc_im[a][b] * kInv4Pi;
        } else {
          pvv[e] = acc_re[a][b] * kInv4Pi;
        }
      }
  }
  if (!out) return;
#pragma unroll
  for (int b = 0; b < NBS; ++b) {
    const int64_t col = static_cast<int64_t>(__ldg(sdofs + static_cast<int64_t>(sc) * NBS + b)) * ld;
#pragma unroll
    for (int a = 0; a < NBT; ++a) {
      const int64_t o = col + __ldg(tdofs + static_cast<int64_t>(tc) * NBT + a);
      // the transposed entry: test cell sc's function b against trial cell tc's function a
      const int64_t om = static_cast<int64_t>(__ldg(sdofs + static_cast<int64_t>(tc) * NBS + a)) * ld +
                         __ldg(tdofs + static_cast<int64_t>(sc) * NBT + b);
      const bool mirror = !SING && symmetric && tc > sc;
      if (kC) {
        atomicAdd(out + 2 * o, acc_re[a][b] * kInv4Pi);
        atomicAdd(out + 2 * o + 1, acc_im[a][b] * kInv4Pi);
        if (mirror) {
          atomicAdd(out + 2 * om, acc_re[a][b] * kInv4Pi);
          atomicAdd(out + 2 * om + 1, acc_im[a][b] * kInv4Pi);
        }
      } else {
        atomicAdd(out + o, acc_re[a][b] * kInv4Pi);
        if (mirror) atomicAdd(out + om, acc_re[a][b] * kInv4Pi);
      }
    }
  }
}

template <int KER, int OP, int NBT, int NBS>
cudaError_t launch_pairs(const QuadPairArgs& g, cudaStream_t stream) {
  if (g.singular) {
    if (g.pairs.npairs <= 0) return cudaSuccess;
    const int blocks = (g.pairs.npairs + kWarpsPerBlock - 1) / kWarpsPerBlock;
    quad_pairs<KER, OP, NBT, NBS, true><<<blocks, kThreads, 0, stream>>>(
        g.test, g.test_dofs, g.trial, g.trial_dofs, g.rule, g.rules, g.pairs, g.same_grid, g.k,
        static_cast<double*>(g.out), g.ld, g.trial_lo, g.trial_hi, g.pair_values, 0);
    return cudaGetLastError();
  }
  const int lo = g.trial_lo, hi = g.trial_hi < g.trial.ncells ? g.trial_hi : g.trial.ncells;
  if (hi <= lo || g.test.ncells <= 0) return cudaSuccess;
  const int64_t warps = static_cast<int64_t>(hi - lo) * g.test.ncells;
  const int64_t blocks = (warps + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
  quad_pairs<KER, OP, NBT, NBS, false><<<static_cast<unsigned>(blocks), kThreads, 0, stream>>>(
      g.test, g.test_dofs, g.trial, g.trial_dofs, g.rule, g.rules, g.pairs, g.same_grid, g.k,
      static_cast<double*>(g.out), g.ld, lo, hi, nullptr, g.symmetric);
  return cudaGetLastError();
}

template <int KER, int OP>
cudaError_t launch_nb(const QuadPairArgs& g, cudaStream_t stream) {
  switch (g.nbt * 10 + g.nbs) {
    case 11: return launch_pairs<KER, OP, 1, 1>(g, stream);
    case 14: return launch_pairs<KER, OP, 1, 4>(g, stream);
    case 41: return launch_pairs<KER, OP, 4, 1>(g, stream);
    case 44: return launch_pairs<KER, OP, 4, 4>(g, stream);
    default: return cudaErrorInvalidValue;
  }
}

template <int KER>
cudaError_t launch_op(const QuadPairArgs& g, cudaStream_t stream) {
  switch (g.op) {
    case kSL: return launch_nb<KER, kSL>(g, stream);
    case kDL: return launch_nb<KER, kDL>(g, stream);
    case kADL: return launch_nb<KER, kADL>(g, stream);
    case kHS: return launch_nb<KER, kHS>(g, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_quad_geometry(const QuadCells& cells, const QuadGaussRule& rule, double* out,
                                 cudaStream_t stream) {
  const int64_t total = static_cast<int64_t>(cells.ncells) * rule.n * rule.n;
  if (total <= 0) return cudaSuccess;
  const int64_t blocks = (total + 255) / 256;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
  quad_geometry_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(cells, rule, out);
  return cudaGetLastError();
}

cudaError_t launch_quad_pairs(const QuadPairArgs& g, cudaStream_t stream) {
  return g.kernel == kLaplace ? launch_op<kLaplace>(g, stream) : launch_op<kHelmholtz>(g, stream);
}

}  // namespace bempp_b200
