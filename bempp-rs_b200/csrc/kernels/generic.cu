// Cell-pair quadrature for spaces of any Lagrange degree up to 2 (P2 / DP2 and their
// pairings with DP0 / P1 / DP1), FP64: one warp per cell pair, lanes over the points of
// the pair's rule, every basis pair accumulated per lane and reduced by shuffles.
//
// Restates the same cell-pair sums as the specialised regular and singular kernels
// (src/boundary_assemblers/cell_pair_assemblers.rs:109-152,283-339 with the integrands of
// src/boundary_assemblers/integrands/*.rs), with the basis tabulated at each point
// instead of P1 closed forms: entry[a][b] = sum_i w_i jdet_x jdet_y f(x_i, y_i, a, b) where
// the rule is the Q x Q tensor product of the regular rule (cell pairs that share no
// vertex) or the Duffy rule of the pair's adjacency configuration.  The hypersingular
// integrand uses the surface curls of the basis at each point,
//   curl phi_a . curl psi_b = [d0 phi d0 psi (t1x.t1y) - d0 phi d1 psi (t1x.t0y)
//                              - d1 phi d0 psi (t0x.t1y) + d1 phi d1 psi (t0x.t0y)]
//                             / (jdet_x jdet_y),
// and for Helmholtz subtracts k^2 (n_x.n_y) G phi_a psi_b (src/helmholtz.rs:98-104).
// Blocks are added into the zero-initialised dense output with atomics (or stored per
// pair for the CSR singular path).  This path serves the element degrees the tiled
// kernels are not specialised for; it is not tuned for speed.
#include "launch.h"

namespace bempp_b200 {
namespace {

constexpr int kThreads = 128;
constexpr int kWarpsPerBlock = kThreads / 32;

struct PairCell {
  double v0[3], t0[3], t1[3], n[3], jdet;
};

__device__ __forceinline__ void load_pair_cell(const CellSet& cs, int c, PairCell& d) {
  const int s = cs.stride;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    d.v0[k] = g(cs.geom, kV0x + k, s, c);
    d.t0[k] = g(cs.geom, kT0x + k, s, c);
    d.t1[k] = g(cs.geom, kT1x + k, s, c);
    d.n[k] = g(cs.geom, kNx + k, s, c);
  }
  d.jdet = g(cs.geom, kJdet, s, c);
}

// SING: the pairs are the singular list (Duffy rules), else every (test, trial) cell pair
// with trial cell in [trial_lo, trial_hi), vertex-sharing pairs skipped on one grid.
template <int KER, int OP, int NBT, int NBS, bool SING>
__global__ void __launch_bounds__(kThreads)
    pair_generic(CellSet test, const int* __restrict__ tdofs, CellSet trial,
                 const int* __restrict__ sdofs, RegularRule rule, SingularRules srules,
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
      const int s = test.stride;
      const int a0 = __ldg(test.vids + tc), a1 = __ldg(test.vids + s + tc),
                a2 = __ldg(test.vids + 2 * s + tc);
      const int b0 = __ldg(trial.vids + sc), b1 = __ldg(trial.vids + s + sc),
                b2 = __ldg(trial.vids + 2 * s + sc);
      if (share_vertex(a0, a1, a2, b0, b1, b2)) return;  // the singular part's pair
    }
    npts = rule.npts * rule.npts;
  }
  if (sc < trial_lo || sc >= trial_hi) return;  // warp-uniform
  PairCell x, y;
  load_pair_cell(test, tc, x);
  load_pair_cell(trial, sc, y);
  double tt[2][2];  // (t_i of x) . (t_j of y): t0 = index 0, t1 = index 1
  {
    const double* tx[2] = {x.t0, x.t1};
    const double* ty[2] = {y.t0, y.t1};
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
        tt[i][j] = tx[i][0] * ty[j][0] + tx[i][1] * ty[j][1] + tx[i][2] * ty[j][2];
  }
  const double inv_jj = 1.0 / (x.jdet * y.jdet);
  const double nn = x.n[0] * y.n[0] + x.n[1] * y.n[1] + x.n[2] * y.n[2];

  double acc_re[NBT][NBS], acc_im[NBT][NBS];
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b) acc_re[a][b] = acc_im[a][b] = 0.0;

  for (int ii = lane; ii < npts; ii += 32) {
    double xi0, xi1, et0, et1, wt;
    if (SING) {
      const int i = off + ii;
      xi0 = __ldg(srules.test_xi + 2 * i);
      xi1 = __ldg(srules.test_xi + 2 * i + 1);
      et0 = __ldg(srules.trial_xi + 2 * i);
      et1 = __ldg(srules.trial_xi + 2 * i + 1);
      wt = __ldg(srules.w + i);
    } else {
      const int p = ii / rule.npts, q = ii - p * rule.npts;
      xi0 = rule.xi[2 * p];
      xi1 = rule.xi[2 * p + 1];
      et0 = rule.xi[2 * q];
      et1 = rule.xi[2 * q + 1];
      wt = rule.w[p] * rule.w[q];
    }
    double d[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      d[c] = (x.v0[c] + xi0 * x.t0[c] + xi1 * x.t1[c]) - (y.v0[c] + et0 * y.t0[c] + et1 * y.t1[c]);
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double rinv = rsqrt_refined(r2);
    // kernel factor (without 1/(4 pi)): G for SL / HS, the normal derivative for DL / ADL
    double kre, kim = 0.0;
    double cs = 1.0, sn = 0.0, r = 0.0;
    if (kC) {
      r = r2 * rinv;
      sincos_cw(k * r, sn, cs);
    }
    if (OP == kSL || OP == kHS) {
      kre = rinv * cs;
      kim = rinv * sn;
    } else {
      const double dn = OP == kDL ? (d[0] * y.n[0] + d[1] * y.n[1] + d[2] * y.n[2])
                                  : -(d[0] * x.n[0] + d[1] * x.n[1] + d[2] * x.n[2]);
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
    double pv[NBT], p0[NBT], p1[NBT], sv[NBS], s0[NBS], s1[NBS];
    lagrange_basis<NBT>(xi0, xi1, pv, p0, p1);
    lagrange_basis<NBS>(et0, et1, sv, s0, s1);
#pragma unroll
    for (int a = 0; a < NBT; ++a)
#pragma unroll
      for (int b = 0; b < NBS; ++b) {
        double f;
        if (OP == kHS) {
          f = (p0[a] * s0[b] * tt[1][1] - p0[a] * s1[b] * tt[1][0] - p1[a] * s0[b] * tt[0][1] +
               p1[a] * s1[b] * tt[0][0]) * inv_jj;
          if (kC) f = fma(-k * k * nn, pv[a] * sv[b], f);
        } else {
          f = pv[a] * sv[b];
        }
        acc_re[a][b] = fma(kre, f, acc_re[a][b]);
        if (kC) acc_im[a][b] = fma(kim, f, acc_im[a][b]);
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
  const double sc4 = x.jdet * y.jdet * kInv4Pi;
  if (SING && pair_values) {
    double* pvv = pair_values + w * NBT * NBS * (kC ? 2 : 1);
#pragma unroll
    for (int b = 0; b < NBS; ++b)
#pragma unroll
      for (int a = 0; a < NBT; ++a) {
        const int e = a + NBT * b;
        if (kC) {
          pvv[2 * e] = acc_re[a][b] * sc4;
          pvv[2 * e + 1] = acc_im[a][b] * sc4;
        } else {
          pvv[e] = acc_re[a][b] * sc4;
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
        atomicAdd(out + 2 * o, acc_re[a][b] * sc4);
        atomicAdd(out + 2 * o + 1, acc_im[a][b] * sc4);
        if (mirror) {
          atomicAdd(out + 2 * om, acc_re[a][b] * sc4);
          atomicAdd(out + 2 * om + 1, acc_im[a][b] * sc4);
        }
      } else {
        atomicAdd(out + o, acc_re[a][b] * sc4);
        if (mirror) atomicAdd(out + om, acc_re[a][b] * sc4);
      }
    }
  }
}

template <int KER, int OP, int NBT, int NBS>
cudaError_t launch_pairs(const GenericPairArgs& g, cudaStream_t stream) {
  if (g.singular) {
    if (g.pairs.npairs <= 0) return cudaSuccess;
    const int blocks = (g.pairs.npairs + kWarpsPerBlock - 1) / kWarpsPerBlock;
    pair_generic<KER, OP, NBT, NBS, true><<<blocks, kThreads, 0, stream>>>(
        g.test, g.test_dofs, g.trial, g.trial_dofs, g.rule, g.rules, g.pairs, g.same_grid, g.k,
        static_cast<double*>(g.out), g.ld, g.trial_lo, g.trial_hi, g.pair_values, 0);
    return cudaGetLastError();
  }
  const int lo = g.trial_lo, hi = g.trial_hi < g.trial.ncells ? g.trial_hi : g.trial.ncells;
  if (hi <= lo || g.test.ncells <= 0) return cudaSuccess;
  const int64_t warps = static_cast<int64_t>(hi - lo) * g.test.ncells;
  const int64_t blocks = (warps + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
  pair_generic<KER, OP, NBT, NBS, false><<<static_cast<unsigned>(blocks), kThreads, 0, stream>>>(
      g.test, g.test_dofs, g.trial, g.trial_dofs, g.rule, g.rules, g.pairs, g.same_grid, g.k,
      static_cast<double*>(g.out), g.ld, lo, hi, nullptr, g.symmetric);
  return cudaGetLastError();
}

template <int KER, int OP>
cudaError_t launch_nb(const GenericPairArgs& g, cudaStream_t stream) {
  // pairings with a degree-2 side (the others have specialised kernels)
  switch (g.nbt * 10 + g.nbs) {
    case 16: return launch_pairs<KER, OP, 1, 6>(g, stream);
    case 36: return launch_pairs<KER, OP, 3, 6>(g, stream);
    case 61: return launch_pairs<KER, OP, 6, 1>(g, stream);
    case 63: return launch_pairs<KER, OP, 6, 3>(g, stream);
    case 66: return launch_pairs<KER, OP, 6, 6>(g, stream);
    default: return cudaErrorInvalidValue;
  }
}

template <int KER>
cudaError_t launch_op(const GenericPairArgs& g, cudaStream_t stream) {
  switch (g.op) {
    case kSL: return launch_nb<KER, kSL>(g, stream);
    case kDL: return launch_nb<KER, kDL>(g, stream);
    case kADL: return launch_nb<KER, kADL>(g, stream);
    case kHS: return launch_nb<KER, kHS>(g, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_generic_pairs(const GenericPairArgs& g, cudaStream_t stream) {
  return g.kernel == kLaplace ? launch_op<kLaplace>(g, stream) : launch_op<kHelmholtz>(g, stream);
}

}  // namespace bempp_b200
