// Regular (non-singular) quadrature of all operators and space pairs, FP64 or mixed.
//
// Replaces the hot loop of bempp-rs assemble_nonsingular_part / assemble_batch_nonadjacent
// (src/boundary_assemblers.rs:396-521,689-773) and NonsingularCellPairAssemblerWithTest-
// Caching::assemble (src/boundary_assemblers/cell_pair_assemblers.rs:283-339) with the
// integrands of src/boundary_assemblers/integrands/*.rs: entry[a][b] of a cell pair is
// sum_p sum_q w_p w_q jdet_x jdet_y f(x_p, y_q) phi_a(p) psi_b(q), vertex-sharing pairs
// are left to the singular kernel (src/boundary_assemblers.rs:754-756), and the Helmholtz
// hypersingular operator is curl-curl - k^2 normal-normal (src/helmholtz.rs:98-104).
//
// Mapping.  A CTA of 4 warps owns a tile of 32 test cells x 32 trial cells; both tiles
// (quadrature points and per-cell geometry) are staged once in shared memory.  Lane l
// handles test cell l of the tile and reads its points from its own shared-memory column;
// warp w handles trial cells w, w+4, ..., read as warp-wide broadcasts.  Per pair the
// point loop is factorised: U_b(p) = sum_q K(x_p, y_q) psi_b(q) w_q and block[a][b] =
// sum_p phi_a(p) w_p U_b(p).
//   DIRECT  (DP0 x DP0, single/double/adjoint double layer): each thread stores its
//           entries; consecutive lanes write consecutive rows of a column (coalesced).
//   SCATTER (any other pair of spaces): local blocks are added with shared-memory atomics
//           into a matrix over the DOFs the two tiles touch, flushed once per CTA with
//           global atomic adds into the zero-initialised output.  The reference avoids
//           races by cell colouring (src/function.rs:281-351) instead.
//
// Mixed precision.  A pair is near when |c_x - c_y| < 2 max(diam_x, diam_y) (centroids,
// longest edges, decided in FP64).  Near pairs are queued in shared memory and integrated
// in FP64 after the main loop, so the hot loop carries FP32 code only.  Far pairs:
//   * centroid-relative coordinates d_pq = dc + (dx_p - dy_q), dc = c_x - c_y rounded
//     once from FP64, dx_p, dy_q stored in FP32;
//   * the normal-derivative factors in the cells' tangent coordinates, x_p - c_x =
//     u_p t0 + v_p t1 with (u_p, v_p) = xi_p - (1/3, 1/3), every dot product formed in
//     FP64 once per pair: (x_p - y_q).n_y = dc.n_y + u_p t0_x.n_y + v_p t1_x.n_y, so no
//     FP32 cancellation for nearly coplanar pairs;
//   * s_pq = |d_pq|^2 - |dc|^2 = 2 dc.D + D.D, D = dx_p - dy_q, free of cancellation,
//     evaluated as A_p + |dy_q|^2 + w_p.dy_q with A_p = |dx_p|^2 + 2 dc.dx_p and
//     w_p = -2 (dc + dx_p) formed once per test point (4 operations per point pair);
//     Laplace: r^2 = |dc|^2 + s_pq;
//   * Helmholtz: e^{ikr} = e^{ik r0} e^{ik delta}, r0 = |dc| in FP64, delta = r - r0 =
//     s_pq / (r + r0); e^{ik delta} from minimax polynomials of cos / sin on |t| <= 0.8
//     (degree 8 / 7) when |k delta| <= k (rad_x + rad_y) <= 0.8 holds for every lane of
//     the warp, else the same polynomials after a Cody-Waite reduction by pi/2;
//     e^{ik r0} from the same polynomials after an FP64 reduction of k r0 by pi/2;
//   * DP0 entries sum their 6 inner sums with Kahan compensation; P1 blocks are formed
//     in FP32 and accumulated into the matrix in FP64.
#include "launch.h"
#include <algorithm>

#include "tiles.cuh"

namespace bempp_b200 {
namespace {

constexpr float kSmallPhaseMax = 0.8f;
constexpr float kWidePhaseMax = 1.6f;

// Blocks whose tile copies did not complete within the bounded wait (never expected).
__device__ unsigned g_stage_timeouts = 0;
// Polls of a block's first wait for its tile copies.  Tests lower it to make that wait
// run out; the second wait, which drains the copies before the block returns, always
// polls kStagePolls times.
__device__ int g_stage_poll_limit = tiles::kStagePolls;
using namespace tiles;

// Curls of the basis functions of a flat cell: t1 d0(phi) - t0 d1(phi); zero for DP0.
template <int NB>
__device__ __forceinline__ void curls(const Tile& t, int c, double cu[NB][3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double u0 = t.G(fT0x + d, c), u1 = t.G(fT1x + d, c);
    if (NB == 3) {
      cu[0][d] = u0 - u1;
      cu[1][d] = u1;
      cu[2][d] = -u0;
    } else {
      cu[0][d] = 0.0;
    }
  }
}

// Final scaling of a pair's sums into the local block (shared by both precisions).
// blk: sum_p w_p phi_a(p) sum_q w_q psi_b(q) K_pq (times the DL/ADL factors);
// S: sum_pq w_p w_q G (hypersingular only).
template <int KER, int OP, int NBT, int NBS>
__device__ __forceinline__ void finish_block(const Tile& T, int it, const Tile& S, int js, double k,
                                             const double blk_re[NBT][NBS],
                                             const double blk_im[NBT][NBS], double S_re,
                                             double S_im, double ore[NBT][NBS],
                                             double oim[NBT][NBS]) {
  const double jj = T.G(fJdet, it) * S.G(fJdet, js);
  if constexpr (OP != kHS) {
    const double sc = jj * kInv4Pi;
#pragma unroll
    for (int a = 0; a < NBT; ++a)
#pragma unroll
      for (int b = 0; b < NBS; ++b) {
        ore[a][b] = blk_re[a][b] * sc;
        oim[a][b] = blk_im[a][b] * sc;
      }
  } else {
    double ct[NBT][3], cs[NBS][3];
    curls<NBT>(T, it, ct);
    curls<NBS>(S, js, cs);
    const double nn = T.G(fNx, it) * S.G(fNx, js) + T.G(fNy, it) * S.G(fNy, js) +
                      T.G(fNz, it) * S.G(fNz, js);
    const double nnsc = -k * k * nn * jj;
#pragma unroll
    for (int a = 0; a < NBT; ++a)
#pragma unroll
      for (int b = 0; b < NBS; ++b) {
        const double cc = ct[a][0] * cs[b][0] + ct[a][1] * cs[b][1] + ct[a][2] * cs[b][2];
        double re = S_re * cc, im = S_im * cc;
        if (KER == kHelmholtz) {
          re = fma(nnsc, blk_re[a][b], re);
          im = fma(nnsc, blk_im[a][b], im);
        }
        ore[a][b] = re * kInv4Pi;
        oim[a][b] = im * kInv4Pi;
      }
  }
}

// How an FP64 Helmholtz block forms e^{ikr}: CUDA's sincos (any phase), the in-tree
// Cody-Waite sincos_cw (the FP64 near pairs of mixed assemblies), or referenced to the
// pair, e^{ikr} = e^{ik r0} e^{ik (r - r0)} with r0 = |c_x - c_y|: e^{ik r0} once per pair
// and e^{ik (r - r0)} from the Taylor series of sincos_small, valid when
// k (rad_x + rad_y) <= 0.8 bounds every |k (r - r0)| (checked on the host).
enum F64Phase : int { kF64Sincos = 0, kF64Reduced = 1, kF64Referenced = 2 };

// FP64 local block, test points outermost (every operator but the Laplace adjoint double
// layer).
template <int QT, int KER, int OP, int NBT, int NBS, bool kUnroll, int FPH>
__device__ __forceinline__ void block_fp64_pq(const Tile& T, int it, const Tile& S, int js,
                                        const RegularRule& rule, double k,
                                        double ore[NBT][NBS], double oim[NBT][NBS]) {
  constexpr bool kC = KER == kHelmholtz;
  constexpr bool kNeedBasis = OP != kHS || kC;
  const int Q = QT > 0 ? QT : rule.npts;
  double blk_re[NBT][NBS], blk_im[NBT][NBS];
  double S_re = 0.0, S_im = 0.0;
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b) blk_re[a][b] = blk_im[a][b] = 0.0;
  // normal-derivative factors in the cells' tangent coordinates, free of the cancellation
  // of x.n - h far from the origin: with dc = c_x - c_y and (u, v) = xi - (1/3, 1/3),
  // DL (x_p - y).n_y = dc.n_y + u_p t0_x.n_y + v_p t1_x.n_y (y on the trial plane),
  // ADL (y_q - x).n_x = -dc.n_x + u_q t0_y.n_x + v_q t1_y.n_x (x on the test plane)
  double f0 = 0.0, f1 = 0.0, f2 = 0.0;
  if (OP == kDL || OP == kADL) {
    const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
                 dcz = T.G(fCz, it) - S.G(fCz, js);
    const Tile& N = OP == kDL ? S : T;    // the cell whose normal is used
    const Tile& D = OP == kDL ? T : S;    // the cell whose tangents are used
    const int cn = OP == kDL ? js : it, cd = OP == kDL ? it : js;
    const double nx = N.G(fNx, cn), ny = N.G(fNy, cn), nz = N.G(fNz, cn);
    f0 = (OP == kDL ? 1.0 : -1.0) * (dcx * nx + dcy * ny + dcz * nz);
    f1 = D.G(fT0x, cd) * nx + D.G(fT0y, cd) * ny + D.G(fT0z, cd) * nz;
    f2 = D.G(fT1x, cd) * nx + D.G(fT1y, cd) * ny + D.G(fT1z, cd) * nz;
  }
  // reference distance of the pair and its phase (kF64Referenced)
  double kr0 = 0.0, ph_c = 1.0, ph_s = 0.0;
  if (kC && FPH == kF64Referenced) {
    const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
                 dcz = T.G(fCz, it) - S.G(fCz, js);
    const double r0sq = dcx * dcx + dcy * dcy + dcz * dcz;
    kr0 = k * (r0sq * rsqrt_refined(r0sq));
    sincos_cw(kr0, ph_s, ph_c);
  }
#pragma unroll 1
  for (int p = 0; p < Q; ++p) {
    const double x0 = T.P(p, 0, it), x1 = T.P(p, 1, it), x2 = T.P(p, 2, it);
    const double ap = OP == kDL ? fma(rule.u[p], f1, fma(rule.v[p], f2, f0)) : 1.0;
    double u_re[NBS], u_im[NBS], g_re = 0.0, g_im = 0.0;
#pragma unroll
    for (int b = 0; b < NBS; ++b) u_re[b] = u_im[b] = 0.0;
#pragma unroll(kUnroll ? 6 : 1)
    for (int q = 0; q < Q; ++q) {
      const double y0 = S.P(q, 0, js), y1 = S.P(q, 1, js), y2 = S.P(q, 2, js);
      const double dx = x0 - y0, dy = x1 - y1, dz = x2 - y2;
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (KER == kLaplace) {
        // 1/r or 1/r^3 straight from the refined hardware seed; the weight (times the
        // basis value for P1) enters as a rule constant of the accumulating FMA
        double kern = (OP == kSL || OP == kHS) ? rsqrt_refined(r2) : rinv3_refined(r2);
        if (OP == kADL) kern *= fma(rule.u[q], f1, fma(rule.v[q], f2, f0));
        if (OP == kHS) {
          g_re = fma(kern, rule.w[q], g_re);
        } else if (NBS == 1) {
          u_re[0] = fma(kern, rule.w[q], u_re[0]);
        } else {
#pragma unroll
          for (int b = 0; b < NBS; ++b) u_re[b] = fma(kern, rule_wphi<NBS>(rule, b, q), u_re[b]);
        }
        continue;
      }
      const double rinv = rsqrt_refined(r2);
      double wq = rule.w[q];
      if (OP == kADL) wq *= fma(rule.u[q], f1, fma(rule.v[q], f2, f0));
      double kre, kim = 0.0;
      {
        const double r = r2 * rinv;
        double sn, cs;
        if (FPH == kF64Referenced)
          sincos_small(fma(k, r, -kr0), sn, cs);  // e^{ik (r - r0)}
        else if (FPH == kF64Reduced)
          sincos_cw(k * r, sn, cs);
        else
          sincos(k * r, &sn, &cs);
        if (OP == kSL || OP == kHS) {
          const double f = wq * rinv;
          kre = f * cs;
          kim = f * sn;
        } else {
          const double f = wq * rinv * rinv * rinv, kr = k * r;
          kre = f * fma(kr, sn, cs);
          kim = f * fma(-kr, cs, sn);
        }
      }
      if (OP == kHS) {
        g_re += kre;
        if (kC) g_im += kim;
      }
      if (kNeedBasis) {
        if (NBS == 1) {
          u_re[0] += kre;
          if (kC) u_im[0] += kim;
        } else {
#pragma unroll
          for (int b = 0; b < NBS; ++b) {
            u_re[b] = fma(kre, rule_phi<NBS>(rule, b, q), u_re[b]);
            if (kC) u_im[b] = fma(kim, rule_phi<NBS>(rule, b, q), u_im[b]);
          }
        }
      }
    }
    if (OP == kHS) {
      S_re = fma(rule.w[p], g_re, S_re);
      if (kC) S_im = fma(rule.w[p], g_im, S_im);
    }
    if (kNeedBasis) {
      const double wp = rule.w[p] * ap;
#pragma unroll
      for (int a = 0; a < NBT; ++a) {
        const double f = NBT == 1 ? wp : wp * rule_phi<NBT>(rule, a, p);
#pragma unroll
        for (int b = 0; b < NBS; ++b) {
          blk_re[a][b] = fma(f, u_re[b], blk_re[a][b]);
          if (kC) blk_im[a][b] = fma(f, u_im[b], blk_im[a][b]);
        }
      }
    }
  }
  if (kC && FPH == kF64Referenced) {
    // apply the pair's reference phase e^{ik r0}
    const double re = S_re * ph_c - S_im * ph_s, im = S_re * ph_s + S_im * ph_c;
    S_re = re;
    S_im = im;
#pragma unroll
    for (int a = 0; a < NBT; ++a)
#pragma unroll
      for (int b = 0; b < NBS; ++b) {
        const double br = blk_re[a][b] * ph_c - blk_im[a][b] * ph_s;
        const double bi = blk_re[a][b] * ph_s + blk_im[a][b] * ph_c;
        blk_re[a][b] = br;
        blk_im[a][b] = bi;
      }
  }
  finish_block<KER, OP, NBT, NBS>(T, it, S, js, k, blk_re, blk_im, S_re, S_im, ore, oim);
}

// Laplace adjoint double layer, FP64: the normal factor (y_q - x).n_x depends on the trial
// point only, so the trial points are the outer loop and the factor multiplies once per
// trial point (as the double layer's does per test point in block_fp64_pq).
template <int QT, int NBT, int NBS, bool kUnroll>
__device__ __forceinline__ void block_fp64_adl_laplace(const Tile& T, int it, const Tile& S,
                                                       int js, const RegularRule& rule,
                                                       double ore[NBT][NBS], double oim[NBT][NBS]) {
  const int Q = QT > 0 ? QT : rule.npts;
  double blk_re[NBT][NBS], blk_im[NBT][NBS];
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b) blk_re[a][b] = blk_im[a][b] = 0.0;
  // (y_q - x).n_x = -dc.n_x + u_q t0_y.n_x + v_q t1_y.n_x, (u, v) = eta - (1/3, 1/3)
  const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
               dcz = T.G(fCz, it) - S.G(fCz, js);
  const double nx = T.G(fNx, it), ny = T.G(fNy, it), nz = T.G(fNz, it);
  const double f0 = -(dcx * nx + dcy * ny + dcz * nz);
  const double f1 = S.G(fT0x, js) * nx + S.G(fT0y, js) * ny + S.G(fT0z, js) * nz;
  const double f2 = S.G(fT1x, js) * nx + S.G(fT1y, js) * ny + S.G(fT1z, js) * nz;
#pragma unroll 1
  for (int q = 0; q < Q; ++q) {
    const double y0 = S.P(q, 0, js), y1 = S.P(q, 1, js), y2 = S.P(q, 2, js);
    const double bq = fma(rule.u[q], f1, fma(rule.v[q], f2, f0));
    double v[NBT];
#pragma unroll
    for (int a = 0; a < NBT; ++a) v[a] = 0.0;
#pragma unroll(kUnroll ? 6 : 1)
    for (int p = 0; p < Q; ++p) {
      const double dx = T.P(p, 0, it) - y0, dy = T.P(p, 1, it) - y1, dz = T.P(p, 2, it) - y2;
      const double kern = rinv3_refined(dx * dx + dy * dy + dz * dz);
      if (NBT == 1) {
        v[0] = fma(kern, rule.w[p], v[0]);
      } else {
#pragma unroll
        for (int a = 0; a < NBT; ++a) v[a] = fma(kern, rule_wphi<NBT>(rule, a, p), v[a]);
      }
    }
#pragma unroll
    for (int b = 0; b < NBS; ++b) {
      const double f = rule_wphi<NBS>(rule, b, q) * bq;
#pragma unroll
      for (int a = 0; a < NBT; ++a) blk_re[a][b] = fma(v[a], f, blk_re[a][b]);
    }
  }
  finish_block<kLaplace, kADL, NBT, NBS>(T, it, S, js, 0.0, blk_re, blk_im, 0.0, 0.0, ore, oim);
}

// FP64 local block of test cell `it` (tile T) and trial cell `js` (tile S); FPH: how the
// Helmholtz phase is formed (F64Phase).
template <int QT, int KER, int OP, int NBT, int NBS, bool kUnroll = true, int FPH = kF64Sincos>
__device__ __forceinline__ void block_fp64(const Tile& T, int it, const Tile& S, int js,
                                        const RegularRule& rule, double k,
                                        double ore[NBT][NBS], double oim[NBT][NBS]) {
  if constexpr (KER == kLaplace && OP == kADL)
    block_fp64_adl_laplace<QT, NBT, NBS, kUnroll>(T, it, S, js, rule, ore, oim);
  else
    block_fp64_pq<QT, KER, OP, NBT, NBS, kUnroll, FPH>(T, it, S, js, rule, k, ore, oim);
}

// Laplace double layer of a cell pair in both orders, FP64, for one P1 / DP1 space on both
// sides (the same rule on both cells): from one 1/r^3 per point pair (x_p in cell i of the
// test tile, y_q in cell j of the trial tile)
//   dij[a][b] = DL(test i, trial j)_ab = sum_p w_p phi_a(p) (x_p - y).n_j sum_q w_q phi_b(q) / r^3
//   dji[a][b] = DL(test j, trial i)_ba = sum_p w_p phi_a(p) sum_q w_q phi_b(q) (y_q - x).n_i / r^3
// ((x - y).n is constant over the plane of the normal's cell, in the tangent coordinates of
// block_fp64_pq).  Both trial-point sums close per test point; the reverse order's normal
// factor is formed per point pair (3 FP64 operations), which keeps 15 fewer doubles live
// than summing per trial point and applying it at the end (8 % faster at 20,480 cells).
// The adjoint double layer is the same pair of blocks swapped: ADL(i, j)_ab = DL(j, i)_ba.
template <int Q>
__device__ __forceinline__ void block_fp64_dl_pair(const Tile& T, int it, const Tile& S,
                                                        int js, const RegularRule& rule,
                                                        double dij[3][3], double dji[3][3]) {
  static_assert(Q > 0, "the paired double layer needs a compile-time rule size");
  const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
               dcz = T.G(fCz, it) - S.G(fCz, js);
  const double njx = S.G(fNx, js), njy = S.G(fNy, js), njz = S.G(fNz, js);
  const double nix = T.G(fNx, it), niy = T.G(fNy, it), niz = T.G(fNz, it);
  const double f0 = dcx * njx + dcy * njy + dcz * njz;
  const double f1 = T.G(fT0x, it) * njx + T.G(fT0y, it) * njy + T.G(fT0z, it) * njz;
  const double f2 = T.G(fT1x, it) * njx + T.G(fT1y, it) * njy + T.G(fT1z, it) * njz;
  const double g0 = -(dcx * nix + dcy * niy + dcz * niz);
  const double g1 = S.G(fT0x, js) * nix + S.G(fT0y, js) * niy + S.G(fT0z, js) * niz;
  const double g2 = S.G(fT1x, js) * nix + S.G(fT1y, js) * niy + S.G(fT1z, js) * niz;
  double bij[3][3], bji[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) bij[a][b] = bji[a][b] = 0.0;
#pragma unroll 1
  for (int p = 0; p < Q; ++p) {
    const double x0 = T.P(p, 0, it), x1 = T.P(p, 1, it), x2 = T.P(p, 2, it);
    double u0 = 0.0, u1 = 0.0, u2 = 0.0, v0 = 0.0, v1 = 0.0, v2 = 0.0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const double dx = x0 - S.P(q, 0, js), dy = x1 - S.P(q, 1, js), dz = x2 - S.P(q, 2, js);
      const double kern = rinv3_refined(dx * dx + dy * dy + dz * dz);
      u0 = fma(kern, rule.wphi[0][q], u0);
      u1 = fma(kern, rule.wphi[1][q], u1);
      u2 = fma(kern, rule.wphi[2][q], u2);
      const double kb = kern * fma(rule.u[q], g1, fma(rule.v[q], g2, g0));
      v0 = fma(kb, rule.wphi[0][q], v0);
      v1 = fma(kb, rule.wphi[1][q], v1);
      v2 = fma(kb, rule.wphi[2][q], v2);
    }
    const double ap = fma(rule.u[p], f1, fma(rule.v[p], f2, f0));
    const double c[3] = {rule.wphi[0][p], rule.wphi[1][p], rule.wphi[2][p]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double e = c[a] * ap;
      bij[a][0] = fma(e, u0, bij[a][0]);
      bij[a][1] = fma(e, u1, bij[a][1]);
      bij[a][2] = fma(e, u2, bij[a][2]);
      bji[a][0] = fma(c[a], v0, bji[a][0]);
      bji[a][1] = fma(c[a], v1, bji[a][1]);
      bji[a][2] = fma(c[a], v2, bji[a][2]);
    }
  }
  const double sc = T.G(fJdet, it) * S.G(fJdet, js) * kInv4Pi;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      dij[a][b] = bij[a][b] * sc;
      dji[a][b] = bji[a][b] * sc;
    }
}

// The Helmholtz double layer of a cell pair in both orders, FP64, as block_fp64_dl_pair:
// one kernel value e^{ikr} (1 - ikr) / r^3 per point pair, the phase referenced to the
// pair (e^{ikr} = e^{ik r0} e^{ik (r - r0)}, |k (r - r0)| <= 0.8 checked on the host), both
// blocks rotated by e^{ik r0} at the end.
template <int Q>
__device__ __forceinline__ void block_fp64_dl_pair_helmholtz(
    const Tile& T, int it, const Tile& S, int js, const RegularRule& rule, double k,
    double dij_re[3][3], double dij_im[3][3], double dji_re[3][3], double dji_im[3][3]) {
  static_assert(Q > 0, "the paired double layer needs a compile-time rule size");
  const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
               dcz = T.G(fCz, it) - S.G(fCz, js);
  const double njx = S.G(fNx, js), njy = S.G(fNy, js), njz = S.G(fNz, js);
  const double nix = T.G(fNx, it), niy = T.G(fNy, it), niz = T.G(fNz, it);
  const double f0 = dcx * njx + dcy * njy + dcz * njz;
  const double f1 = T.G(fT0x, it) * njx + T.G(fT0y, it) * njy + T.G(fT0z, it) * njz;
  const double f2 = T.G(fT1x, it) * njx + T.G(fT1y, it) * njy + T.G(fT1z, it) * njz;
  const double g0 = -(dcx * nix + dcy * niy + dcz * niz);
  const double g1 = S.G(fT0x, js) * nix + S.G(fT0y, js) * niy + S.G(fT0z, js) * niz;
  const double g2 = S.G(fT1x, js) * nix + S.G(fT1y, js) * niy + S.G(fT1z, js) * niz;
  const double r0sq = dcx * dcx + dcy * dcy + dcz * dcz;
  const double kr0 = k * (r0sq * rsqrt_refined(r0sq));
  double bij_re[3][3], bij_im[3][3], bji_re[3][3], bji_im[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) bij_re[a][b] = bij_im[a][b] = bji_re[a][b] = bji_im[a][b] = 0.0;
#pragma unroll 1
  for (int p = 0; p < Q; ++p) {
    const double x0 = T.P(p, 0, it), x1 = T.P(p, 1, it), x2 = T.P(p, 2, it);
    double ur[3] = {0.0, 0.0, 0.0}, ui[3] = {0.0, 0.0, 0.0};
    double vr[3] = {0.0, 0.0, 0.0}, vi[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const double dx = x0 - S.P(q, 0, js), dy = x1 - S.P(q, 1, js), dz = x2 - S.P(q, 2, js);
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double rinv = rsqrt_refined(r2);
      const double r = r2 * rinv, kr = k * r;
      double sn, cs;
      sincos_small(fma(k, r, -kr0), sn, cs);  // e^{ik (r - r0)}
      const double f = rinv * rinv * rinv;
      const double kre = f * fma(kr, sn, cs), kim = f * fma(-kr, cs, sn);
      const double bq = fma(rule.u[q], g1, fma(rule.v[q], g2, g0));
      const double bre = kre * bq, bim = kim * bq;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const double w = rule.wphi[b][q];
        ur[b] = fma(kre, w, ur[b]);
        ui[b] = fma(kim, w, ui[b]);
        vr[b] = fma(bre, w, vr[b]);
        vi[b] = fma(bim, w, vi[b]);
      }
    }
    const double ap = fma(rule.u[p], f1, fma(rule.v[p], f2, f0));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double c = rule.wphi[a][p], e = c * ap;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        bij_re[a][b] = fma(e, ur[b], bij_re[a][b]);
        bij_im[a][b] = fma(e, ui[b], bij_im[a][b]);
        bji_re[a][b] = fma(c, vr[b], bji_re[a][b]);
        bji_im[a][b] = fma(c, vi[b], bji_im[a][b]);
      }
    }
  }
  double ps, pc;
  sincos_cw(kr0, ps, pc);
  const double sc = T.G(fJdet, it) * S.G(fJdet, js) * kInv4Pi;
  const double cr = pc * sc, ci = ps * sc;  // e^{ik r0} jdet_i jdet_j / (4 pi)
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      dij_re[a][b] = bij_re[a][b] * cr - bij_im[a][b] * ci;
      dij_im[a][b] = bij_re[a][b] * ci + bij_im[a][b] * cr;
      dji_re[a][b] = bji_re[a][b] * cr - bji_im[a][b] * ci;
      dji_im[a][b] = bji_re[a][b] * ci + bji_im[a][b] * cr;
    }
}

// Per-pair constants of the FP32 far-pair quadrature.
template <int QT>
struct FarPair {
  static constexpr int kCap = QT > 0 ? QT : kMaxRegularPoints;
  float m2dx, m2dy, m2dz;   // -2 dc, dc = c_x - c_y in FP32
  float fa0, fa1, fa2;      // normal-derivative factors in tangent coordinates
  float r0f, r0sq, kf;      // reference distance (Helmholtz), |dc|^2, wavenumber
  // Helmholtz, packed loop: s is carried as s' = ks s (ks = k, or 1e-20 when k = 0), so
  // that k (r - r0) = s' / (r + r0) needs no multiply by k: ks times -2 dc, and 1 / ks
  float ksm2dx, ksm2dy, ksm2dz, ks, ks_inv;
  float wq[kCap];           // ADL: trial weights times the normal-derivative factor
};

// Sums of one far pair in FP32: blk[a][b] and S (see block_fp64 for their meaning),
// without the reference phase e^{ik r0}.  kSmallPhase: |k (r - r0)| <= 0.8 for every
// point pair (polynomial cos / sin, fully unrolled inner loop); otherwise the phase is
// reduced by multiples of pi/2 first.  Test and trial points are read from shared memory
// as float4 (offset from the centroid, squared length): one load per point.
template <int QT, int KER, int OP, int NBT, int NBS, bool kSmallPhase>
__device__ __forceinline__ void far_sums(const Tile& T, int it, const Tile& S, int js,
                                         const RegularRule& rule, const FarPair<QT>& fp,
                                         float blk_re[NBT][NBS],
                                         float blk_im[NBT][NBS], float& S_re, float& S_im) {
  constexpr bool kC = KER == kHelmholtz;
  constexpr bool kNeedBasis = OP != kHS || kC;
  constexpr bool kKahan = NBT == 1 && NBS == 1;
  const int Q = QT > 0 ? QT : rule.npts;
  float cmp_re = 0.f, cmp_im = 0.f;
#pragma unroll 1
  for (int p = 0; p < Q; ++p) {
    const float4 a = T.R4(p, it);
    const float apf = OP == kDL ? fmaf(rule.uf[p], fp.fa1, fmaf(rule.vf[p], fp.fa2, fp.fa0)) : 1.f;
    // s_pq = A_p + |y_q|^2 + w_p . y_q; Laplace adds |dc|^2 so that it is r^2 itself
    const float wx = fmaf(-2.f, a.x, fp.m2dx), wy = fmaf(-2.f, a.y, fp.m2dy),
                wz = fmaf(-2.f, a.z, fp.m2dz);
    const float Ap = fmaf(-a.x, fp.m2dx, fmaf(-a.y, fp.m2dy, fmaf(-a.z, fp.m2dz,
                                                                  a.w + (kC ? 0.f : fp.r0sq))));
    float u_re[NBS], u_im[NBS], g_re = 0.f, g_im = 0.f;
#pragma unroll
    for (int b = 0; b < NBS; ++b) u_re[b] = u_im[b] = 0.f;
#pragma unroll(kSmallPhase ? 6 : 1)
    for (int q = 0; q < Q; ++q) {
      const float4 y = S.R4(q, js);  // the same address in every lane: a broadcast
      const float wq = OP != kADL ? rule.wf[q]
                       : kSmallPhase ? fp.wq[q]
                                    : rule.wf[q] * fmaf(rule.uf[q], fp.fa1, fmaf(rule.vf[q], fp.fa2, fp.fa0));
      const float s = fmaf(wx, y.x, fmaf(wy, y.y, fmaf(wz, y.z, Ap + y.w)));
      float kre, kim = 0.f;
      if (!kC) {
        const float rinv = rsqrt_approx(s);  // s is r^2 here
        kre = (OP == kSL || OP == kHS) ? wq * rinv : wq * (rinv * rinv * rinv);
      } else {
        const float r2 = fp.r0sq + s;
        const float rinv = rsqrt_approx(r2);
        const float t = fp.kf * s * rcp_approx(fmaf(r2, rinv, fp.r0f));  // k (r - r0)
        float cs, sn;
        if (kSmallPhase)
          poly_cos_sin(t, cs, sn);
        else
          reduced_cos_sin(t, cs, sn);
        if (OP == kSL || OP == kHS) {
          const float f = wq * rinv;
          kre = f * cs;
          kim = f * sn;
        } else {
          // (1 - ik r) e^{ik r} / r^3 with e^{ik r0} applied per pair
          const float f = wq * (rinv * rinv * rinv), kr = fp.kf * (r2 * rinv);
          kre = f * fmaf(kr, sn, cs);
          kim = f * fmaf(-kr, cs, sn);
        }
      }
      if (OP == kHS) {
        g_re += kre;
        if (kC) g_im += kim;
      }
      if (kNeedBasis) {
        if (NBS == 1) {
          u_re[0] += kre;
          if (kC) u_im[0] += kim;
        } else {
#pragma unroll
          for (int b = 0; b < NBS; ++b) {
            u_re[b] = fmaf(kre, rule.phif[b][q], u_re[b]);
            if (kC) u_im[b] = fmaf(kim, rule.phif[b][q], u_im[b]);
          }
        }
      }
    }
    if (OP == kHS) {
      S_re = fmaf(rule.wf[p], g_re, S_re);
      if (kC) S_im = fmaf(rule.wf[p], g_im, S_im);
    }
    if (kNeedBasis) {
      const float wp = rule.wf[p] * apf;
      if (kKahan) {
        kahan_add(blk_re[0][0], cmp_re, wp * u_re[0]);
        if (kC) kahan_add(blk_im[0][0], cmp_im, wp * u_im[0]);
      } else {
#pragma unroll
        for (int a = 0; a < NBT; ++a) {
          const float f = NBT == 1 ? wp : wp * rule.phif[a][p];
#pragma unroll
          for (int b = 0; b < NBS; ++b) {
            blk_re[a][b] = fmaf(f, u_re[b], blk_re[a][b]);
            if (kC) blk_im[a][b] = fmaf(f, u_im[b], blk_im[a][b]);
          }
        }
      }
    }
  }
}

// far_sums for rules with an even number of points and no phase reduction (Laplace, or
// Helmholtz with |k (r - r0)| <= 0.8): trial points 2j and 2j + 1 go through packed FP32x2
// instructions together (each half rounded as the scalar operation), which halves the
// issue slots of the inner loop; both points arrive in two 128-bit shared-memory loads
// (the paired layout of the FP32 offsets).  Even and odd trial points are summed
// separately and added per test point.
// kWide: the phases may reach |k (r - r0)| <= 1.6 (poly_cos_sin_wide2).
template <int QT, int KER, int OP, int NBT, int NBS, bool kWide = false>
__device__ __forceinline__ void far_sums_x2(const Tile& T, int it, const Tile& S, int js,
                                            const RegularRule& rule, const FarPair<QT>& fp,
                                            float blk_re[NBT][NBS], float blk_im[NBT][NBS],
                                            float& S_re, float& S_im) {
  static_assert(QT > 0 && QT % 2 == 0, "pairs of trial points");
  constexpr bool kC = KER == kHelmholtz;
  constexpr bool kNeedBasis = OP != kHS || kC;
  constexpr bool kKahan = NBT == 1 && NBS == 1;
  float cmp_re = 0.f, cmp_im = 0.f;
  const float2 r0sq2 = f2(fp.r0sq), r0f2 = f2(fp.r0f), kf2 = f2(fp.kf), nkf2 = f2(-fp.kf);
  const float2 ks2 = f2(fp.ks), ksinv2 = f2(fp.ks_inv);
#pragma unroll 1
  for (int p = 0; p < QT; ++p) {
    const float4 a = T.R4(p, it);
    const float apf = OP == kDL ? fmaf(rule.uf[p], fp.fa1, fmaf(rule.vf[p], fp.fa2, fp.fa0)) : 1.f;
    // s_pq = A_p + |y_q|^2 + w_p . y_q; Laplace adds |dc|^2 so that it is r^2 itself;
    // Helmholtz carries s' = ks s (every term of s times ks)
    const float m2 = kC ? -2.f * fp.ks : -2.f;
    const float mx = kC ? fp.ksm2dx : fp.m2dx, my = kC ? fp.ksm2dy : fp.m2dy,
                mz = kC ? fp.ksm2dz : fp.m2dz;
    const float2 wx = f2(fmaf(m2, a.x, mx)), wy = f2(fmaf(m2, a.y, my)), wz = f2(fmaf(m2, a.z, mz));
    const float2 Ap = f2(fmaf(-a.x, mx, fmaf(-a.y, my, fmaf(-a.z, mz,
                                                        kC ? fp.ks * a.w : a.w + fp.r0sq))));
    float2 u_re[NBS], u_im[NBS], g_re = f2(0.f), g_im = f2(0.f);
#pragma unroll
    for (int b = 0; b < NBS; ++b) u_re[b] = u_im[b] = f2(0.f);
#pragma unroll
    for (int j = 0; j < QT / 2; ++j) {
      const float4 A = S.RA(j, js), B = S.RB(j, js);  // the same address in every lane
      const float2 wq = OP != kADL ? make_float2(rule.wf[2 * j], rule.wf[2 * j + 1])
                                   : make_float2(fp.wq[2 * j], fp.wq[2 * j + 1]);
      const float2 s = ffma2(wx, make_float2(A.x, A.y),
                             ffma2(wy, make_float2(A.z, A.w),
                                   ffma2(wz, make_float2(B.x, B.y),
                                         kC ? ffma2(ks2, make_float2(B.z, B.w), Ap)
                                            : fadd2(Ap, make_float2(B.z, B.w)))));
      float2 f, c = f2(1.f), sn = f2(0.f);  // kernel value = f (c + i sn)
      if (!kC) {
        const float2 rinv = rsqrt_approx2(s);  // s is r^2 here
        f = (OP == kSL || OP == kHS) ? fmul2(wq, rinv) : fmul2(wq, fmul2(fmul2(rinv, rinv), rinv));
      } else {
        const float2 r2 = ffma2(s, ksinv2, r0sq2);  // s is s' = ks s here
        const float2 rinv = rsqrt_approx2(r2);
        // k (r - r0) = s' / (r + r0) (exactly when ks = k; 1e-20 s / (r + r0) when k = 0)
        const float2 t = fmul2(s, rcp_approx2(ffma2(r2, rinv, r0f2)));
        float2 cs, ss;
        if (kWide)
          poly_cos_sin_wide2(t, cs, ss);
        else
          poly_cos_sin2(t, cs, ss);
        if (OP == kSL || OP == kHS) {
          f = fmul2(wq, rinv);
          c = cs;
          sn = ss;
        } else {
          // (1 - ik r) e^{ik r} / r^3 with e^{ik r0} applied per pair
          const float2 rr = fmul2(r2, rinv);
          f = fmul2(wq, fmul2(fmul2(rinv, rinv), rinv));
          c = ffma2(fmul2(kf2, rr), ss, cs);
          sn = ffma2(fmul2(nkf2, rr), cs, ss);
        }
      }
      if (OP == kHS) {
        if (kC) {
          g_re = ffma2(f, c, g_re);
          g_im = ffma2(f, sn, g_im);
        } else {
          g_re = fadd2(g_re, f);
        }
      }
      if (kNeedBasis) {
        if (NBS == 1) {
          if (kC) {
            u_re[0] = ffma2(f, c, u_re[0]);
            u_im[0] = ffma2(f, sn, u_im[0]);
          } else {
            u_re[0] = fadd2(u_re[0], f);
          }
        } else {
          const float2 kre = kC ? fmul2(f, c) : f, kim = fmul2(f, sn);
#pragma unroll
          for (int b = 0; b < NBS; ++b) {
            const float2 phi = make_float2(rule.phif[b][2 * j], rule.phif[b][2 * j + 1]);
            u_re[b] = ffma2(kre, phi, u_re[b]);
            if (kC) u_im[b] = ffma2(kim, phi, u_im[b]);
          }
        }
      }
    }
    if (OP == kHS) {
      S_re = fmaf(rule.wf[p], g_re.x + g_re.y, S_re);
      if (kC) S_im = fmaf(rule.wf[p], g_im.x + g_im.y, S_im);
    }
    if (kNeedBasis) {
      const float wp = rule.wf[p] * apf;
      if (kKahan) {
        kahan_add(blk_re[0][0], cmp_re, wp * (u_re[0].x + u_re[0].y));
        if (kC) kahan_add(blk_im[0][0], cmp_im, wp * (u_im[0].x + u_im[0].y));
      } else {
#pragma unroll
        for (int a = 0; a < NBT; ++a) {
          const float fa = NBT == 1 ? wp : wp * rule.phif[a][p];
#pragma unroll
          for (int b = 0; b < NBS; ++b) {
            blk_re[a][b] = fmaf(fa, u_re[b].x + u_re[b].y, blk_re[a][b]);
            if (kC) blk_im[a][b] = fmaf(fa, u_im[b].x + u_im[b].y, blk_im[a][b]);
          }
        }
      }
    }
  }
}

// The double layer of a far cell pair in both orders, mixed precision, for one P1 / DP1
// space on both sides (the paired launch): the FP32 packed loop of far_sums_x2 with the
// phase referenced to the pair (|k (r - r0)| <= 0.8, the launch's bound), one kernel value
// per point pair for DL(test i, trial j) (the normal factor (x_p - y).n_j per test point)
// and DL(test j, trial i) (the factor (y_q - x).n_i per point pair, folded per test point
// like block_fp64_dl_pair); geometry, the reference phase e^{ik r0} and the blocks' final
// scaling in FP64.  dij / dji as in block_fp64_dl_pair.
template <int QT, int KER>
__device__ __forceinline__ void block_fp32_dl_pair(const Tile& T, int it, const Tile& S, int js,
                                                   const RegularRule& rule, double k,
                                                   double dij_re[3][3], double dij_im[3][3],
                                                   double dji_re[3][3], double dji_im[3][3]) {
  static_assert(QT > 0 && QT % 2 == 0, "pairs of trial points");
  constexpr bool kC = KER == kHelmholtz;
  const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
               dcz = T.G(fCz, it) - S.G(fCz, js);
  const double njx = S.G(fNx, js), njy = S.G(fNy, js), njz = S.G(fNz, js);
  const double nix = T.G(fNx, it), niy = T.G(fNy, it), niz = T.G(fNz, it);
  // (x_p - y).n_j = fa0 + u_p fa1 + v_p fa2; (y_q - x).n_i = fb0 + u_q fb1 + v_q fb2
  const float fa0 = static_cast<float>(dcx * njx + dcy * njy + dcz * njz);
  const float fa1 = static_cast<float>(T.G(fT0x, it) * njx + T.G(fT0y, it) * njy + T.G(fT0z, it) * njz);
  const float fa2 = static_cast<float>(T.G(fT1x, it) * njx + T.G(fT1y, it) * njy + T.G(fT1z, it) * njz);
  const float fb0 = static_cast<float>(-(dcx * nix + dcy * niy + dcz * niz));
  const float fb1 = static_cast<float>(S.G(fT0x, js) * nix + S.G(fT0y, js) * niy + S.G(fT0z, js) * niz);
  const float fb2 = static_cast<float>(S.G(fT1x, js) * nix + S.G(fT1y, js) * niy + S.G(fT1z, js) * niz);
  const float fdx = static_cast<float>(dcx), fdy = static_cast<float>(dcy),
              fdz = static_cast<float>(dcz);
  const double r0sq = dcx * dcx + dcy * dcy + dcz * dcz;
  // s = r^2 - r0^2 (Helmholtz carries s' = ks s, ks = k or 1e-20 when k = 0), as in
  // far_sums_x2
  const float kf = static_cast<float>(k), ks = kf != 0.f ? kf : 1e-20f, ks_inv = 1.f / ks;
  const float m2 = kC ? -2.f * ks : -2.f;
  const float mx = (kC ? ks : 1.f) * (-2.f * fdx), my = (kC ? ks : 1.f) * (-2.f * fdy),
              mz = (kC ? ks : 1.f) * (-2.f * fdz);
  float r0f = 0.f, r0sqf = fmaf(fdx, fdx, fmaf(fdy, fdy, fdz * fdz));
  double ph_c = 1.0, ph_s = 0.0;
  if (kC) {
    const double r0 = r0sq * rsqrt_refined(r0sq);
    r0f = static_cast<float>(r0);
    r0sqf = static_cast<float>(r0sq);
    float pc, ps;
    phase_cos_sin(k * r0, pc, ps);
    ph_c = pc;
    ph_s = ps;
  }
  const float2 r0sq2 = f2(r0sqf), r0f2 = f2(r0f), kf2 = f2(kf), nkf2 = f2(-kf);
  const float2 ks2 = f2(ks), ksinv2 = f2(ks_inv);
  float bij_re[3][3], bij_im[3][3], bji_re[3][3], bji_im[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) bij_re[a][b] = bij_im[a][b] = bji_re[a][b] = bji_im[a][b] = 0.f;
#pragma unroll 1
  for (int p = 0; p < QT; ++p) {
    const float4 a = T.R4(p, it);
    const float apf = fmaf(rule.uf[p], fa1, fmaf(rule.vf[p], fa2, fa0));
    const float2 wx = f2(fmaf(m2, a.x, mx)), wy = f2(fmaf(m2, a.y, my)), wz = f2(fmaf(m2, a.z, mz));
    const float2 Ap = f2(fmaf(-a.x, mx, fmaf(-a.y, my, fmaf(-a.z, mz, kC ? ks * a.w : a.w + r0sqf))));
    float2 ur[3], ui[3], vr[3], vi[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) ur[b] = ui[b] = vr[b] = vi[b] = f2(0.f);
#pragma unroll
    for (int j = 0; j < QT / 2; ++j) {
      const float4 A = S.RA(j, js), B = S.RB(j, js);
      const float2 wq = make_float2(rule.wf[2 * j], rule.wf[2 * j + 1]);
      const float2 sv = ffma2(wx, make_float2(A.x, A.y),
                              ffma2(wy, make_float2(A.z, A.w),
                                    ffma2(wz, make_float2(B.x, B.y),
                                          kC ? ffma2(ks2, make_float2(B.z, B.w), Ap)
                                             : fadd2(Ap, make_float2(B.z, B.w)))));
      float2 kre, kim = f2(0.f);
      if (!kC) {
        const float2 rinv = rsqrt_approx2(sv);  // sv is r^2 here
        kre = fmul2(wq, fmul2(fmul2(rinv, rinv), rinv));
      } else {
        const float2 r2 = ffma2(sv, ksinv2, r0sq2);
        const float2 rinv = rsqrt_approx2(r2);
        const float2 t = fmul2(sv, rcp_approx2(ffma2(r2, rinv, r0f2)));
        float2 cs, ss;
        poly_cos_sin2(t, cs, ss);
        const float2 rr = fmul2(r2, rinv);
        const float2 f = fmul2(wq, fmul2(fmul2(rinv, rinv), rinv));
        // (1 - ik r) e^{ik (r - r0)} / r^3
        kre = fmul2(f, ffma2(fmul2(kf2, rr), ss, cs));
        kim = fmul2(f, ffma2(fmul2(nkf2, rr), cs, ss));
      }
      const float2 bq = ffma2(make_float2(rule.uf[2 * j], rule.uf[2 * j + 1]), f2(fb1),
                              ffma2(make_float2(rule.vf[2 * j], rule.vf[2 * j + 1]), f2(fb2), f2(fb0)));
      const float2 bre = fmul2(kre, bq), bim = kC ? fmul2(kim, bq) : f2(0.f);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const float2 phi = make_float2(rule.phif[b][2 * j], rule.phif[b][2 * j + 1]);
        ur[b] = ffma2(kre, phi, ur[b]);
        vr[b] = ffma2(bre, phi, vr[b]);
        if (kC) {
          ui[b] = ffma2(kim, phi, ui[b]);
          vi[b] = ffma2(bim, phi, vi[b]);
        }
      }
    }
    const float wp = rule.wf[p];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float c = wp * rule.phif[a][p], e = c * apf;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        bij_re[a][b] = fmaf(e, ur[b].x + ur[b].y, bij_re[a][b]);
        bji_re[a][b] = fmaf(c, vr[b].x + vr[b].y, bji_re[a][b]);
        if (kC) {
          bij_im[a][b] = fmaf(e, ui[b].x + ui[b].y, bij_im[a][b]);
          bji_im[a][b] = fmaf(c, vi[b].x + vi[b].y, bji_im[a][b]);
        }
      }
    }
  }
  const double sc = T.G(fJdet, it) * S.G(fJdet, js) * kInv4Pi;
  const double cr = ph_c * sc, ci = ph_s * sc;  // e^{ik r0} jdet_i jdet_j / (4 pi)
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const double xr = bij_re[a][b], xi = bij_im[a][b], yr = bji_re[a][b], yi = bji_im[a][b];
      dij_re[a][b] = xr * cr - xi * ci;
      dij_im[a][b] = xr * ci + xi * cr;
      dji_re[a][b] = yr * cr - yi * ci;
      dji_im[a][b] = yr * ci + yi * cr;
    }
}

// Phase handling of a launch (Helmholtz far pairs): kPhaseRuntime chooses per warp (the
// unreduced polynomials of |t| <= 0.8 or, for even rules, of |t| <= 1.6 when the warp's
// k (rad_x + rad_y) allows it, else the reduction), kPhaseSmall assumes |k (r - r0)| <= 0.8
// for every pair of the launch (the host checks k (max rad_x + max rad_y) <= 0.8),
// kPhaseGeneral reduces every phase.
enum PhaseMode : int { kPhaseRuntime = 0, kPhaseSmall = 1, kPhaseGeneral = 2 };

// FP32 local block of a far pair (see the file comment for the formulation).
template <int QT, int KER, int OP, int NBT, int NBS, int PH>
__device__ __forceinline__ void block_fp32(const Tile& T, int it, const Tile& S, int js,
                                           const RegularRule& rule, double k,
                                           double ore[NBT][NBS], double oim[NBT][NBS]) {
  constexpr bool kC = KER == kHelmholtz;
  const int Q = QT > 0 ? QT : rule.npts;
  FarPair<QT> fp;
  const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
               dcz = T.G(fCz, it) - S.G(fCz, js);
  const float fdx = static_cast<float>(dcx), fdy = static_cast<float>(dcy),
              fdz = static_cast<float>(dcz);
  fp.m2dx = -2.f * fdx;
  fp.m2dy = -2.f * fdy;
  fp.m2dz = -2.f * fdz;
  fp.fa0 = fp.fa1 = fp.fa2 = 0.f;
  if (OP == kDL) {
    const double nx = S.G(fNx, js), ny = S.G(fNy, js), nz = S.G(fNz, js);
    fp.fa0 = static_cast<float>(dcx * nx + dcy * ny + dcz * nz);
    fp.fa1 = static_cast<float>(T.G(fT0x, it) * nx + T.G(fT0y, it) * ny + T.G(fT0z, it) * nz);
    fp.fa2 = static_cast<float>(T.G(fT1x, it) * nx + T.G(fT1y, it) * ny + T.G(fT1z, it) * nz);
  } else if (OP == kADL) {
    const double nx = T.G(fNx, it), ny = T.G(fNy, it), nz = T.G(fNz, it);
    fp.fa0 = static_cast<float>(-(dcx * nx + dcy * ny + dcz * nz));
    fp.fa1 = static_cast<float>(S.G(fT0x, js) * nx + S.G(fT0y, js) * ny + S.G(fT0z, js) * nz);
    fp.fa2 = static_cast<float>(S.G(fT1x, js) * nx + S.G(fT1y, js) * ny + S.G(fT1z, js) * nz);
  }
  float ph_c = 1.f, ph_s = 0.f;
  bool small_phase = PH != kPhaseGeneral;  // kPhaseRuntime: decided per warp below
  bool wide_phase = false;
  fp.r0f = fp.kf = 0.f;
  fp.r0sq = fmaf(fdx, fdx, fmaf(fdy, fdy, fdz * fdz));
  if (kC) {
    const double r0sq = dcx * dcx + dcy * dcy + dcz * dcz;
    const double r0 = r0sq * rsqrt_refined(r0sq);
    fp.r0f = static_cast<float>(r0);
    fp.r0sq = static_cast<float>(r0sq);
    fp.kf = static_cast<float>(k);
    fp.ks = fp.kf != 0.f ? fp.kf : 1e-20f;
    fp.ks_inv = 1.f / fp.ks;
    fp.ksm2dx = fp.ks * fp.m2dx;
    fp.ksm2dy = fp.ks * fp.m2dy;
    fp.ksm2dz = fp.ks * fp.m2dz;
    phase_cos_sin(k * r0, ph_c, ph_s);
    // warp-uniform choice, so that a warp never runs two variants
    if (PH == kPhaseRuntime) {
      const double bound = k * (T.G(fRad, it) + S.G(fRad, js));
      const unsigned active = __activemask();
      small_phase = __all_sync(active, bound <= static_cast<double>(kSmallPhaseMax));
      wide_phase = __all_sync(active, bound <= static_cast<double>(kWidePhaseMax));
    }
  }
  if (OP == kADL) {
#pragma unroll
    for (int q = 0; q < Q; ++q)
      fp.wq[q] = rule.wf[q] * fmaf(rule.uf[q], fp.fa1, fmaf(rule.vf[q], fp.fa2, fp.fa0));
  }
  float blk_re[NBT][NBS], blk_im[NBT][NBS], S_re = 0.f, S_im = 0.f;
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b) blk_re[a][b] = blk_im[a][b] = 0.f;
  constexpr bool kPacked = QT > 0 && QT % 2 == 0;
  auto small = [&] {
    if constexpr (kPacked) {
      far_sums_x2<QT, KER, OP, NBT, NBS>(T, it, S, js, rule, fp, blk_re, blk_im, S_re, S_im);
    } else {
      far_sums<QT, KER, OP, NBT, NBS, true>(T, it, S, js, rule, fp, blk_re, blk_im, S_re, S_im);
    }
  };
  if (!kC || PH == kPhaseSmall) {
    small();
  } else if (PH == kPhaseGeneral) {
    far_sums<QT, KER, OP, NBT, NBS, false>(T, it, S, js, rule, fp, blk_re, blk_im, S_re, S_im);
  } else {
    if (small_phase) {
      small();
    } else if (kPacked && wide_phase) {
      if constexpr (kPacked)
        far_sums_x2<QT, KER, OP, NBT, NBS, true>(T, it, S, js, rule, fp, blk_re, blk_im, S_re, S_im);
    } else {
      far_sums<QT, KER, OP, NBT, NBS, false>(T, it, S, js, rule, fp, blk_re, blk_im, S_re, S_im);
    }
  }
  // back to FP64, applying the reference phase e^{ik r0}
  double bre[NBT][NBS], bim[NBT][NBS];
  double Sre = S_re, Sim = S_im;
  const double pc = ph_c, ps = ph_s;
  if (kC) {
    const double re = Sre * pc - Sim * ps, im = Sre * ps + Sim * pc;
    Sre = re;
    Sim = im;
  }
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b) {
      double re = blk_re[a][b], im = blk_im[a][b];
      if (kC) {
        const double r2 = re * pc - im * ps, i2 = re * ps + im * pc;
        re = r2;
        im = i2;
      }
      bre[a][b] = re;
      bim[a][b] = im;
    }
  finish_block<KER, OP, NBT, NBS>(T, it, S, js, k, bre, bim, Sre, Sim, ore, oim);
}

__device__ __forceinline__ bool near_pair(const Tile& T, int it, const Tile& S, int js) {
  const double dx = T.G(fCx, it) - S.G(fCx, js), dy = T.G(fCy, it) - S.G(fCy, js),
               dz = T.G(fCz, it) - S.G(fCz, js);
  const double lim = 2.0 * fmax(T.G(fDiam, it), S.G(fDiam, js));
  return dx * dx + dy * dy + dz * dz < lim * lim;
}

template <int NBT, int NBS, bool kC>
__device__ __forceinline__ void deposit(double* acc_re, double* acc_im, int ndt, const Tile& T,
                                        int it, const Tile& S, int js,
                                        const double ore[NBT][NBS], const double oim[NBT][NBS]) {
#pragma unroll
  for (int b = 0; b < NBS; ++b) {
    const int ls = S.ldof[b * kTile + js];
#pragma unroll
    for (int a = 0; a < NBT; ++a) {
      const int idx = T.ldof[a * kTile + it] + ndt * ls;
      atomicAdd(acc_re + idx, ore[a][b]);
      if (kC) atomicAdd(acc_im + idx, oim[a][b]);
    }
  }
}

template <bool kC>
__device__ __forceinline__ void mirror_put(double* mir, int it, int js, double re, double im) {
  if (kC) {
    mir[2 * (js * (kTile + 1) + it)] = re;
    mir[2 * (js * (kTile + 1) + it) + 1] = im;
  } else {
    mir[js * (kTile + 1) + it] = re;
  }
}

// Near-pair handling of a launch.  kNearInKernel: every pair is tested in the kernel and
// near pairs are queued in shared memory and integrated in FP64 after the main loop (the
// FP64 kernels skip the test); kNearMasked: the pairs marked in the near-field masks are
// skipped (FP32 far pairs only; near_pairs_fp64 integrates the near ones).
enum NearMode : int { kNearInKernel = 0, kNearMasked = 1 };

// Resident CTAs per SM the register allocation must allow: 5 for the FP64 Laplace
// hypersingular kernel (it fits in 96 registers without spills), 6 for the mixed
// Helmholtz DP0 kernels (80 registers; with no FP64 points in their tiles six CTAs also
// fit in shared memory), 3 for the paired FP64 Helmholtz double layer (168 registers; at
// 128 it spills 228 bytes, and four CTAs per SM ran 17 % slower), 4 elsewhere (the paired
// Laplace double layer too: at 128 registers it spills 48 bytes; the paired mixed
// Helmholtz one, which stages the real and imaginary parts of its blocks in turn to fit
// four CTAs in shared memory, needs 127 registers without spills).
template <int KER, int OP, bool MIXED, bool DIRECT, bool PAIRED = false>
constexpr int min_ctas() {
  return (PAIRED && KER == kHelmholtz && !MIXED)   ? 3
         : (KER == kLaplace && OP == kHS && !MIXED) ? 5
         : (MIXED && DIRECT && KER == kHelmholtz)   ? 6
                                                    : 4;
}

// PAIRED (Laplace DL / ADL, FP64, one P1 / DP1 space on both sides, Q = 6): the tile
// pairs tx >= sy, each off-diagonal one integrated in both orders from one evaluation of
// the kernel per point pair (block_fp64_dl_pair), the (sy, tx) blocks accumulated
// separately and added at the transposed entries.
template <int QT, int KER, int OP, int NBT, int NBS, bool MIXED, bool DIRECT, int PH, int NM,
          bool PAIRED = false>
__global__ void __launch_bounds__(kThreads, min_ctas<KER, OP, MIXED, DIRECT, PAIRED>())
    regular_tiles(CellSet test, SpaceTiles tt, CellSet trial, SpaceTiles st, RegularRule rule,
                  double k, int same_grid, double* __restrict__ out, int64_t ld, int tile_y0,
                  int tile_y1, NearArgs near, int symmetric, int acc_copies) {
  static_assert(!PAIRED || ((OP == kDL || OP == kADL) && NBT == 3 && NBS == 3 && !DIRECT &&
                            QT == 6 && (KER == kLaplace || PH == kPhaseSmall) &&
                            (!MIXED || NM == kNearMasked)),
                "paired blocks: DL / ADL, P1 / DP1, 6-point rule (Helmholtz: phases "
                "referenced to the pair; mixed: near pairs masked)");
  constexpr bool kC = KER == kHelmholtz;
  constexpr bool kQueue = MIXED && NM == kNearInKernel;
  constexpr bool kRel = MIXED;  // FP32 offsets staged
  constexpr bool kPts = !MIXED || NM == kNearInKernel;  // FP64 points staged
  // P1 (or DP1) test space: the lanes' local blocks go through a per-warp stage and are
  // summed per test DOF (lane = DOF) before the accumulator, so that no two lanes of a
  // warp update the same entry (test cells share vertex DOFs)
  constexpr bool kGather = !DIRECT && NBT == 3;
  // complex blocks gathered through one real stage, real parts first (paired mixed
  // Helmholtz: four CTAs per SM fit in shared memory)
  constexpr bool kSplitStage = kGather && kC && PAIRED && MIXED;
  // real FP64 P1 blocks (not the hypersingular kernel, which keeps 5 CTAs per SM; not the
  // mixed kernels, whose larger tiles would then limit the CTAs per SM): one accumulator
  // per warp, updated with plain adds, summed at the flush
  constexpr int kAccMax = (kGather && !kC && !MIXED && OP != kHS && !PAIRED) ? kWarps : 1;
  // the host passes 1 when kAccMax copies of the largest DOF block do not fit in shared
  // memory (DP1 x DP1: 96 x 96 DOFs per tile pair); the warps then add with atomics
  const int kAcc = kAccMax > 1 && acc_copies > 1 ? kAccMax : 1;
  const int Q = QT > 0 ? QT : rule.npts;
  // symmetric operator on one space (single layer, hypersingular): only the tile pairs with
  // tx >= sy are computed, the blocks with tx > sy also written transposed
  int tx, sy;
  if (symmetric) {
    lower_tile_pair(blockIdx.x, (test.ncells + kTile - 1) / kTile, tile_y0, tile_y1, tx, sy);
  } else {
    tx = blockIdx.x;
    sy = blockIdx.y + tile_y0;
  }
  const bool mirror = symmetric && tx > sy;
  const int moff = NM == kNearMasked
                       ? __ldg(near.tile_mask + static_cast<int64_t>(tx) * near.trial_tiles + sy)
                       : -1;
  const int ti0 = tx * kTile, sj0 = sy * kTile;
  const int nti = min(kTile, test.ncells - ti0), nsj = min(kTile, trial.ncells - sj0);

  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);  // completion of the tile copies
  unsigned char* cursor = smem + 16;
  double* acc_re = nullptr;
  double* acc_im = nullptr;
  int ndt = 0, nds = 0, tdof0 = 0, sdof0 = 0, cap = 0;
  if (!DIRECT) {
    tdof0 = tt.tile_dof_off[tx];
    ndt = tt.tile_dof_off[tx + 1] - tdof0;
    sdof0 = st.tile_dof_off[sy];
    nds = st.tile_dof_off[sy + 1] - sdof0;
    cap = tt.max_tile_dofs * st.max_tile_dofs;
    acc_re = reinterpret_cast<double*>(cursor);
    acc_im = acc_re + cap;
    cursor += sizeof(double) * cap * (kC ? 2 : 1) * kAcc;
  }
  // PAIRED: the (sy, tx) blocks, indexed as acc_re (test-tile DOF + ndt * trial-tile DOF),
  // imaginary parts (Helmholtz) cap further on
  double* acc_t = reinterpret_cast<double*>(cursor);
  if (PAIRED) cursor += sizeof(double) * cap * (kC ? 2 : 1);
  double* stage_re = nullptr;  // kGather: [warp][(a * NBS + b) * kTile + lane]
  double* stage_im = nullptr;
  uint8_t* inc_off = nullptr;  // kGather: the test tile's DOF incidence
  uint8_t* inc_ent = nullptr;
  if (kGather) {
    constexpr int kStage = kWarps * kTile * NBT * NBS;
    stage_re = reinterpret_cast<double*>(cursor);
    stage_im = stage_re + kStage;
    cursor += sizeof(double) * kStage * ((kC && !kSplitStage) ? 2 : 1);
    inc_off = cursor;
    inc_ent = cursor + 3 * kTile + 1;
    cursor += 6 * kTile + 1;
  }
  const Tile T = carve_tile(cursor, Q, kRel, NBT, kPts);
  const Tile S = carve_tile(cursor, Q, kRel, NBS, kPts);
  // DIRECT, symmetric: the block's entries, [js * (kTile + 1) + it], for the transposed
  // write; padded rows keep both access patterns free of bank conflicts
  double* mir = reinterpret_cast<double*>(cursor);
  if (DIRECT && symmetric) cursor += sizeof(double) * kTile * (kTile + 1) * (kC ? 2 : 1);
  unsigned short* queue = reinterpret_cast<unsigned short*>(cursor);  // kQueue: near pairs
  int* qcount = reinterpret_cast<int*>(cursor + sizeof(unsigned short) * kTile * kTile);

  // Both tiles arrive by bulk (TMA) copies issued by one thread and completed on the
  // mbarrier, while the other threads clear the accumulator and load local DOF indices.
  if (threadIdx.x == 0) mbar_init(mbar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(mbar, 2 * bulk_tile_bytes(Q, kRel, kPts));
    stage_tile_bulk(T, test, ti0, Q, kRel, mbar, kPts);
    stage_tile_bulk(S, trial, sj0, Q, kRel, mbar, kPts);
  }
  if (!DIRECT) {
    for (int w = 0; w < kAcc; ++w)
      for (int idx = threadIdx.x; idx < ndt * nds; idx += kThreads) {
        acc_re[w * cap + idx] = 0.0;
        if (kC) acc_im[idx] = 0.0;
      }
    if (PAIRED)
      for (int idx = threadIdx.x; idx < ndt * nds; idx += kThreads) {
        acc_t[idx] = 0.0;
        if (kC) acc_t[cap + idx] = 0.0;
      }
    load_ldof(T, ti0, nti, tt.cell_ldof, NBT);
    load_ldof(S, sj0, nsj, st.cell_ldof, NBS);
    if (kGather)
      for (int i = threadIdx.x; i < 6 * kTile + 1; i += kThreads)
        inc_off[i] = i <= 3 * kTile ? __ldg(tt.inc_off + static_cast<int64_t>(tx) * (3 * kTile + 1) + i)
                                    : __ldg(tt.inc_ent + static_cast<int64_t>(tx) * 3 * kTile + i - (3 * kTile + 1));
  }
  if (kQueue && threadIdx.x == 0) *qcount = 0;
  const bool staged = mbar_wait_bounded(mbar, 0, g_stage_poll_limit);
  if (__syncthreads_or(!staged)) {
    // the copies did not complete in time: record it, give them a last bounded wait and
    // leave this block's entries unwritten (the host reports the failure)
    if (threadIdx.x == 0) atomicAdd(&g_stage_timeouts, 1u);
    mbar_wait_bounded(mbar, 0);
    return;
  }

  const int it = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool lane_cell = it < nti;
  int a0 = -1, a1 = -2, a2 = -3;
  unsigned mword = 0u;
  if (lane_cell) {
    a0 = T.vid[it];
    a1 = T.vid[kTile + it];
    a2 = T.vid[2 * kTile + it];
    if (NM != kNearInKernel && moff >= 0)
      mword = __ldg(near.masks + static_cast<int64_t>(moff) * kTile + it);
  }
  for (int js = warp; js < nsj; js += kWarps) {  // warp-uniform trip count
    double ore[NBT][NBS], oim[NBT][NBS];
    double otr[NBT][NBS], oti[NBT][NBS];  // PAIRED: the (sy, tx) block, [test-tile
                                          // basis][trial-tile basis], real and imaginary
    bool have = false;
    if (lane_cell) {
      const int64_t o = static_cast<int64_t>(sj0 + js) * ld + ti0 + it;
      const bool skip = NM == kNearMasked
                            ? ((mword >> js) & 1u) != 0u
                            : same_grid && share_vertex(a0, a1, a2, S.vid[js], S.vid[kTile + js],
                                                        S.vid[2 * kTile + js]);
      if (skip) {
        // DP0: a vertex-sharing entry is written here (zero) and then by the singular
        // kernel; the masked entries of the mixed path are written by the near-pair and
        // singular kernels alone (which may run concurrently with this one)
        if (DIRECT && NM == kNearInKernel) {
          if (kC)
            reinterpret_cast<double2*>(out)[o] = make_double2(0.0, 0.0);
          else
            out[o] = 0.0;
          if (mirror) mirror_put<kC>(mir, it, js, 0.0, 0.0);
        }
      } else if (kQueue && near_pair(T, it, S, js)) {
        const int slot = atomicAdd(qcount, 1);
        queue[slot] = static_cast<unsigned short>(it | (js << 8));
      } else {
        if constexpr (PAIRED && MIXED) {
          // far pair, FP32 (near and vertex-sharing pairs are masked)
          if (OP == kDL)
            block_fp32_dl_pair<QT, KER>(T, it, S, js, rule, k, ore, oim, otr, oti);
          else
            block_fp32_dl_pair<QT, KER>(T, it, S, js, rule, k, otr, oti, ore, oim);
        } else if constexpr (PAIRED) {
          // DL: (i, j) block here, (j, i) at the transposed entries; ADL: swapped
          if constexpr (KER == kLaplace) {
#pragma unroll
            for (int a = 0; a < NBT; ++a)
#pragma unroll
              for (int b = 0; b < NBS; ++b) oim[a][b] = oti[a][b] = 0.0;  // real blocks
            if (OP == kDL)
              block_fp64_dl_pair<QT>(T, it, S, js, rule, ore, otr);
            else
              block_fp64_dl_pair<QT>(T, it, S, js, rule, otr, ore);
          } else {
            if (OP == kDL)
              block_fp64_dl_pair_helmholtz<QT>(T, it, S, js, rule, k, ore, oim, otr, oti);
            else
              block_fp64_dl_pair_helmholtz<QT>(T, it, S, js, rule, k, otr, oti, ore, oim);
          }
        } else if (MIXED) {
          block_fp32<QT, KER, OP, NBT, NBS, PH>(T, it, S, js, rule, k, ore, oim);
        } else {
          block_fp64<QT, KER, OP, NBT, NBS, true,
                     PH == kPhaseSmall ? kF64Referenced : kF64Sincos>(T, it, S, js, rule, k, ore, oim);
        }
        have = true;
        if (DIRECT) {
          if (kC)
            reinterpret_cast<double2*>(out)[o] = make_double2(ore[0][0], oim[0][0]);
          else
            out[o] = ore[0][0];
          if (mirror) mirror_put<kC>(mir, it, js, ore[0][0], oim[0][0]);
        } else if (!kGather) {
          deposit<NBT, NBS, kC>(acc_re, acc_im, ndt, T, it, S, js, ore, oim);
        }
      }
    }
    // PAIRED off the diagonal: a second block gathers the (sy, tx) blocks into acc_t;
    // kSplitStage: each block in two passes, real then imaginary parts
    constexpr int kParts = kSplitStage ? 2 : 1;
#pragma unroll 1
    for (int pass = 0; pass < ((PAIRED && mirror) ? 2 : (kGather ? 1 : 0)) * kParts; ++pass) {
      const int blk = pass / kParts, part = pass % kParts;
      double* sr = stage_re + warp * (kTile * NBT * NBS);
      double* si = stage_im + warp * (kTile * NBT * NBS);
      double* acc = blk == 0 ? (part == 0 ? acc_re : acc_im) : (part == 0 ? acc_t : acc_t + cap);
      double* acci = blk == 0 ? acc_im : acc_t + cap;
#pragma unroll
      for (int a = 0; a < NBT; ++a)
#pragma unroll
        for (int b = 0; b < NBS; ++b) {
          const double re = blk == 0 ? ore[a][b] : otr[a][b];
          const double im = blk == 0 ? oim[a][b] : oti[a][b];
          sr[(a * NBS + b) * kTile + it] = have ? (part == 0 ? re : im) : 0.0;
          if (kC && !kSplitStage) si[(a * NBS + b) * kTile + it] = have ? im : 0.0;
        }
      __syncwarp();
      for (int d = it; d < ndt; d += kTile) {
        double g_re[NBS], g_im[NBS];
#pragma unroll
        for (int b = 0; b < NBS; ++b) g_re[b] = g_im[b] = 0.0;
        for (int e = inc_off[d]; e < inc_off[d + 1]; ++e) {
          const int ab = inc_ent[e];  // a * kTile + cell
          const int a = ab >> 5, c = ab & (kTile - 1);
#pragma unroll
          for (int b = 0; b < NBS; ++b) {
            g_re[b] += sr[(a * NBS + b) * kTile + c];
            if (kC && !kSplitStage) g_im[b] += si[(a * NBS + b) * kTile + c];
          }
        }
#pragma unroll
        for (int b = 0; b < NBS; ++b) {
          const int idx = d + ndt * S.ldof[b * kTile + js];
          if (kAcc > 1) {
            acc[warp * cap + idx] += g_re[b];  // this warp's copy; distinct per lane
          } else {
            atomicAdd(acc + idx, g_re[b]);
            if (kC && !kSplitStage) atomicAdd(acci + idx, g_im[b]);
          }
        }
      }
      __syncwarp();
    }
  }
  if (kQueue) {
    __syncthreads();
    const int nq = *qcount;
    for (int e = threadIdx.x; e < nq; e += kThreads) {
      const int pi = queue[e] & 0xff, pj = queue[e] >> 8;
      double ore[NBT][NBS], oim[NBT][NBS];
      block_fp64<QT, KER, OP, NBT, NBS, false>(T, pi, S, pj, rule, k, ore, oim);
      if (DIRECT) {
        const int64_t o = static_cast<int64_t>(sj0 + pj) * ld + ti0 + pi;
        if (kC)
          reinterpret_cast<double2*>(out)[o] = make_double2(ore[0][0], oim[0][0]);
        else
          out[o] = ore[0][0];
        if (mirror) mirror_put<kC>(mir, pi, pj, ore[0][0], oim[0][0]);
      } else {
        deposit<NBT, NBS, kC>(acc_re, acc_im, ndt, T, pi, S, pj, ore, oim);
      }
    }
  }
  if (DIRECT && mirror) {
    // the transposed block, entry (row sj0 + j, column ti0 + i), j fastest: coalesced
    __syncthreads();
    for (int idx = threadIdx.x; idx < kTile * kTile; idx += kThreads) {
      const int i = idx / kTile, j = idx % kTile;
      if (i >= nti || j >= nsj) continue;
      if (NM == kNearMasked && moff >= 0 &&
          ((__ldg(near.masks + static_cast<int64_t>(moff) * kTile + i) >> j) & 1u))
        continue;  // a near or vertex-sharing pair: written by the near-pair / singular kernels
      const int64_t o = static_cast<int64_t>(ti0 + i) * ld + sj0 + j;
      if (kC)
        reinterpret_cast<double2*>(out)[o] =
            make_double2(mir[2 * (j * (kTile + 1) + i)], mir[2 * (j * (kTile + 1) + i) + 1]);
      else
        out[o] = mir[j * (kTile + 1) + i];
    }
  }
  if (!DIRECT) {
    __syncthreads();
    const int* tdofs = tt.tile_dofs + tdof0;
    const int* sdofs = st.tile_dofs + sdof0;
    for (int idx = threadIdx.x; idx < ndt * nds; idx += kThreads) {
      const int a = idx % ndt, b = idx / ndt;
      const int64_t o = static_cast<int64_t>(sdofs[b]) * ld + tdofs[a];
      double re = acc_re[idx];
#pragma unroll
      for (int w = 1; w < kAcc; ++w) re += acc_re[w * cap + idx];
      // symmetric, tx > sy: the same value at the transposed entry
      const int64_t om = static_cast<int64_t>(tdofs[a]) * ld + sdofs[b];
      if (kC && PAIRED) {
        const double im = acc_im[idx];
        if (re != 0.0 || im != 0.0) {
          atomicAdd(out + 2 * o, re);
          atomicAdd(out + 2 * o + 1, im);
        }
        const double tre = acc_t[idx], tim = acc_t[cap + idx];
        if (mirror && (tre != 0.0 || tim != 0.0)) {
          atomicAdd(out + 2 * om, tre);
          atomicAdd(out + 2 * om + 1, tim);
        }
      } else if (kC) {
        const double im = acc_im[idx];
        if (re != 0.0 || im != 0.0) {
          atomicAdd(out + 2 * o, re);
          atomicAdd(out + 2 * o + 1, im);
          if (mirror) {
            atomicAdd(out + 2 * om, re);
            atomicAdd(out + 2 * om + 1, im);
          }
        }
      } else if (PAIRED) {
        if (re != 0.0) atomicAdd(out + o, re);
        if (mirror && acc_t[idx] != 0.0) atomicAdd(out + om, acc_t[idx]);
      } else if (re != 0.0) {
        atomicAdd(out + o, re);
        if (mirror) atomicAdd(out + om, re);
      }
    }
  }
}

// FP64 near pairs of a mixed-precision assembly: one thread per pair of the near list
// (test cell, trial cell), each staging its two cells into its own column of a per-warp
// pair of shared-memory tiles and integrating them with block_fp64 (phases referenced to
// the pair, or the in-tree reduced sincos: FPH).
// Only pairs whose trial cell lies in [trial_lo, trial_hi) (a chunk) are done.  DP0 x DP0
// entries are stored; other spaces add into the output with atomics.
template <int QT, int KER, int OP, int NBT, int NBS, bool DIRECT, int FPH>
__global__ void __launch_bounds__(kThreads)
    near_pairs_fp64(CellSet test, CellSet trial, RegularRule rule, double k, NearArgs near,
                    double* __restrict__ out, int64_t ld, int trial_lo, int trial_hi) {
  constexpr bool kC = KER == kHelmholtz;
  const int Q = QT > 0 ? QT : rule.npts;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;  // blockDim.x = 32 x warps
  unsigned char* cursor = smem + static_cast<size_t>(warp) * 2 *
                                     (sizeof(double) * tile_doubles(Q) + sizeof(int) * tile_ints(1) + 16);
  const Tile T = carve_tile(cursor, Q, false, 1);
  const Tile S = carve_tile(cursor, Q, false, 1);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= near.npairs) return;
  const int2 pr = __ldg(near.pairs + e);
  if (pr.y < trial_lo || pr.y >= trial_hi) return;
  stage_cell(T, lane, test, pr.x, Q);  // this lane's column only: no synchronisation
  stage_cell(S, lane, trial, pr.y, Q);
  double ore[NBT][NBS], oim[NBT][NBS];
  block_fp64<QT, KER, OP, NBT, NBS, false, FPH>(T, lane, S, lane, rule, k, ore, oim);
  if (DIRECT) {
    const int64_t o = static_cast<int64_t>(pr.y) * ld + pr.x;
    if (kC)
      reinterpret_cast<double2*>(out)[o] = make_double2(ore[0][0], oim[0][0]);
    else
      out[o] = ore[0][0];
  } else {
#pragma unroll
    for (int b = 0; b < NBS; ++b) {
      const int64_t col = static_cast<int64_t>(__ldg(near.trial_dofs + pr.y * NBS + b)) * ld;
#pragma unroll
      for (int a = 0; a < NBT; ++a) {
        const int64_t o = col + __ldg(near.test_dofs + pr.x * NBT + a);
        if (kC) {
          atomicAdd(out + 2 * o, ore[a][b]);
          atomicAdd(out + 2 * o + 1, oim[a][b]);
        } else {
          atomicAdd(out + o, ore[a][b]);
        }
      }
    }
  }
}

// ------------------------------------------------------------------------------------
// Batched Helmholtz single-layer DP0 sweep over many wavenumbers and meshes.
//
// One persistent launch for the far pairs: every CTA repeatedly takes the next work item
// (mesh, chunk of wavenumbers, super-tile pair) from a global counter (items of the
// largest mesh first), stages the tiles once, and for each wavenumber of its chunk writes
// the far-pair entries of its 32 x 32 blocks in FP32 (block_fp32), complex64.  The pairs
// the mesh's near field marks (centroid distance below twice the larger diameter, or a
// shared vertex: the same masks as the one-off mixed assembly) are left to two FP64
// launches that run beside it (forked in the same captured graph): near pairs by the
// 6-point rule with the pair-referenced phase, vertex-sharing pairs by their Duffy rules.
// The single layer is symmetric on one mesh, so only tile pairs (test tile >= trial tile)
// are items: an off-diagonal block is also written transposed (through shared memory,
// coalesced).  No two launches or items write the same entry, so nothing orders them;
// the only shared state is the item counter (reset before every launch).

// TS: tile shape of a work item, TS x TS tiles of 32 cells on each side (a super-tile
// pair: 1 x 1 or 2 x 2 tile pairs staged together); MINB: CTAs per SM the register
// allocation must allow (4: up to 128 registers, 6: up to 80).  Far pairs only: the pairs
// marked in the mesh's near-field masks (near or vertex-sharing) are written by
// sweep_near_fp64 / sweep_duffy_fp64.
template <int TS, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    sweep_sl_dp0(SweepArgs a, RegularRule rule) {
  const int Q = 6;
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);  // completion of the tile copies
  unsigned char* cursor = smem + 16;
  Tile Tt[TS], St[TS];
#pragma unroll
  for (int i = 0; i < TS; ++i) Tt[i] = carve_tile(cursor, Q, true, 1, false);
#pragma unroll
  for (int i = 0; i < TS; ++i) St[i] = carve_tile(cursor, Q, true, 1, false);
  long long* s_item = reinterpret_cast<long long*>(cursor);
  float2* mir = reinterpret_cast<float2*>(s_item + 2);  // [js * (kTile + 1) + it]
  unsigned* skip = reinterpret_cast<unsigned*>(mir + kTile * (kTile + 1));  // [it]: bit js
  const int it = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) mbar_init(mbar, 1);
  unsigned phase = 0;  // parity of the mbarrier phase of the current item's copies
  for (;;) {
    if (threadIdx.x == 0) *s_item = static_cast<long long>(atomicAdd(a.counter, 1ull));
    __syncthreads();
    const long long item = *s_item;
    if (item >= a.nitems) break;
    int m = 0;
    while (m + 1 < a.nmesh && item >= a.mesh[m + 1].item_begin) ++m;
    const SweepMesh& M = a.mesh[m];
    const long long local = item - M.item_begin;
    // wavenumber chunk outermost: the items resident at one time write one output
    // matrix (one chunk of them), in the banded order of the super-tile pairs
    const int nsup = (M.ntiles + TS - 1) / TS;
    const long long npairs = lower_tile_pair_count(nsup, 0, nsup);
    const int kc = static_cast<int>(local / npairs);
    int TT, ST;
    lower_tile_pair(local % npairs, nsup, 0, nsup, TT, ST);
    const int nc = M.cells.ncells;
    // every tile of the two super-tiles by bulk (TMA) copies on the mbarrier (no FP64
    // points: the far pairs use the FP32 offsets); the previous item's reads of the tiles
    // ended at the barriers that closed it
    if (threadIdx.x == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      unsigned bytes = 0;
      for (int i = 0; i < TS; ++i) {
        if (TS * TT + i < M.ntiles) bytes += bulk_tile_bytes(Q, true, false);
        if (TS * ST + i < M.ntiles) bytes += bulk_tile_bytes(Q, true, false);
      }
      mbar_expect_tx(mbar, bytes);
      for (int i = 0; i < TS; ++i) {
        if (TS * TT + i < M.ntiles)
          stage_tile_bulk(Tt[i], M.cells, (TS * TT + i) * kTile, Q, true, mbar, false);
        if (TS * ST + i < M.ntiles)
          stage_tile_bulk(St[i], M.cells, (TS * ST + i) * kTile, Q, true, mbar, false);
      }
    }
    const bool staged = mbar_wait_bounded(mbar, phase);
    phase ^= 1u;
    if (__syncthreads_or(!staged)) {
      // the copies did not complete in time (never expected): record it, give them a last
      // bounded wait and stop this CTA (the item's entries stay unwritten; the host's
      // completion check reports it)
      if (threadIdx.x == 0) atomicAdd(&g_stage_timeouts, 1u);
      mbar_wait_bounded(mbar, phase ^ 1u);
      return;
    }
#pragma unroll 1
    for (int sub = 0; sub < TS * TS; ++sub) {
      const int tt = TS * TT + sub / TS, st = TS * ST + sub % TS;
      if (tt >= M.ntiles || st >= M.ntiles || tt < st) continue;  // block-uniform
      const Tile& T = Tt[sub / TS];
      const Tile& S = St[sub % TS];
      const bool mirror = tt > st;
      const int ti0 = tt * kTile, sj0 = st * kTile;
      const int nti = min(kTile, nc - ti0), nsj = min(kTile, nc - sj0);
      // the near and vertex-sharing pairs of this tile pair (the relation is symmetric, so
      // the same bits mark the transposed block)
      const int moff = __ldg(M.tile_mask + static_cast<int64_t>(tt) * M.ntiles + st);
      if (threadIdx.x < kTile)
        skip[threadIdx.x] = moff >= 0 ? __ldg(M.masks + static_cast<int64_t>(moff) * kTile + threadIdx.x) : 0u;
      __syncthreads();
      const unsigned skip_it = it < nti ? skip[it] : ~0u;
      const int k0 = kc * a.kchunk, k1 = min(a.nk, k0 + a.kchunk);
      for (int kk = k0; kk < k1; ++kk) {
        const double k = a.ks[kk];
        float2* out = M.out + static_cast<long long>(kk) * nc * nc;
        if (it < nti) {
          for (int js = warp; js < nsj; js += kWarps) {
            if ((skip_it >> js) & 1u) continue;
            double ore[1][1], oim[1][1];
            block_fp32<6, kHelmholtz, kSL, 1, 1, kPhaseRuntime>(T, it, S, js, rule, k, ore, oim);
            const float2 v = make_float2(static_cast<float>(ore[0][0]), static_cast<float>(oim[0][0]));
            out[static_cast<long long>(sj0 + js) * nc + ti0 + it] = v;
            if (mirror) mir[js * (kTile + 1) + it] = v;
          }
        }
        if (mirror) {
          // the transposed block, entry (row sj0 + j, column ti0 + i), j fastest: coalesced
          __syncthreads();
          for (int idx = threadIdx.x; idx < kTile * kTile; idx += kThreads) {
            const int i = idx / kTile, j = idx % kTile;
            if (i < nti && j < nsj && !((skip[i] >> j) & 1u))
              out[static_cast<long long>(ti0 + i) * nc + sj0 + j] = mir[j * (kTile + 1) + i];
          }
          __syncthreads();  // mir is reused by the next wavenumber
        }
      }
      __syncthreads();  // the skip words are reused by the next tile pair
    }
  }
}

// Single-layer DP0 entry of one cell pair (test i, trial j) by the 6-point rule in FP64,
// points and geometry from the grid arrays: phase referenced to the pair when
// k (rad_i + rad_j) <= 0.8, else sincos_cw.
__device__ double2 sl_dp0_pair_fp64(const CellSet& cs, int i, int j, const RegularRule& rule,
                                    double k) {
  const int64_t S = cs.stride;
  const double dcx = g(cs.geom, kCx, cs.stride, i) - g(cs.geom, kCx, cs.stride, j);
  const double dcy = g(cs.geom, kCy, cs.stride, i) - g(cs.geom, kCy, cs.stride, j);
  const double dcz = g(cs.geom, kCz, cs.stride, i) - g(cs.geom, kCz, cs.stride, j);
  const bool ref = k * (g(cs.geom, kRad, cs.stride, i) + g(cs.geom, kRad, cs.stride, j)) <=
                   static_cast<double>(kSmallPhaseMax);
  double kr0 = 0.0, pc = 1.0, ps = 0.0;
  if (ref) {
    const double r0sq = dcx * dcx + dcy * dcy + dcz * dcz;
    kr0 = k * (r0sq * rsqrt_refined(r0sq));
    sincos_cw(kr0, ps, pc);
  }
  double yq[6][3];
#pragma unroll
  for (int q = 0; q < 6; ++q)
#pragma unroll
    for (int d = 0; d < 3; ++d) yq[q][d] = __ldg(cs.qpts + (q * 3 + d) * S + j);
  double re = 0.0, im = 0.0;
#pragma unroll 1
  for (int p = 0; p < 6; ++p) {
    const double x0 = __ldg(cs.qpts + (p * 3) * S + i), x1 = __ldg(cs.qpts + (p * 3 + 1) * S + i),
                 x2 = __ldg(cs.qpts + (p * 3 + 2) * S + i);
    double ur = 0.0, ui = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const double dx = x0 - yq[q][0], dy = x1 - yq[q][1], dz = x2 - yq[q][2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double rinv = rsqrt_refined(r2);
      const double r = r2 * rinv;
      double sn, cs_;
      if (ref)
        sincos_small(fma(k, r, -kr0), sn, cs_);
      else
        sincos_cw(k * r, sn, cs_);
      const double f = rule.w[q] * rinv;
      ur = fma(f, cs_, ur);
      ui = fma(f, sn, ui);
    }
    re = fma(rule.w[p], ur, re);
    im = fma(rule.w[p], ui, im);
  }
  const double sc = g(cs.geom, kJdet, cs.stride, i) * g(cs.geom, kJdet, cs.stride, j) * kInv4Pi;
  return make_double2((re * pc - im * ps) * sc, (re * ps + im * pc) * sc);
}

// The near pairs (no shared vertex) of every mesh and wavenumber: one thread per (pair,
// wavenumber), wavenumber fastest.
__global__ void __launch_bounds__(kThreads)
    sweep_near_fp64(SweepArgs a, RegularRule rule) {
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= a.near_begin[a.nmesh]) return;
  int m = 0;
  while (m + 1 < a.nmesh && t >= a.near_begin[m + 1]) ++m;
  const SweepMesh& M = a.mesh[m];
  const long long local = t - a.near_begin[m];
  const int e = static_cast<int>(local / a.nk), kk = static_cast<int>(local % a.nk);
  const int2 pr = __ldg(M.near_pairs + e);
  const double2 v = sl_dp0_pair_fp64(M.cells, pr.x, pr.y, rule, a.ks[kk]);
  const int nc = M.cells.ncells;
  M.out[static_cast<long long>(kk) * nc * nc + static_cast<long long>(pr.y) * nc + pr.x] =
      make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
}

// The vertex-sharing pairs of every mesh and wavenumber by their Duffy rules: one warp
// per (pair, wavenumber), wavenumber fastest; lanes over the rule's points.
__global__ void __launch_bounds__(kThreads)
    sweep_duffy_fp64(SweepArgs a, SingularRules rules) {
  const long long w = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= a.sing_begin[a.nmesh]) return;  // warp-uniform
  int m = 0;
  while (m + 1 < a.nmesh && w >= a.sing_begin[m + 1]) ++m;
  const SweepMesh& M = a.mesh[m];
  const long long local = w - a.sing_begin[m];
  const int e = static_cast<int>(local / a.nk), kk = static_cast<int>(local % a.nk);
  const double k = a.ks[kk];
  const CellSet& cs = M.cells;
  const int tc = __ldg(M.sing.test_cell + e), sc = __ldg(M.sing.trial_cell + e);
  const int cfg = __ldg(M.sing.config + e);
  double t0x[3], t1x[3], t0y[3], t1y[3], dv[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    t0x[d] = g(cs.geom, kT0x + d, cs.stride, tc);
    t1x[d] = g(cs.geom, kT1x + d, cs.stride, tc);
    t0y[d] = g(cs.geom, kT0x + d, cs.stride, sc);
    t1y[d] = g(cs.geom, kT1x + d, cs.stride, sc);
    dv[d] = g(cs.geom, kV0x + d, cs.stride, tc) - g(cs.geom, kV0x + d, cs.stride, sc);
  }
  const int off = __ldg(rules.offset + cfg), npts = __ldg(rules.offset + cfg + 1) - off;
  // |k r| <= k (diam_x + diam_y): no reduction of the phase when that is below pi/4
  const bool small_phase =
      k * (g(cs.geom, kDiam, cs.stride, tc) + g(cs.geom, kDiam, cs.stride, sc)) <= 0.78;
  const double2* txi = reinterpret_cast<const double2*>(rules.test_xi);
  const double2* sxi = reinterpret_cast<const double2*>(rules.trial_xi);
  double sr = 0.0, si = 0.0;
  for (int ii = lane; ii < npts; ii += 32) {
    const int i = off + ii;
    const double2 xi = __ldg(txi + i), et = __ldg(sxi + i);
    const double wt = __ldg(rules.w + i);
    double r2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double dd = fma(xi.x, t0x[d], fma(xi.y, t1x[d], fma(-et.x, t0y[d], fma(-et.y, t1y[d], dv[d]))));
      r2 = fma(dd, dd, r2);
    }
    const double rinv = rsqrt_refined(r2);
    double sn, cs_;
    if (small_phase)
      sincos_taylor(k * r2 * rinv, sn, cs_);
    else
      sincos_cw(k * r2 * rinv, sn, cs_);
    sr = fma(wt * rinv, cs_, sr);
    si = fma(wt * rinv, sn, si);
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, s);
    si += __shfl_xor_sync(0xffffffffu, si, s);
  }
  if (lane == 0) {
    const double scl = g(cs.geom, kJdet, cs.stride, tc) * g(cs.geom, kJdet, cs.stride, sc) * kInv4Pi;
    const int nc = cs.ncells;
    M.out[static_cast<long long>(kk) * nc * nc + static_cast<long long>(sc) * nc + tc] =
        make_float2(static_cast<float>(sr * scl), static_cast<float>(si * scl));
  }
}

size_t smem_bytes(int q, bool rel, bool queue, bool direct, bool cplx, int max_t, int max_s,
                  int nbt, int nbs, int acc_copies, bool mirror, bool pts, bool split_stage) {
  size_t b = 16;  // the mbarrier
  if (!direct) b += sizeof(double) * static_cast<size_t>(max_t) * max_s * (cplx ? 2 : 1) * acc_copies;
  if (direct && mirror) b += sizeof(double) * kTile * (kTile + 1) * (cplx ? 2 : 1) + 16;
  if (!direct && nbt == 3)  // stage and DOF incidence of the gather
    b += sizeof(double) * kWarps * kTile * nbt * nbs * ((cplx && !split_stage) ? 2 : 1) +
         6 * kTile + 1;
  for (int nb : {nbt, nbs}) {
    b = (b + 15) & ~size_t(15);
    b += sizeof(double) * tile_doubles(q, pts) + sizeof(float) * tile_floats(q, rel) +
         sizeof(int) * tile_ints(nb);
    b = (b + 15) & ~size_t(15);
  }
  if (queue) b += sizeof(unsigned short) * kTile * kTile + sizeof(int);
  return b + 16;
}

template <int QT, int KER, int OP, int NBT, int NBS, bool MIXED, bool DIRECT, int PH, int NM,
          bool PAIRED = false>
cudaError_t launch_mode(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                        const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                        int ty0, int ty1, cudaStream_t stream) {
  // accumulator copies: one per warp for the real FP64 P1 blocks; PAIRED: one for the
  // (tx, sy) and one for the (sy, tx) blocks
  constexpr int kAcc = PAIRED ? 2
                              : (!DIRECT && NBT == 3 && KER != kHelmholtz && !MIXED && OP != kHS)
                                    ? kWarps
                                    : 1;
  auto bytes = [&](int copies) {
    return smem_bytes(rule.npts, MIXED, MIXED && NM == kNearInKernel, DIRECT, KER == kHelmholtz,
                      tt.max_tile_dofs, st.max_tile_dofs, NBT, NBS, copies, a.symmetric != 0,
                      !MIXED || NM == kNearInKernel,
                      !DIRECT && NBT == 3 && KER == kHelmholtz && PAIRED && MIXED);
  };
  int copies = kAcc;
  size_t smem = bytes(copies);
  if (copies == kWarps) {
    int device = 0, limit = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    if (smem > static_cast<size_t>(limit)) {  // one shared accumulator, atomic adds
      copies = 1;
      smem = bytes(1);
    }
  }
  auto fn = regular_tiles<QT, KER, OP, NBT, NBS, MIXED, DIRECT, PH, NM, PAIRED>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) {
    cudaGetLastError();  // not sticky: clear it, so that it is not reported by a later launch
    return e;
  }
  const int ntt = (test.ncells + kTile - 1) / kTile;
  dim3 grid(ntt, ty1 - ty0);
  if (a.symmetric) {
    // tile pairs (tx >= sy) of trial tiles [ty0, ty1), in bands of trial tiles
    const long long count = lower_tile_pair_count(ntt, ty0, ty1);
    if (count > 0x7fffffffLL) return cudaErrorInvalidValue;
    grid = dim3(static_cast<unsigned>(count), 1);
  }
  fn<<<grid, kThreads, smem, stream>>>(test, tt, trial, st, rule, a.k, a.same_grid,
                                       static_cast<double*>(a.out), a.ld, ty0, ty1, a.near,
                                       a.symmetric, copies);
  return cudaGetLastError();
}

template <int QT, int KER, int OP, int NBT, int NBS, bool DIRECT>
cudaError_t launch_near_pairs(const CellSet& test, const CellSet& trial, const RegularRule& rule,
                              const RegularArgs& a, int ty0, int ty1, cudaStream_t stream) {
  if (a.near.npairs <= 0) return cudaSuccess;
  if (!DIRECT && (!a.near.test_dofs || !a.near.trial_dofs)) return cudaErrorInvalidValue;
  // two tiles per warp (each lane stages its own column); up to 4 warps within 200 KB
  const size_t per_warp = 2 * (sizeof(double) * tile_doubles(rule.npts) + sizeof(int) * tile_ints(1) + 16);
  const int warps = static_cast<int>(std::max<size_t>(1, std::min<size_t>(kWarps, (200u << 10) / per_warp)));
  const size_t smem = warps * per_warp + 16;
  // phases referenced to the pair when the launch's bound k (rad_x + rad_y) <= 0.8 holds
  auto fn = a.small_phase ? near_pairs_fp64<QT, KER, OP, NBT, NBS, DIRECT, kF64Referenced>
                          : near_pairs_fp64<QT, KER, OP, NBT, NBS, DIRECT, kF64Reduced>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) {
    cudaGetLastError();  // not sticky: clear it, so that it is not reported by a later launch
    return e;
  }
  const int threads = 32 * warps;
  const int blocks = (a.near.npairs + threads - 1) / threads;
  const int lo = ty0 * kTile;
  const int hi = ty1 * kTile >= trial.ncells ? 0x7fffffff : ty1 * kTile;
  fn<<<blocks, threads, smem, stream>>>(test, trial, rule, a.k, a.near,
                                        static_cast<double*>(a.out), a.ld, lo, hi);
  return cudaGetLastError();
}

template <int QT, int KER, int OP, int NBT, int NBS, bool MIXED, bool DIRECT>
cudaError_t launch_one(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                       const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                       cudaStream_t stream) {
  const int trial_tiles = (trial.ncells + kTile - 1) / kTile;
  if (a.trial_tile0 < 0 || a.trial_tile0 > trial_tiles || a.trial_tiles < 0)
    return cudaErrorInvalidValue;
  const int ny = a.trial_tiles > 0 ? std::min(a.trial_tiles, trial_tiles - a.trial_tile0)
                                   : trial_tiles - a.trial_tile0;
  if (ny <= 0) return cudaSuccess;
  const int ty0 = a.trial_tile0, ty1 = a.trial_tile0 + ny;
  if constexpr (!MIXED) {
    if (a.symmetric == 2) {
      // one P1 / DP1 space, DL / ADL: both orders of each pair from one kernel evaluation
      // (the host asks for it only there, for Helmholtz only with phases referenced to the
      // pair)
      if constexpr ((OP == kDL || OP == kADL) && NBT == 3 && NBS == 3 && !DIRECT && QT == 6) {
        if (KER == kHelmholtz && !a.small_phase) return cudaErrorInvalidValue;
        return launch_mode<QT, KER, OP, NBT, NBS, false, DIRECT, kPhaseSmall, kNearInKernel, true>(
            test, tt, trial, st, rule, a, ty0, ty1, stream);
      } else {
        return cudaErrorInvalidValue;
      }
    }
    // FP64 Helmholtz: phases referenced to the pair (kPhaseSmall) when the host's bound
    // allows it, else CUDA's sincos of every phase
    if (KER == kHelmholtz && !a.small_phase)
      return launch_mode<QT, KER, OP, NBT, NBS, false, DIRECT, kPhaseGeneral, kNearInKernel>(
          test, tt, trial, st, rule, a, ty0, ty1, stream);
    return launch_mode<QT, KER, OP, NBT, NBS, false, DIRECT, kPhaseSmall, kNearInKernel>(
        test, tt, trial, st, rule, a, ty0, ty1, stream);
  } else {
    if (!a.near.tile_mask) {
      // no near field: pairs tested in the kernel (DP0 only; the assembler always builds one)
      if constexpr (DIRECT) {
        if (KER == kHelmholtz && !a.small_phase)
          return launch_mode<QT, KER, OP, NBT, NBS, true, DIRECT, kPhaseGeneral, kNearInKernel>(
              test, tt, trial, st, rule, a, ty0, ty1, stream);
        return launch_mode<QT, KER, OP, NBT, NBS, true, DIRECT, kPhaseSmall, kNearInKernel>(
            test, tt, trial, st, rule, a, ty0, ty1, stream);
      } else {
        return cudaErrorInvalidValue;
      }
    }
    if (a.near.trial_tiles != trial_tiles) return cudaErrorInvalidValue;
    cudaError_t e;
    if (a.symmetric == 2) {
      // one P1 / DP1 space, DL / ADL: both orders of each far pair from one kernel
      // evaluation (Helmholtz only with phases within the polynomial range)
      if constexpr ((OP == kDL || OP == kADL) && NBT == 3 && NBS == 3 && !DIRECT && QT == 6) {
        if (KER == kHelmholtz && !a.small_phase) return cudaErrorInvalidValue;
        e = launch_mode<QT, KER, OP, NBT, NBS, true, DIRECT, kPhaseSmall, kNearMasked, true>(
            test, tt, trial, st, rule, a, ty0, ty1, stream);
        if (e != cudaSuccess) return e;
        return launch_near_pairs<QT, KER, OP, NBT, NBS, DIRECT>(test, trial, rule, a, ty0, ty1,
                                                                stream);
      } else {
        return cudaErrorInvalidValue;
      }
    }
    // the launch-wide bound failed: each warp still takes the unreduced polynomial phase
    // when its own pairs allow it (most pairs of a mesh whose largest cells set the bound)
    if (KER == kHelmholtz && !a.small_phase)
      e = launch_mode<QT, KER, OP, NBT, NBS, true, DIRECT, kPhaseRuntime, kNearMasked>(
          test, tt, trial, st, rule, a, ty0, ty1, stream);
    else
      e = launch_mode<QT, KER, OP, NBT, NBS, true, DIRECT, kPhaseSmall, kNearMasked>(
          test, tt, trial, st, rule, a, ty0, ty1, stream);
    if (e != cudaSuccess) return e;
    return launch_near_pairs<QT, KER, OP, NBT, NBS, DIRECT>(test, trial, rule, a, ty0, ty1, stream);
  }
}

template <int QT, int KER, int OP, bool MIXED>
cudaError_t launch_spaces(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                          const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                          cudaStream_t stream, bool direct) {
  if (direct) {
    if (OP == kHS) return cudaErrorInvalidValue;
    return launch_one<QT, KER, OP == kHS ? kSL : OP, 1, 1, MIXED, true>(test, tt, trial, st, rule, a, stream);
  }
  if (tt.nbasis == 1 && st.nbasis == 1)
    return launch_one<QT, KER, OP, 1, 1, MIXED, false>(test, tt, trial, st, rule, a, stream);
  if (tt.nbasis == 1 && st.nbasis == 3)
    return launch_one<QT, KER, OP, 1, 3, MIXED, false>(test, tt, trial, st, rule, a, stream);
  if (tt.nbasis == 3 && st.nbasis == 1)
    return launch_one<QT, KER, OP, 3, 1, MIXED, false>(test, tt, trial, st, rule, a, stream);
  if (tt.nbasis == 3 && st.nbasis == 3)
    return launch_one<QT, KER, OP, 3, 3, MIXED, false>(test, tt, trial, st, rule, a, stream);
  if constexpr (!MIXED && KER == kLaplace && OP != kHS) {
    // degree 2 on both sides (P2 / DP2), FP64
    if (tt.nbasis == 6 && st.nbasis == 6)
      return launch_one<QT, KER, OP, 6, 6, false, false>(test, tt, trial, st, rule, a, stream);
  }
  return cudaErrorInvalidValue;
}

template <int QT, int KER, bool MIXED>
cudaError_t launch_op(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                      const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                      cudaStream_t stream, bool direct) {
  switch (a.op) {
    case kSL: return launch_spaces<QT, KER, kSL, MIXED>(test, tt, trial, st, rule, a, stream, direct);
    case kDL: return launch_spaces<QT, KER, kDL, MIXED>(test, tt, trial, st, rule, a, stream, direct);
    case kADL: return launch_spaces<QT, KER, kADL, MIXED>(test, tt, trial, st, rule, a, stream, direct);
    case kHS: return launch_spaces<QT, KER, kHS, MIXED>(test, tt, trial, st, rule, a, stream, direct);
    default: return cudaErrorInvalidValue;
  }
}

template <int QT, bool MIXED>
cudaError_t launch_kernel(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                          const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                          cudaStream_t stream, bool direct) {
  return a.kernel == kLaplace
             ? launch_op<QT, kLaplace, MIXED>(test, tt, trial, st, rule, a, stream, direct)
             : launch_op<QT, kHelmholtz, MIXED>(test, tt, trial, st, rule, a, stream, direct);
}

cudaError_t dispatch(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                     const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                     cudaStream_t stream, bool direct) {
  if (test.ncells <= 0 || trial.ncells <= 0) return cudaSuccess;
  const bool mixed = a.precision == kRegularMixed;
  if (rule.npts == 6)
    return mixed ? launch_kernel<6, true>(test, tt, trial, st, rule, a, stream, direct)
                 : launch_kernel<6, false>(test, tt, trial, st, rule, a, stream, direct);
  return mixed ? launch_kernel<0, true>(test, tt, trial, st, rule, a, stream, direct)
               : launch_kernel<0, false>(test, tt, trial, st, rule, a, stream, direct);
}

}  // namespace

int scatter_tile_cells() { return kTile; }

namespace {
int g_host_poll_limit = tiles::kStagePolls;  // host copy of g_stage_poll_limit
}  // namespace

cudaError_t set_stage_poll_limit(int polls) {
  g_host_poll_limit = polls;
  return cudaMemcpyToSymbol(g_stage_poll_limit, &polls, sizeof(int));
}

cudaError_t stage_wait_state(unsigned** counter, int* polls) {
  *polls = g_host_poll_limit;
  return cudaGetSymbolAddress(reinterpret_cast<void**>(counter), g_stage_timeouts);
}

cudaError_t take_stage_timeouts(unsigned* count) {
  cudaError_t e = cudaMemcpyFromSymbol(count, g_stage_timeouts, sizeof(unsigned));
  if (e != cudaSuccess || *count == 0) return e;
  const unsigned zero = 0;
  return cudaMemcpyToSymbol(g_stage_timeouts, &zero, sizeof(unsigned));
}

size_t sweep_smem_bytes(int ts) {
  size_t b = 16;  // the mbarrier
  for (int t = 0; t < 2 * ts; ++t) {  // tiles without FP64 points
    b += sizeof(double) * tile_doubles(6, false) + sizeof(float) * tile_floats(6, true) +
         sizeof(int) * tile_ints(1);
    b = (b + 15) & ~size_t(15);
  }
  return b + 2 * sizeof(long long) + sizeof(float2) * kTile * (kTile + 1) +
         sizeof(unsigned) * kTile + 32;
}

namespace {
template <int TS, int MINB>
cudaError_t launch_sweep_shape(const SweepArgs& args, const RegularRule& rule, int blocks,
                               cudaStream_t stream) {
  const size_t smem = sweep_smem_bytes(TS);
  auto fn = sweep_sl_dp0<TS, MINB>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) {
    cudaGetLastError();  // not sticky: clear it, so that it is not reported by a later launch
    return e;
  }
  fn<<<blocks, kThreads, smem, stream>>>(args, rule);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_sweep_sl(const SweepArgs& args, const RegularRule& rule,
                            const SingularRules& rules, int blocks_per_sm, int sms,
                            cudaStream_t stream) {
  (void)rules;
  if (rule.npts != 6) return cudaErrorInvalidValue;
  if (args.tile_shape != 1 && args.tile_shape != 2) return cudaErrorInvalidValue;
  const int blocks = blocks_per_sm * sms;
  // the register cap follows the CTAs per SM asked for (at most 6)
  if (args.tile_shape == 1)
    return blocks_per_sm > 4 ? launch_sweep_shape<1, 6>(args, rule, blocks, stream)
                             : launch_sweep_shape<1, 4>(args, rule, blocks, stream);
  return blocks_per_sm > 4 ? launch_sweep_shape<2, 6>(args, rule, blocks, stream)
                           : launch_sweep_shape<2, 4>(args, rule, blocks, stream);
}

cudaError_t launch_sweep_near_singular(const SweepArgs& args, const RegularRule& rule,
                                       const SingularRules& rules, cudaStream_t stream) {
  if (rule.npts != 6) return cudaErrorInvalidValue;
  const long long nn = args.near_begin[args.nmesh], ns = args.sing_begin[args.nmesh];
  if (nn > 0) {
    const long long blocks = (nn + kThreads - 1) / kThreads;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    sweep_near_fp64<<<static_cast<unsigned>(blocks), kThreads, 0, stream>>>(args, rule);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (ns > 0) {
    const long long blocks = (ns * 32 + kThreads - 1) / kThreads;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    sweep_duffy_fp64<<<static_cast<unsigned>(blocks), kThreads, 0, stream>>>(args, rules);
    return cudaGetLastError();
  }
  return cudaSuccess;
}

cudaError_t launch_regular_dp0(const CellSet& test, const CellSet& trial,
                               const RegularRule& rule, const RegularArgs& a,
                               cudaStream_t stream) {
  SpaceTiles none{};
  none.nbasis = 1;
  none.tile_cells = kTile;
  return dispatch(test, none, trial, none, rule, a, stream, true);
}

cudaError_t launch_regular_scatter(const CellSet& test, const SpaceTiles& tt,
                                   const CellSet& trial, const SpaceTiles& st,
                                   const RegularRule& rule, const RegularArgs& a,
                                   cudaStream_t stream) {
  // degree 2 on both sides, Laplace single / double / adjoint double layer, FP64: the
  // tiled kernel (6 x 6 blocks per cell pair)
  // (when the DOF block of a tile pair fits in shared memory: P2, not DP2)
  const bool tiled_p2 = tt.nbasis == 6 && st.nbasis == 6 && a.kernel == kLaplace &&
                        a.op != kHS && a.precision == kRegularFP64 &&
                        static_cast<size_t>(tt.max_tile_dofs) * st.max_tile_dofs * sizeof(double) <=
                            (size_t(96) << 10);
  if ((tt.nbasis > 3 || st.nbasis > 3) && !tiled_p2) {
    // other pairings with a degree-2 side: the generic warp-per-pair kernel (FP64) over
    // this launch's trial cells
    GenericPairArgs g;
    g.kernel = a.kernel;
    g.op = a.op;
    g.k = a.k;
    g.nbt = tt.nbasis;
    g.nbs = st.nbasis;
    g.test = test;
    g.trial = trial;
    g.test_dofs = tt.cell_dofs;
    g.trial_dofs = st.cell_dofs;
    g.rule = rule;
    g.rules = SingularRules{};
    g.pairs = SingularPairs{};
    g.singular = false;
    g.same_grid = a.same_grid;
    g.symmetric = a.symmetric == 1 ? 1 : 0;
    g.out = a.out;
    g.ld = a.ld;
    const int tiles = (trial.ncells + kTile - 1) / kTile;
    const int ny = a.trial_tiles > 0 ? std::min(a.trial_tiles, tiles - a.trial_tile0)
                                     : tiles - a.trial_tile0;
    g.trial_lo = a.trial_tile0 * kTile;
    g.trial_hi = std::min(trial.ncells, (a.trial_tile0 + std::max(ny, 0)) * kTile);
    return launch_generic_pairs(g, stream);
  }
  if (tt.tile_cells != kTile || st.tile_cells != kTile) return cudaErrorInvalidValue;
  return dispatch(test, tt, trial, st, rule, a, stream, false);
}

}  // namespace bempp_b200
