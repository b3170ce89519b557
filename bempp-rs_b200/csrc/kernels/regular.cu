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
//   * Helmholtz: e^{ikr} = e^{ik r0} e^{ik delta}, r0 = |dc| in FP64, delta = r - r0 =
//     (2 dc.D + D.D) / (r + r0), D = dx_p - dy_q, free of cancellation; e^{ik delta} from
//     the Taylor series of cos / sin (degree 10 / 9, truncation < 3e-8) when
//     |k delta| <= k (rad_x + rad_y) <= 0.8, else CUDA's sincosf; e^{ik r0} from an FP64
//     reduction of k r0 modulo 2 pi followed by sincosf;
//   * DP0 entries sum their 6 inner sums with Kahan compensation; P1 blocks are formed
//     in FP32 and accumulated into the matrix in FP64.
#include "launch.h"

namespace bempp_b200 {
namespace {

constexpr int kTile = 32;
constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr float kTaylorMax = 0.8f;

enum TileField : int {
  fJdet = 0, fNx, fNy, fNz, fH, fT0x, fT0y, fT0z, fT1x, fT1y, fT1z, fCx, fCy, fCz, fDiam,
  fRad, kTileFields
};

// Shared-memory image of a tile of kTile cells.
struct Tile {
  double* pts;  // [(q*3+d) * kTile + c] absolute FP64 points
  float* rel;   // [(q*3+d) * kTile + c] FP32 offsets from the centroid (mixed only)
  double* geo;  // [f * kTile + c]
  int* vid;     // [v * kTile + c]
  int* ldof;    // [b * kTile + c]
  __device__ __forceinline__ double P(int q, int d, int c) const { return pts[(q * 3 + d) * kTile + c]; }
  __device__ __forceinline__ float R(int q, int d, int c) const { return rel[(q * 3 + d) * kTile + c]; }
  __device__ __forceinline__ double G(int f, int c) const { return geo[f * kTile + c]; }
};

__host__ __device__ inline size_t tile_doubles(int q) { return (3 * q + kTileFields) * kTile; }
__host__ __device__ inline size_t tile_floats(int q, bool mixed) { return mixed ? 3 * q * kTile : 0; }
__host__ __device__ inline size_t tile_ints(int nb) { return (3 + nb) * kTile; }

// Carves a tile out of shared memory starting at *cursor (8-byte aligned).
__device__ Tile carve_tile(unsigned char*& cursor, int q, bool mixed, int nb) {
  Tile t;
  t.pts = reinterpret_cast<double*>(cursor);
  t.geo = t.pts + 3 * q * kTile;
  cursor = reinterpret_cast<unsigned char*>(t.geo + kTileFields * kTile);
  t.rel = reinterpret_cast<float*>(cursor);
  cursor += sizeof(float) * tile_floats(q, mixed);
  t.vid = reinterpret_cast<int*>(cursor);
  t.ldof = t.vid + 3 * kTile;
  cursor += sizeof(int) * tile_ints(nb);
  cursor = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(cursor) + 15) & ~uintptr_t(15));
  return t;
}

__device__ void load_tile(const Tile& t, const CellSet& cs, int c0, int n, int q, bool mixed,
                          const uint8_t* cell_ldof, int nb) {
  const int N = cs.ncells;
  for (int idx = threadIdx.x; idx < 3 * q * kTile; idx += kThreads) {
    const int c = idx % kTile, pd = idx / kTile;
    const int64_t src = static_cast<int64_t>(pd) * N + c0 + min(c, n - 1);
    t.pts[idx] = __ldg(cs.qpts + src);
    if (mixed) t.rel[idx] = __ldg(cs.qrel + src);
  }
  for (int c = threadIdx.x; c < kTile; c += kThreads) {
    const int cell = c0 + min(c, n - 1);
    const double nx = g(cs.geom, kNx, N, cell), ny = g(cs.geom, kNy, N, cell),
                 nz = g(cs.geom, kNz, N, cell);
    t.geo[fJdet * kTile + c] = g(cs.geom, kJdet, N, cell);
    t.geo[fNx * kTile + c] = nx;
    t.geo[fNy * kTile + c] = ny;
    t.geo[fNz * kTile + c] = nz;
    t.geo[fH * kTile + c] = g(cs.geom, kV0x, N, cell) * nx + g(cs.geom, kV0y, N, cell) * ny +
                            g(cs.geom, kV0z, N, cell) * nz;
    for (int f = 0; f < 6; ++f) t.geo[(fT0x + f) * kTile + c] = g(cs.geom, kT0x + f, N, cell);
    for (int f = 0; f < 3; ++f) t.geo[(fCx + f) * kTile + c] = g(cs.geom, kCx + f, N, cell);
    t.geo[fDiam * kTile + c] = g(cs.geom, kDiam, N, cell);
    t.geo[fRad * kTile + c] = g(cs.geom, kRad, N, cell);
    for (int v = 0; v < 3; ++v) t.vid[v * kTile + c] = c < n ? __ldg(cs.vids + v * N + cell) : -1 - v;
    for (int b = 0; b < nb; ++b) t.ldof[b * kTile + c] = cell_ldof ? cell_ldof[cell * nb + b] : 0;
  }
}

__device__ __forceinline__ void kahan_add(float& sum, float& comp, float v) {
  const float y = v - comp;
  const float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

// cos(t), sin(t) for |t| <= 0.8 from their Taylor series (degree 10 and 9).
__device__ __forceinline__ void taylor_cos_sin(float t, float& c, float& s) {
  const float z = t * t;
  c = fmaf(z, fmaf(z, fmaf(z, fmaf(z, fmaf(z, -2.7557319e-7f, 2.4801587e-5f), -1.3888889e-3f),
                           4.1666668e-2f), -0.5f), 1.0f);
  s = t * fmaf(z, fmaf(z, fmaf(z, fmaf(z, 2.7557319e-6f, -1.9841270e-4f), 8.3333333e-3f),
                       -0.16666667f), 1.0f);
}

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
  if (OP != kHS) {
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

// FP64 local block of test cell `it` (tile T) and trial cell `js` (tile S).
template <int QT, int KER, int OP, int NBT, int NBS>
__device__ __forceinline__ void block_fp64(const Tile& T, int it, const Tile& S, int js,
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
  const double nxi = T.G(fNx, it), nyi = T.G(fNy, it), nzi = T.G(fNz, it), hi = T.G(fH, it);
  const double nxj = S.G(fNx, js), nyj = S.G(fNy, js), nzj = S.G(fNz, js), hj = S.G(fH, js);
#pragma unroll 1
  for (int p = 0; p < Q; ++p) {
    const double x0 = T.P(p, 0, it), x1 = T.P(p, 1, it), x2 = T.P(p, 2, it);
    const double ap = OP == kDL ? x0 * nxj + x1 * nyj + x2 * nzj - hj : 1.0;
    double u_re[NBS], u_im[NBS], g_re = 0.0, g_im = 0.0;
#pragma unroll
    for (int b = 0; b < NBS; ++b) u_re[b] = u_im[b] = 0.0;
#pragma unroll 6
    for (int q = 0; q < Q; ++q) {
      const double y0 = S.P(q, 0, js), y1 = S.P(q, 1, js), y2 = S.P(q, 2, js);
      const double dx = x0 - y0, dy = x1 - y1, dz = x2 - y2;
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double rinv = rsqrt_refined(r2);
      double wq = rule.w[q];
      if (OP == kADL) wq *= y0 * nxi + y1 * nyi + y2 * nzi - hi;
      double kre, kim = 0.0;
      if (KER == kLaplace) {
        kre = (OP == kSL || OP == kHS) ? wq * rinv : wq * rinv * rinv * rinv;
      } else {
        const double r = r2 * rinv;
        double sn, cs;
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
            u_re[b] = fma(kre, rule.phi[b][q], u_re[b]);
            if (kC) u_im[b] = fma(kim, rule.phi[b][q], u_im[b]);
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
        const double f = NBT == 1 ? wp : wp * rule.phi[a][p];
#pragma unroll
        for (int b = 0; b < NBS; ++b) {
          blk_re[a][b] = fma(f, u_re[b], blk_re[a][b]);
          if (kC) blk_im[a][b] = fma(f, u_im[b], blk_im[a][b]);
        }
      }
    }
  }
  finish_block<KER, OP, NBT, NBS>(T, it, S, js, k, blk_re, blk_im, S_re, S_im, ore, oim);
}

// FP32 local block of a far pair (see the file comment for the formulation).
template <int QT, int KER, int OP, int NBT, int NBS>
__device__ __forceinline__ void block_fp32(const Tile& T, int it, const Tile& S, int js,
                                           const RegularRule& rule, double k,
                                           double ore[NBT][NBS], double oim[NBT][NBS]) {
  constexpr bool kC = KER == kHelmholtz;
  constexpr bool kNeedBasis = OP != kHS || kC;
  constexpr bool kKahan = NBT == 1 && NBS == 1;
  const int Q = QT > 0 ? QT : rule.npts;
  const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
               dcz = T.G(fCz, it) - S.G(fCz, js);
  const float fdx = static_cast<float>(dcx), fdy = static_cast<float>(dcy),
              fdz = static_cast<float>(dcz);
  // normal-derivative factors in tangent coordinates
  float fa0 = 0.f, fa1 = 0.f, fa2 = 0.f;
  if (OP == kDL) {
    const double nx = S.G(fNx, js), ny = S.G(fNy, js), nz = S.G(fNz, js);
    fa0 = static_cast<float>(dcx * nx + dcy * ny + dcz * nz);
    fa1 = static_cast<float>(T.G(fT0x, it) * nx + T.G(fT0y, it) * ny + T.G(fT0z, it) * nz);
    fa2 = static_cast<float>(T.G(fT1x, it) * nx + T.G(fT1y, it) * ny + T.G(fT1z, it) * nz);
  } else if (OP == kADL) {
    const double nx = T.G(fNx, it), ny = T.G(fNy, it), nz = T.G(fNz, it);
    fa0 = static_cast<float>(-(dcx * nx + dcy * ny + dcz * nz));
    fa1 = static_cast<float>(S.G(fT0x, js) * nx + S.G(fT0y, js) * ny + S.G(fT0z, js) * nz);
    fa2 = static_cast<float>(S.G(fT1x, js) * nx + S.G(fT1y, js) * ny + S.G(fT1z, js) * nz);
  }
  float r0f = 0.f, r0sq = 0.f, kf = 0.f, ph_c = 1.f, ph_s = 0.f;
  bool taylor = false;
  if (kC) {
    const double r0 = sqrt(dcx * dcx + dcy * dcy + dcz * dcz);
    r0f = static_cast<float>(r0);
    r0sq = r0f * r0f;
    kf = static_cast<float>(k);
    // e^{ik r0}: k r0 reduced modulo 2 pi in FP64, then FP32 sincos of the remainder
    const double theta = k * r0;
    const double turns = rint(theta * 0.15915494309189533577);
    const double red = fma(-turns, 6.28318530717958647692, theta);
    sincosf(static_cast<float>(red), &ph_s, &ph_c);
    taylor = k * (T.G(fRad, it) + S.G(fRad, js)) <= static_cast<double>(kTaylorMax);
  }
  // per-pair factors of each trial point: ADL weight factor and 2 dc.dy_q
  constexpr int kCap = QT > 0 ? QT : kMaxRegularPoints;
  float wq_s[kCap], beta_s[kCap];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    wq_s[q] = OP == kADL ? rule.wf[q] * fmaf(rule.uf[q], fa1, fmaf(rule.vf[q], fa2, fa0))
                         : rule.wf[q];
    if (kC) beta_s[q] = 2.f * fmaf(fdx, S.R(q, 0, js), fmaf(fdy, S.R(q, 1, js), fdz * S.R(q, 2, js)));
  }
  float blk_re[NBT][NBS], blk_im[NBT][NBS], cmp_re = 0.f, cmp_im = 0.f;
  float S_re = 0.f, S_im = 0.f;
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b) blk_re[a][b] = blk_im[a][b] = 0.f;
#pragma unroll 1
  for (int p = 0; p < Q; ++p) {
    const float ax = T.R(p, 0, it), ay = T.R(p, 1, it), az = T.R(p, 2, it);
    const float apf = OP == kDL ? fmaf(rule.uf[p], fa1, fmaf(rule.vf[p], fa2, fa0)) : 1.f;
    const float alpha = kC ? 2.f * fmaf(fdx, ax, fmaf(fdy, ay, fdz * az)) : 0.f;
    const float px = fdx + ax, py = fdy + ay, pz = fdz + az;
    float u_re[NBS], u_im[NBS], g_re = 0.f, g_im = 0.f;
#pragma unroll
    for (int b = 0; b < NBS; ++b) u_re[b] = u_im[b] = 0.f;
#pragma unroll 6
    for (int q = 0; q < Q; ++q) {
      const float yx = S.R(q, 0, js), yy = S.R(q, 1, js), yz = S.R(q, 2, js);
      const float wq = wq_s[q];
      float kre, kim = 0.f;
      if (!kC) {
        const float dx = px - yx, dy = py - yy, dz = pz - yz;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float rinv = rsqrtf(r2);
        kre = (OP == kSL || OP == kHS) ? wq * rinv : wq * (rinv * rinv * rinv);
      } else {
        const float Dx = ax - yx, Dy = ay - yy, Dz = az - yz;
        const float s = (alpha - beta_s[q]) + fmaf(Dx, Dx, fmaf(Dy, Dy, Dz * Dz));  // r^2 - r0^2
        const float r2 = r0sq + s;
        const float rinv = rsqrtf(r2);
        const float r = r2 * rinv;
        const float t = kf * __fdividef(s, r + r0f);
        float cs, sn;
        if (taylor)
          taylor_cos_sin(t, cs, sn);
        else
          sincosf(t, &sn, &cs);
        if (OP == kSL || OP == kHS) {
          const float f = wq * rinv;
          kre = f * cs;
          kim = f * sn;
        } else {
          const float f = wq * (rinv * rinv * rinv), kr = kf * r;
          // (1 - ik r) e^{ik r} = (1 - ik r) e^{ik r0} e^{ik delta}; e^{ik r0} applied below
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
  // back to FP64, applying the reference phase e^{ik r0}
  double bre[NBT][NBS], bim[NBT][NBS];
  double Sre = S_re, Sim = S_im;
  if (kC) {
    const double c = ph_c, s = ph_s;
    const double re = Sre * c - Sim * s, im = Sre * s + Sim * c;
    Sre = re;
    Sim = im;
  }
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b) {
      double re = blk_re[a][b], im = blk_im[a][b];
      if (kC) {
        const double c = ph_c, s = ph_s;
        const double r2 = re * c - im * s, i2 = re * s + im * c;
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

template <int QT, int KER, int OP, int NBT, int NBS, bool MIXED, bool DIRECT>
__global__ void __launch_bounds__(kThreads, 4)
    regular_tiles(CellSet test, SpaceTiles tt, CellSet trial, SpaceTiles st, RegularRule rule,
                  double k, int same_grid, double* __restrict__ out, int64_t ld) {
  constexpr bool kC = KER == kHelmholtz;
  const int Q = QT > 0 ? QT : rule.npts;
  const int ti0 = blockIdx.x * kTile, sj0 = blockIdx.y * kTile;
  const int nti = min(kTile, test.ncells - ti0), nsj = min(kTile, trial.ncells - sj0);

  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* cursor = smem;
  double* acc_re = nullptr;
  double* acc_im = nullptr;
  int ndt = 0, nds = 0, tdof0 = 0, sdof0 = 0;
  if (!DIRECT) {
    tdof0 = tt.tile_dof_off[blockIdx.x];
    ndt = tt.tile_dof_off[blockIdx.x + 1] - tdof0;
    sdof0 = st.tile_dof_off[blockIdx.y];
    nds = st.tile_dof_off[blockIdx.y + 1] - sdof0;
    const int cap = tt.max_tile_dofs * st.max_tile_dofs;
    acc_re = reinterpret_cast<double*>(cursor);
    acc_im = acc_re + cap;
    cursor += sizeof(double) * cap * (kC ? 2 : 1);
  }
  const Tile T = carve_tile(cursor, Q, MIXED, NBT);
  const Tile S = carve_tile(cursor, Q, MIXED, NBS);
  unsigned short* queue = reinterpret_cast<unsigned short*>(cursor);  // MIXED: near pairs
  int* qcount = reinterpret_cast<int*>(cursor + sizeof(unsigned short) * kTile * kTile);

  if (!DIRECT)
    for (int idx = threadIdx.x; idx < ndt * nds; idx += kThreads) {
      acc_re[idx] = 0.0;
      if (kC) acc_im[idx] = 0.0;
    }
  if (MIXED && threadIdx.x == 0) *qcount = 0;
  load_tile(T, test, ti0, nti, Q, MIXED, DIRECT ? nullptr : tt.cell_ldof, NBT);
  load_tile(S, trial, sj0, nsj, Q, MIXED, DIRECT ? nullptr : st.cell_ldof, NBS);
  __syncthreads();

  const int it = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (it < nti) {
    const int a0 = T.vid[it], a1 = T.vid[kTile + it], a2 = T.vid[2 * kTile + it];
    for (int js = warp; js < nsj; js += kWarps) {
      const bool adjacent = same_grid && share_vertex(a0, a1, a2, S.vid[js], S.vid[kTile + js],
                                                      S.vid[2 * kTile + js]);
      const int64_t o = static_cast<int64_t>(sj0 + js) * ld + ti0 + it;
      if (adjacent) {
        if (DIRECT) {
          if (kC)
            reinterpret_cast<double2*>(out)[o] = make_double2(0.0, 0.0);
          else
            out[o] = 0.0;
        }
        continue;
      }
      double ore[NBT][NBS], oim[NBT][NBS];
      if (MIXED) {
        if (near_pair(T, it, S, js)) {
          const int slot = atomicAdd(qcount, 1);
          queue[slot] = static_cast<unsigned short>(it | (js << 8));
          continue;
        }
        block_fp32<QT, KER, OP, NBT, NBS>(T, it, S, js, rule, k, ore, oim);
      } else {
        block_fp64<QT, KER, OP, NBT, NBS>(T, it, S, js, rule, k, ore, oim);
      }
      if (DIRECT) {
        if (kC)
          reinterpret_cast<double2*>(out)[o] = make_double2(ore[0][0], oim[0][0]);
        else
          out[o] = ore[0][0];
      } else {
        deposit<NBT, NBS, kC>(acc_re, acc_im, ndt, T, it, S, js, ore, oim);
      }
    }
  }
  if (MIXED) {
    __syncthreads();
    const int nq = *qcount;
    for (int e = threadIdx.x; e < nq; e += kThreads) {
      const int pi = queue[e] & 0xff, pj = queue[e] >> 8;
      double ore[NBT][NBS], oim[NBT][NBS];
      block_fp64<QT, KER, OP, NBT, NBS>(T, pi, S, pj, rule, k, ore, oim);
      if (DIRECT) {
        const int64_t o = static_cast<int64_t>(sj0 + pj) * ld + ti0 + pi;
        if (kC)
          reinterpret_cast<double2*>(out)[o] = make_double2(ore[0][0], oim[0][0]);
        else
          out[o] = ore[0][0];
      } else {
        deposit<NBT, NBS, kC>(acc_re, acc_im, ndt, T, pi, S, pj, ore, oim);
      }
    }
  }
  if (!DIRECT) {
    __syncthreads();
    const int* tdofs = tt.tile_dofs + tdof0;
    const int* sdofs = st.tile_dofs + sdof0;
    for (int idx = threadIdx.x; idx < ndt * nds; idx += kThreads) {
      const int a = idx % ndt, b = idx / ndt;
      const int64_t o = static_cast<int64_t>(sdofs[b]) * ld + tdofs[a];
      const double re = acc_re[idx];
      if (kC) {
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
}

size_t smem_bytes(int q, bool mixed, bool direct, bool cplx, int max_t, int max_s, int nbt,
                  int nbs) {
  size_t b = 0;
  if (!direct) b += sizeof(double) * static_cast<size_t>(max_t) * max_s * (cplx ? 2 : 1);
  for (int nb : {nbt, nbs}) {
    b += sizeof(double) * tile_doubles(q) + sizeof(float) * tile_floats(q, mixed) +
         sizeof(int) * tile_ints(nb);
    b = (b + 15) & ~size_t(15);
  }
  if (mixed) b += sizeof(unsigned short) * kTile * kTile + sizeof(int);
  return b + 16;
}

template <int QT, int KER, int OP, int NBT, int NBS, bool MIXED, bool DIRECT>
cudaError_t launch_one(const CellSet& test, const SpaceTiles& tt, const CellSet& trial,
                       const SpaceTiles& st, const RegularRule& rule, const RegularArgs& a,
                       cudaStream_t stream) {
  const size_t smem = smem_bytes(rule.npts, MIXED, DIRECT, KER == kHelmholtz, tt.max_tile_dofs,
                                 st.max_tile_dofs, NBT, NBS);
  auto fn = regular_tiles<QT, KER, OP, NBT, NBS, MIXED, DIRECT>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  dim3 grid((test.ncells + kTile - 1) / kTile, (trial.ncells + kTile - 1) / kTile);
  fn<<<grid, kThreads, smem, stream>>>(test, tt, trial, st, rule, a.k, a.same_grid,
                                       static_cast<double*>(a.out), a.ld);
  return cudaGetLastError();
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
  if (tt.tile_cells != kTile || st.tile_cells != kTile) return cudaErrorInvalidValue;
  return dispatch(test, tt, trial, st, rule, a, stream, false);
}

}  // namespace bempp_b200
