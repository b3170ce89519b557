// Adjoint gradient of J = Re(lambda^H A(x, k) mu) for the Helmholtz single-layer operator
// on DP0 x DP0, with respect to every vertex coordinate and the wavenumber, without
// forming dA.
//
// A_ij = (1/4pi) jdet_i jdet_j sum_n w_n e^{ik r_n} / r_n over the rule of the pair
// (regular tensor rule, or the Duffy rule of an adjacent pair), r_n = |x_n - y_n| with
// x_n = sum_a phi_a(xi_n) V_{i,a} and y_n = sum_b phi_b(eta_n) V_{j,b} (phi the P1
// barycentric weights, V the cell vertices).  The discrete sum is differentiated
// exactly:
//   dA_ij/dV_{i,a} = (1/4pi) [ djdet_i/dV_a jdet_j sum_n w_n G_n
//                              + jdet_i jdet_j sum_n w_n phi_a(xi_n) grad_x G_n ],
//   grad_x (e^{ikr}/r) = e^{ikr} (ikr - 1) (x - y) / r^3,  grad_y = -grad_x,
//   djdet/dV1 = t1 x n, djdet/dV2 = n x t0, djdet/dV0 = -(t1 x n + n x t0),
//   dA_ij/dk = (1/4pi) jdet_i jdet_j sum_n w_n i e^{ikr_n}.
// Each pair contributes Re(conj(lambda_i) mu_j dA_ij) to 9 + 9 vertex coordinates of
// its two cells and to dJ/dk; contributions are reduced per CTA (test side in
// registers and shared memory, trial side by warp shuffles) and added per cell, then a
// last kernel scatters the per-cell-vertex gradients to the vertices.
//
// Regular pairs use the tiled mapping of regular.cu (32 x 32 cell tiles, lane = test
// cell, both tiles staged in shared memory by TMA bulk copies on an mbarrier with the
// regular kernels' bounded wait and timeout counter); adjacent pairs use one warp per pair
// over their Duffy rule.  FP64, or mixed:
// far pairs (centroid distance >= 2 diameters) in FP32 with centroid-relative points and
// the reference phase e^{ik r0} folded into the pair weight, as in regular.cu.
#include "launch.h"
#include "tiles.cuh"

namespace bempp_b200 {
namespace {

using namespace tiles;

// d jdet / d V_a of a flat cell, a = 0, 1, 2 (3-vectors)
__device__ __forceinline__ void jdet_gradient(const double t0[3], const double t1[3],
                                              const double n[3], double g[3][3]) {
  const double a[3] = {t1[1] * n[2] - t1[2] * n[1], t1[2] * n[0] - t1[0] * n[2],
                       t1[0] * n[1] - t1[1] * n[0]};  // t1 x n
  const double b[3] = {n[1] * t0[2] - n[2] * t0[1], n[2] * t0[0] - n[0] * t0[2],
                       n[0] * t0[1] - n[1] * t0[0]};  // n x t0
  for (int d = 0; d < 3; ++d) {
    g[1][d] = a[d];
    g[2][d] = b[d];
    g[0][d] = -(a[d] + b[d]);
  }
}

template <int QT, bool MIXED>
__global__ void __launch_bounds__(kThreads, 3)
    adjoint_sl_regular(CellSet cs, RegularRule rule, double k, const double2* __restrict__ lam,
                       const double2* __restrict__ mu, double* __restrict__ grad_cell,
                       double* __restrict__ totals, unsigned* __restrict__ stage_timeouts,
                       int stage_polls) {
  const int Q = QT > 0 ? QT : rule.npts;
  // A_ij = A_ji on far pairs (one cell set and one rule on both sides), so only tile pairs
  // tx >= sy are visited; an off-diagonal tile takes c_ij + c_ji for both orders of its pairs
  int tx, sy;
  const int ntt = (cs.ncells + kTile - 1) / kTile;
  lower_tile_pair(blockIdx.x, ntt, 0, ntt, tx, sy);
  const bool both = tx > sy;
  const int ti0 = tx * kTile, sj0 = sy * kTile;
  const int nti = min(kTile, cs.ncells - ti0), nsj = min(kTile, cs.ncells - sj0);
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);  // completion of the tile copies
  unsigned char* cursor = smem + 16;
  const Tile T = carve_tile(cursor, Q, MIXED, 1);
  const Tile S = carve_tile(cursor, Q, MIXED, 1);
  double* s_test = reinterpret_cast<double*>(cursor);  // [kTile][9] test-cell gradients
  double* s_trial = s_test + kTile * 9;                // [kTile][9] trial-cell gradients
  double* s_tot = s_trial + kTile * 9;                 // J, dJ/dk
  // both tiles by bulk (TMA) copies on one mbarrier, issued by one thread, while the
  // others clear the gradient accumulators
  if (threadIdx.x == 0) mbar_init(mbar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(mbar, 2 * bulk_tile_bytes(Q, MIXED));
    stage_tile_bulk(T, cs, ti0, Q, MIXED, mbar);
    stage_tile_bulk(S, cs, sj0, Q, MIXED, mbar);
  }
  for (int e = threadIdx.x; e < 2 * kTile * 9 + 2; e += kThreads) s_test[e] = 0.0;
  const bool staged = mbar_wait_bounded(mbar, 0, stage_polls);
  if (__syncthreads_or(!staged)) {
    // the copies did not complete in time: record it, give them a last bounded wait and
    // add nothing (the host reports the failure)
    if (threadIdx.x == 0) atomicAdd(stage_timeouts, 1u);
    mbar_wait_bounded(mbar, 0);
    return;
  }

  const int it = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool valid = it < nti;
  const double2 li = valid ? lam[ti0 + it] : make_double2(0.0, 0.0);
  const double2 mi = valid && both ? mu[ti0 + it] : make_double2(0.0, 0.0);
  const int a0 = T.vid[it], a1 = T.vid[kTile + it], a2 = T.vid[2 * kTile + it];
  const double jdet_i = T.G(fJdet, it);

  double gt[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // test-cell vertex gradients
  double jval = 0.0, dk = 0.0;
  for (int js = warp; js < nsj; js += kWarps) {
    const bool adjacent = share_vertex(a0, a1, a2, S.vid[js], S.vid[kTile + js],
                                       S.vid[2 * kTile + js]);
    const bool active = valid && !adjacent;
    // c = conj(lambda_i) mu_j (+ conj(lambda_j) mu_i off the diagonal)
    const double2 mj = mu[sj0 + js];
    double c_re = li.x * mj.x + li.y * mj.y, c_im = li.x * mj.y - li.y * mj.x;
    if (both) {
      const double2 lj = lam[sj0 + js];
      c_re += lj.x * mi.x + lj.y * mi.y;
      c_im += lj.x * mi.y - lj.y * mi.x;
    }
    double S0_re = 0.0, S0_im = 0.0, Sk_re = 0.0, Sk_im = 0.0;
    double uq[QT > 0 ? QT : kMaxRegularPoints][3];
#pragma unroll
    for (int q = 0; q < Q; ++q) uq[q][0] = uq[q][1] = uq[q][2] = 0.0;
    double vt[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    bool far = false;
    if (MIXED && active) {
      const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
                   dcz = T.G(fCz, it) - S.G(fCz, js);
      const double dist2 = dcx * dcx + dcy * dcy + dcz * dcz;
      const double lim = 2.0 * fmax(T.G(fDiam, it), S.G(fDiam, js));
      far = dist2 >= lim * lim;
      if (far) {
        // FP32 far pair: centroid-relative points, reference phase folded into the weight
        // c' = c e^{ik r0}, e^{ik r} = e^{ik r0} e^{ik (r - r0)}, r - r0 = s / (r + r0).
        const float fdx = static_cast<float>(dcx), fdy = static_cast<float>(dcy),
                    fdz = static_cast<float>(dcz);
        const double r0 = sqrt(dist2);
        const float r0f = static_cast<float>(r0), r0sq = r0f * r0f, kf = static_cast<float>(k);
        float pc, ps;
        phase_cos_sin(k * r0, pc, ps);
        const float cr = static_cast<float>(c_re * pc - c_im * ps);
        const float ci = static_cast<float>(c_re * ps + c_im * pc);
        const bool taylor = k * (T.G(fRad, it) + S.G(fRad, js)) <= 0.8;
        float fS0r = 0.f, fS0i = 0.f, fSkr = 0.f, fSki = 0.f;
        float fuq[QT > 0 ? QT : kMaxRegularPoints][3];
        float fvt[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int q = 0; q < Q; ++q) fuq[q][0] = fuq[q][1] = fuq[q][2] = 0.f;
#pragma unroll 1
        for (int p = 0; p < Q; ++p) {
          const float ax = T.R(p, 0, it), ay = T.R(p, 1, it), az = T.R(p, 2, it);
          const float alpha = 2.f * fmaf(fdx, ax, fmaf(fdy, ay, fdz * az));
          const float px = fdx + ax, py = fdy + ay, pz = fdz + az;
          float vp0 = 0.f, vp1 = 0.f, vp2 = 0.f, gr = 0.f, gi = 0.f, er = 0.f, ei = 0.f;
          const float wp = rule.wf[p];
#pragma unroll
          for (int q = 0; q < Q; ++q) {
            const float yx = S.R(q, 0, js), yy = S.R(q, 1, js), yz = S.R(q, 2, js);
            const float Dx = ax - yx, Dy = ay - yy, Dz = az - yz;
            const float beta = 2.f * fmaf(fdx, yx, fmaf(fdy, yy, fdz * yz));
            const float sq = (alpha - beta) + fmaf(Dx, Dx, fmaf(Dy, Dy, Dz * Dz));
            const float r2 = r0sq + sq;
            const float rinv = rsqrt_approx(r2);
            const float r = r2 * rinv, kr = kf * r;
            const float t = kf * sq * rcp_approx(r + r0f);
            float csn, sn;
            if (taylor)
              poly_cos_sin(t, csn, sn);
            else
              reduced_cos_sin(t, csn, sn);
            const float wq = rule.wf[q];
            gr = fmaf(wq * rinv, csn, gr);
            gi = fmaf(wq * rinv, sn, gi);
            er = fmaf(wq, csn, er);
            ei = fmaf(wq, sn, ei);
            const float f_re = -csn - kr * sn, f_im = kr * csn - sn;
            const float gs = wq * (cr * f_re - ci * f_im) * (rinv * rinv * rinv);
            const float dx = px - yx, dy = py - yy, dz = pz - yz;
            vp0 = fmaf(gs, dx, vp0);
            vp1 = fmaf(gs, dy, vp1);
            vp2 = fmaf(gs, dz, vp2);
            const float wgs = wp * gs;
            fuq[q][0] = fmaf(wgs, dx, fuq[q][0]);
            fuq[q][1] = fmaf(wgs, dy, fuq[q][1]);
            fuq[q][2] = fmaf(wgs, dz, fuq[q][2]);
          }
          fS0r = fmaf(wp, gr, fS0r);
          fS0i = fmaf(wp, gi, fS0i);
          fSkr = fmaf(wp, er, fSkr);
          fSki = fmaf(wp, ei, fSki);
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const float f = wp * rule.phif[a][p];
            fvt[a][0] = fmaf(f, vp0, fvt[a][0]);
            fvt[a][1] = fmaf(f, vp1, fvt[a][1]);
            fvt[a][2] = fmaf(f, vp2, fvt[a][2]);
          }
        }
        // back to FP64; S0 and Sk pick up e^{ik r0} through c' in R0 and dk below, so
        // express them relative to the original c by rotating: S = e^{ik r0} S'.
        S0_re = static_cast<double>(fS0r) * pc - static_cast<double>(fS0i) * ps;
        S0_im = static_cast<double>(fS0r) * ps + static_cast<double>(fS0i) * pc;
        Sk_re = static_cast<double>(fSkr) * pc - static_cast<double>(fSki) * ps;
        Sk_im = static_cast<double>(fSkr) * ps + static_cast<double>(fSki) * pc;
#pragma unroll
        for (int q = 0; q < Q; ++q)
          for (int d = 0; d < 3; ++d) uq[q][d] = fuq[q][d];
        for (int a = 0; a < 3; ++a)
          for (int d = 0; d < 3; ++d) vt[a][d] = fvt[a][d];
      }
    }
    if (active && !far) {
      // e^{ikr} referenced to the pair (e^{ik r0} e^{ik (r - r0)}, r0 = |c_x - c_y|) when
      // k (rad_x + rad_y) <= 0.8 bounds every phase k (r - r0): c is rotated by e^{ik r0}
      // for the gradient terms and the sums S0, Sk are rotated back after the loop
      const bool ref = k * (T.G(fRad, it) + S.G(fRad, js)) <= 0.8;
      double kr0 = 0.0, pc = 1.0, ps = 0.0, cq_re = c_re, cq_im = c_im;
      if (ref) {
        const double dcx = T.G(fCx, it) - S.G(fCx, js), dcy = T.G(fCy, it) - S.G(fCy, js),
                     dcz = T.G(fCz, it) - S.G(fCz, js);
        const double r0sq = dcx * dcx + dcy * dcy + dcz * dcz;
        kr0 = k * (r0sq * rsqrt_refined(r0sq));
        sincos_cw(kr0, ps, pc);
        cq_re = c_re * pc - c_im * ps;
        cq_im = c_re * ps + c_im * pc;
      }
#pragma unroll 1
      for (int p = 0; p < Q; ++p) {
        const double x0 = T.P(p, 0, it), x1 = T.P(p, 1, it), x2 = T.P(p, 2, it);
        double vp[3] = {0.0, 0.0, 0.0};
        double g_re = 0.0, g_im = 0.0, e_re = 0.0, e_im = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const double dx = x0 - S.P(q, 0, js), dy = x1 - S.P(q, 1, js), dz = x2 - S.P(q, 2, js);
          const double r2 = dx * dx + dy * dy + dz * dz;
          const double rinv = rsqrt_refined(r2);
          const double r = r2 * rinv, kr = k * r;
          double sn, csn;
          if (ref)
            sincos_small(fma(k, r, -kr0), sn, csn);
          else
            sincos(kr, &sn, &csn);
          const double wq = rule.w[q];
          g_re = fma(wq * rinv, csn, g_re);
          g_im = fma(wq * rinv, sn, g_im);
          e_re = fma(wq, csn, e_re);
          e_im = fma(wq, sn, e_im);
          // Re(c e^{ikr} (ikr - 1)) / r^3
          const double f_re = -csn - kr * sn, f_im = kr * csn - sn;
          const double gs = wq * (cq_re * f_re - cq_im * f_im) * rinv * rinv * rinv;
          vp[0] = fma(gs, dx, vp[0]);
          vp[1] = fma(gs, dy, vp[1]);
          vp[2] = fma(gs, dz, vp[2]);
          const double wgs = rule.w[p] * gs;
          uq[q][0] = fma(wgs, dx, uq[q][0]);
          uq[q][1] = fma(wgs, dy, uq[q][1]);
          uq[q][2] = fma(wgs, dz, uq[q][2]);
        }
        const double wp = rule.w[p];
        S0_re = fma(wp, g_re, S0_re);
        S0_im = fma(wp, g_im, S0_im);
        Sk_re = fma(wp, e_re, Sk_re);
        Sk_im = fma(wp, e_im, Sk_im);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double f = wp * rule.phi[a][p];
          vt[a][0] = fma(f, vp[0], vt[a][0]);
          vt[a][1] = fma(f, vp[1], vt[a][1]);
          vt[a][2] = fma(f, vp[2], vt[a][2]);
        }
      }
      if (ref) {
        const double s0r = S0_re * pc - S0_im * ps, s0i = S0_re * ps + S0_im * pc;
        const double skr = Sk_re * pc - Sk_im * ps, ski = Sk_re * ps + Sk_im * pc;
        S0_re = s0r;
        S0_im = s0i;
        Sk_re = skr;
        Sk_im = ski;
      }
    }
    const double jdet_j = S.G(fJdet, js);
    const double jj = jdet_i * jdet_j * kInv4Pi;
    const double R0 = c_re * S0_re - c_im * S0_im;  // Re(c S0)
    // trial-side contributions of this lane, then a warp reduction over the test cells
    double gs_[3][3];
    {
      double tj_t0[3], tj_t1[3], tj_n[3], djj[3][3];
      for (int d = 0; d < 3; ++d) {
        tj_t0[d] = S.G(fT0x + d, js);
        tj_t1[d] = S.G(fT1x + d, js);
      }
      tj_n[0] = S.G(fNx, js);
      tj_n[1] = S.G(fNy, js);
      tj_n[2] = S.G(fNz, js);
      jdet_gradient(tj_t0, tj_t1, tj_n, djj);
      const double rj = R0 * jdet_i * kInv4Pi;
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          double acc = 0.0;
#pragma unroll
          for (int q = 0; q < Q; ++q) acc = fma(rule.phi[b][q], uq[q][d], acc);
          gs_[b][d] = active ? (-jj * acc + rj * djj[b][d]) : 0.0;
        }
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      double v = gs_[e / 3][e % 3];
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
      if (it == 0) s_trial[js * 9 + e] += v;  // each js belongs to one warp
    }
    if (active) {
      double ti_t0[3], ti_t1[3], ti_n[3], dji[3][3];
      for (int d = 0; d < 3; ++d) {
        ti_t0[d] = T.G(fT0x + d, it);
        ti_t1[d] = T.G(fT1x + d, it);
      }
      ti_n[0] = T.G(fNx, it);
      ti_n[1] = T.G(fNy, it);
      ti_n[2] = T.G(fNz, it);
      jdet_gradient(ti_t0, ti_t1, ti_n, dji);
      const double ri = R0 * jdet_j * kInv4Pi;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) gt[a][d] += jj * vt[a][d] + ri * dji[a][d];
      jval += R0 * jj;
      dk += (c_re * (-Sk_im) - c_im * Sk_re) * jj;  // Re(c i Sk)
    }
  }
  if (valid) {
#pragma unroll
    for (int e = 0; e < 9; ++e) atomicAdd(s_test + it * 9 + e, gt[e / 3][e % 3]);
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    jval += __shfl_xor_sync(0xffffffffu, jval, s);
    dk += __shfl_xor_sync(0xffffffffu, dk, s);
  }
  if (it == 0) {
    atomicAdd(s_tot, jval);
    atomicAdd(s_tot + 1, dk);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kTile * 9; e += kThreads) {
    const int c = e / 9;
    if (c < nti) atomicAdd(grad_cell + static_cast<int64_t>(ti0 + c) * 9 + (e % 9), s_test[e]);
    if (c < nsj) atomicAdd(grad_cell + static_cast<int64_t>(sj0 + c) * 9 + (e % 9), s_trial[e]);
  }
  if (threadIdx.x == 0) {
    atomicAdd(totals, s_tot[0]);
    atomicAdd(totals + 1, s_tot[1]);
  }
}

struct CellGeo {
  double v0[3], t0[3], t1[3], n[3], jdet;
};

__device__ __forceinline__ void load_geo(const CellSet& cs, int c, CellGeo& g) {
  const int N = cs.stride;
  for (int d = 0; d < 3; ++d) {
    g.v0[d] = bempp_b200::g(cs.geom, kV0x + d, N, c);
    g.t0[d] = bempp_b200::g(cs.geom, kT0x + d, N, c);
    g.t1[d] = bempp_b200::g(cs.geom, kT1x + d, N, c);
    g.n[d] = bempp_b200::g(cs.geom, kNx + d, N, c);
  }
  g.jdet = bempp_b200::g(cs.geom, kJdet, N, c);
}

// One warp per adjacent pair over its Duffy rule.
__global__ void __launch_bounds__(256)
    adjoint_sl_singular(CellSet cs, SingularRules rules, SingularPairs pairs, double k,
                        const double2* __restrict__ lam, const double2* __restrict__ mu,
                        double* __restrict__ grad_cell, double* __restrict__ totals) {
  const int lane = threadIdx.x & 31;
  const int pair = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (pair >= pairs.npairs) return;
  const int tc = pairs.test_cell[pair], sc = pairs.trial_cell[pair], cfg = pairs.config[pair];
  CellGeo x, y;
  load_geo(cs, tc, x);
  load_geo(cs, sc, y);
  const double2 li = lam[tc], mj = mu[sc];
  const double c_re = li.x * mj.x + li.y * mj.y, c_im = li.x * mj.y - li.y * mj.x;
  const int off = rules.offset[cfg], npts = rules.offset[cfg + 1] - off;
  // |k r| <= k (diam_x + diam_y) for a pair sharing a vertex: no phase reduction needed
  // when that is below pi/4
  const bool small_phase = k * (bempp_b200::g(cs.geom, kDiam, cs.stride, tc) +
                                bempp_b200::g(cs.geom, kDiam, cs.stride, sc)) <= 0.78;
  double S0_re = 0.0, S0_im = 0.0, Sk_re = 0.0, Sk_im = 0.0;
  double gx[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, gy[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int ii = lane; ii < npts; ii += 32) {
    const int i = off + ii;
    const double xi0 = rules.test_xi[2 * i], xi1 = rules.test_xi[2 * i + 1];
    const double et0 = rules.trial_xi[2 * i], et1 = rules.trial_xi[2 * i + 1];
    const double w = rules.w[i];
    double d[3];
    for (int c = 0; c < 3; ++c)
      d[c] = (x.v0[c] + xi0 * x.t0[c] + xi1 * x.t1[c]) - (y.v0[c] + et0 * y.t0[c] + et1 * y.t1[c]);
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double rinv = rsqrt_refined(r2);
    const double r = r2 * rinv, kr = k * r;
    double sn, csn;
    if (small_phase)
      sincos_taylor(kr, sn, csn);
    else
      sincos_cw(kr, sn, csn);
    S0_re = fma(w * rinv, csn, S0_re);
    S0_im = fma(w * rinv, sn, S0_im);
    Sk_re = fma(w, csn, Sk_re);
    Sk_im = fma(w, sn, Sk_im);
    const double f_re = -csn - kr * sn, f_im = kr * csn - sn;
    const double gs = w * (c_re * f_re - c_im * f_im) * rinv * rinv * rinv;
    const double phi[3] = {1.0 - xi0 - xi1, xi0, xi1};
    const double psi[3] = {1.0 - et0 - et1, et0, et1};
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) {
        gx[a][c] = fma(gs * phi[a], d[c], gx[a][c]);
        gy[a][c] = fma(-gs * psi[a], d[c], gy[a][c]);
      }
  }
  for (int s = 16; s > 0; s >>= 1) {
    S0_re += __shfl_xor_sync(0xffffffffu, S0_re, s);
    S0_im += __shfl_xor_sync(0xffffffffu, S0_im, s);
    Sk_re += __shfl_xor_sync(0xffffffffu, Sk_re, s);
    Sk_im += __shfl_xor_sync(0xffffffffu, Sk_im, s);
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) {
        gx[a][c] += __shfl_xor_sync(0xffffffffu, gx[a][c], s);
        gy[a][c] += __shfl_xor_sync(0xffffffffu, gy[a][c], s);
      }
  }
  if (lane != 0) return;
  const double jj = x.jdet * y.jdet * kInv4Pi;
  const double R0 = c_re * S0_re - c_im * S0_im;
  double djx[3][3], djy[3][3];
  jdet_gradient(x.t0, x.t1, x.n, djx);
  jdet_gradient(y.t0, y.t1, y.n, djy);
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 3; ++c) {
      atomicAdd(grad_cell + static_cast<int64_t>(tc) * 9 + a * 3 + c,
                jj * gx[a][c] + R0 * y.jdet * kInv4Pi * djx[a][c]);
      atomicAdd(grad_cell + static_cast<int64_t>(sc) * 9 + a * 3 + c,
                jj * gy[a][c] + R0 * x.jdet * kInv4Pi * djy[a][c]);
    }
  atomicAdd(totals, R0 * jj);
  atomicAdd(totals + 1, (c_re * (-Sk_im) - c_im * Sk_re) * jj);
}

// Per-cell-vertex gradients -> per-point gradients (npoints x 3).
__global__ void cell_to_point_gradient(CellSet cs, const double* __restrict__ grad_cell,
                                       double* __restrict__ grad_points) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cs.ncells) return;
  for (int a = 0; a < 3; ++a) {
    const int v = cs.vids[a * cs.stride + c];
    for (int d = 0; d < 3; ++d)
      atomicAdd(grad_points + 3 * static_cast<int64_t>(v) + d,
                grad_cell[static_cast<int64_t>(c) * 9 + a * 3 + d]);
  }
}

}  // namespace

cudaError_t launch_adjoint_sl(const CellSet& cs, const RegularRule& rule,
                              const SingularRules& rules, const SingularPairs& pairs, double k,
                              const double* lam, const double* mu, double* grad_cell,
                              double* grad_points, int npoints, double* totals, bool mixed,
                              cudaStream_t stream) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(grad_cell, 0, sizeof(double) * 9 * cs.ncells, stream)) != cudaSuccess)
    return e;
  if ((e = cudaMemsetAsync(grad_points, 0, sizeof(double) * 3 * npoints, stream)) != cudaSuccess)
    return e;
  if ((e = cudaMemsetAsync(totals, 0, sizeof(double) * 2, stream)) != cudaSuccess) return e;
  if (cs.ncells <= 0) return cudaSuccess;
  const size_t smem = 16 /* mbarrier */ +
                      2 * (sizeof(double) * tile_doubles(rule.npts) +
                           sizeof(float) * tile_floats(rule.npts, mixed) + sizeof(int) * tile_ints(1) + 16) +
                      sizeof(double) * (2 * kTile * 9 + 2) + 16;
  unsigned* timeouts = nullptr;
  int polls = 0;
  if ((e = stage_wait_state(&timeouts, &polls)) != cudaSuccess) return e;
  const long long ntt = (cs.ncells + kTile - 1) / kTile;
  if (ntt * (ntt + 1) / 2 > 0x7fffffffLL) return cudaErrorInvalidValue;
  const dim3 grid(static_cast<unsigned>(ntt * (ntt + 1) / 2));  // tile pairs tx >= sy
  const double2* l2 = reinterpret_cast<const double2*>(lam);
  const double2* m2 = reinterpret_cast<const double2*>(mu);
  auto fn = rule.npts == 6 ? (mixed ? adjoint_sl_regular<6, true> : adjoint_sl_regular<6, false>)
                           : (mixed ? adjoint_sl_regular<0, true> : adjoint_sl_regular<0, false>);
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  fn<<<grid, kThreads, smem, stream>>>(cs, rule, k, l2, m2, grad_cell, totals, timeouts, polls);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (pairs.npairs > 0) {
    adjoint_sl_singular<<<(pairs.npairs + 7) / 8, 256, 0, stream>>>(cs, rules, pairs, k, l2, m2,
                                                                   grad_cell, totals);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  cell_to_point_gradient<<<(cs.ncells + 255) / 256, 256, 0, stream>>>(cs, grad_cell, grad_points);
  return cudaGetLastError();
}

}  // namespace bempp_b200
