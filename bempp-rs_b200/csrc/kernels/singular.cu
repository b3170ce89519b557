// Singular quadrature for cell pairs that share a vertex, an edge or the whole cell.
//
// Replaces bempp-rs assemble_batch_singular (src/boundary_assemblers.rs:608-685) with
// SingularCellPairAssembler (src/boundary_assemblers/cell_pair_assemblers.rs:109-152):
// entry[a][b] = sum_i f(x(xi_i), y(eta_i)) w_i jdet_x jdet_y over the Duffy rule of the
// pair's adjacency configuration.  The reference emits COO triplets per pair and adds
// them into the dense matrix serially (src/boundary_assemblers.rs:206-213); here one
// warp integrates one pair (lanes stride over the rule's 512-1536 points, a shuffle
// tree reduces the 1-9 block entries) and lane 0 adds the block into the dense output:
// plain read-modify-write when every pair owns its entries (DP0 x DP0), atomics
// otherwise.  It can also store the per-pair blocks for the CSR singular path.
#include "launch.h"

namespace bempp_b200 {
namespace {

constexpr int kThreads = 256;

struct CellData {
  double v0[3], t0[3], t1[3], n[3], jdet, diam;
};

__device__ __forceinline__ void load_cell(const CellSet& cs, int c, CellData& d) {
  const int n = cs.stride;
  for (int k = 0; k < 3; ++k) {
    d.v0[k] = g(cs.geom, kV0x + k, n, c);
    d.t0[k] = g(cs.geom, kT0x + k, n, c);
    d.t1[k] = g(cs.geom, kT1x + k, n, c);
    d.n[k] = g(cs.geom, kNx + k, n, c);
  }
  d.jdet = g(cs.geom, kJdet, n, c);
  d.diam = g(cs.geom, kDiam, n, c);
}

// FP64 throughout, with the refined hardware reciprocal square root (rsqrt_refined,
// rinv3_refined) and sincos_cw; a pair whose phases all satisfy |k r| <= pi/4 (k times
// the sum of the two diameters bounds them) skips the reduction (sincos_taylor).
template <int KER, int OP, int NBT, int NBS>
__global__ void __launch_bounds__(kThreads)
    singular_fp64(CellSet test, const int* __restrict__ tdofs, CellSet trial,
                  const int* __restrict__ sdofs, SingularRules rules, SingularPairs pairs,
                  double k, double* __restrict__ out, int64_t ld, int unique_entries,
                  double* __restrict__ pair_values, int trial_lo, int trial_hi) {
  constexpr bool kCplx = KER == kHelmholtz;
  const int lane = threadIdx.x & 31;
  const int pair = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (pair >= pairs.npairs) return;
  const int tc = __ldg(pairs.test_cell + pair), sc = __ldg(pairs.trial_cell + pair);
  if (sc < trial_lo || sc >= trial_hi) return;  // warp-uniform: one pair per warp
  const int cfg = __ldg(pairs.config + pair);
  CellData x, y;
  load_cell(test, tc, x);
  load_cell(trial, sc, y);
  const int off = __ldg(rules.offset + cfg), npts = __ldg(rules.offset + cfg + 1) - off;
  const double dv[3] = {x.v0[0] - y.v0[0], x.v0[1] - y.v0[1], x.v0[2] - y.v0[2]};
  const bool small_phase = kCplx && k * (x.diam + y.diam) <= 0.78;  // same in the whole warp

  double blk_re[NBT][NBS], blk_im[NBT][NBS];
  double S_re = 0.0, S_im = 0.0;
#pragma unroll
  for (int a = 0; a < NBT; ++a)
#pragma unroll
    for (int b = 0; b < NBS; ++b) blk_re[a][b] = blk_im[a][b] = 0.0;

  const double2* txi = reinterpret_cast<const double2*>(rules.test_xi);
  const double2* sxi = reinterpret_cast<const double2*>(rules.trial_xi);
  for (int ii = lane; ii < npts; ii += 32) {
    const int i = off + ii;
    const double2 xi = __ldg(txi + i), et = __ldg(sxi + i);
    const double w = __ldg(rules.w + i);
    double d[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      d[c] = fma(xi.x, x.t0[c], fma(xi.y, x.t1[c], fma(-et.x, y.t0[c], fma(-et.y, y.t1[c], dv[c]))));
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double kre, kim = 0.0;  // w * (kernel factor), see the regular kernels
    if (KER == kLaplace) {
      if (OP == kSL || OP == kHS) {
        kre = w * rsqrt_refined(r2);
      } else {
        const double dn = OP == kDL ? (d[0] * y.n[0] + d[1] * y.n[1] + d[2] * y.n[2])
                                    : -(d[0] * x.n[0] + d[1] * x.n[1] + d[2] * x.n[2]);
        kre = w * dn * rinv3_refined(r2);
      }
    } else {
      const double rinv = rsqrt_refined(r2);
      const double r = r2 * rinv;
      double sn, cs;
      if (small_phase)
        sincos_taylor(k * r, sn, cs);
      else
        sincos_cw(k * r, sn, cs);
      if (OP == kSL || OP == kHS) {
        kre = w * rinv * cs;
        kim = w * rinv * sn;
      } else {
        const double dn = OP == kDL ? (d[0] * y.n[0] + d[1] * y.n[1] + d[2] * y.n[2])
                                    : -(d[0] * x.n[0] + d[1] * x.n[1] + d[2] * x.n[2]);
        const double f = w * dn * rinv * rinv * rinv;
        const double kr = k * r;
        kre = f * fma(kr, sn, cs);
        kim = f * fma(-kr, cs, sn);
      }
    }
    if (OP == kHS) {
      S_re += kre;
      if (kCplx) S_im += kim;
    }
    if (OP != kHS || kCplx) {
      const double psi[3] = {1.0 - et.x - et.y, et.x, et.y};
      if (NBT == 1) {
#pragma unroll
        for (int b = 0; b < NBS; ++b) {
          const double f = NBS == 1 ? 1.0 : psi[b];
          blk_re[0][b] = fma(kre, f, blk_re[0][b]);
          if (kCplx) blk_im[0][b] = fma(kim, f, blk_im[0][b]);
        }
      } else {
        // (kre phi_a) psi_b: three products, then one FMA per block entry
        const double phi[3] = {1.0 - xi.x - xi.y, xi.x, xi.y};
#pragma unroll
        for (int a = 0; a < NBT; ++a) {
          const double vr = kre * phi[a], vi = kim * phi[a];
#pragma unroll
          for (int b = 0; b < NBS; ++b) {
            const double f = NBS == 1 ? 1.0 : psi[b];
            blk_re[a][b] = fma(vr, f, blk_re[a][b]);
            if (kCplx) blk_im[a][b] = fma(vi, f, blk_im[a][b]);
          }
        }
      }
    }
  }
  // warp reduction
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    if (OP == kHS) {
      S_re += __shfl_xor_sync(0xffffffffu, S_re, s);
      if (kCplx) S_im += __shfl_xor_sync(0xffffffffu, S_im, s);
    }
#pragma unroll
    for (int a = 0; a < NBT; ++a)
#pragma unroll
      for (int b = 0; b < NBS; ++b) {
        blk_re[a][b] += __shfl_xor_sync(0xffffffffu, blk_re[a][b], s);
        if (kCplx) blk_im[a][b] += __shfl_xor_sync(0xffffffffu, blk_im[a][b], s);
      }
  }
  if (lane != 0) return;

  const double jj = x.jdet * y.jdet;
  double o_re[NBT][NBS], o_im[NBT][NBS];
  if (OP != kHS) {
#pragma unroll
    for (int a = 0; a < NBT; ++a)
#pragma unroll
      for (int b = 0; b < NBS; ++b) {
        o_re[a][b] = blk_re[a][b] * jj * kInv4Pi;
        o_im[a][b] = blk_im[a][b] * jj * kInv4Pi;
      }
  } else {
    double ct[NBT][3], cs[NBS][3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (NBT == 3) {
        ct[0][d] = x.t0[d] - x.t1[d];
        ct[1][d] = x.t1[d];
        ct[2][d] = -x.t0[d];
      } else {
        ct[0][d] = 0.0;
      }
      if (NBS == 3) {
        cs[0][d] = y.t0[d] - y.t1[d];
        cs[1][d] = y.t1[d];
        cs[2][d] = -y.t0[d];
      } else {
        cs[0][d] = 0.0;
      }
    }
    const double nn = x.n[0] * y.n[0] + x.n[1] * y.n[1] + x.n[2] * y.n[2];
    const double nnsc = -k * k * nn * jj;
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
        o_re[a][b] = re * kInv4Pi;
        o_im[a][b] = im * kInv4Pi;
      }
  }
  if (pair_values) {
    double* pv = pair_values + static_cast<int64_t>(pair) * NBT * NBS * (kCplx ? 2 : 1);
#pragma unroll
    for (int b = 0; b < NBS; ++b)
#pragma unroll
      for (int a = 0; a < NBT; ++a) {
        const int e = a + NBT * b;
        if (kCplx) {
          pv[2 * e] = o_re[a][b];
          pv[2 * e + 1] = o_im[a][b];
        } else {
          pv[e] = o_re[a][b];
        }
      }
  }
  if (out) {
#pragma unroll
    for (int b = 0; b < NBS; ++b) {
      const int64_t col = static_cast<int64_t>(__ldg(sdofs + sc * NBS + b)) * ld;
#pragma unroll
      for (int a = 0; a < NBT; ++a) {
        const int64_t o = col + __ldg(tdofs + tc * NBT + a);
        if (unique_entries) {  // DP0 x DP0: this pair owns the entry
          if (kCplx) {
            reinterpret_cast<double2*>(out)[o] = make_double2(o_re[a][b], o_im[a][b]);
          } else {
            out[o] = o_re[a][b];
          }
        } else {
          if (kCplx) {
            atomicAdd(out + 2 * o, o_re[a][b]);
            atomicAdd(out + 2 * o + 1, o_im[a][b]);
          } else {
            atomicAdd(out + o, o_re[a][b]);
          }
        }
      }
    }
  }
}

template <int KER, int OP, int NBT, int NBS>
cudaError_t launch_one(const CellSet& test, const int* tdofs, const CellSet& trial,
                       const int* sdofs, const SingularRules& rules, const SingularPairs& pairs,
                       const SingularArgs& a, cudaStream_t stream) {
  const int warps = kThreads / 32;
  const int blocks = (pairs.npairs + warps - 1) / warps;
  singular_fp64<KER, OP, NBT, NBS><<<blocks, kThreads, 0, stream>>>(
      test, tdofs, trial, sdofs, rules, pairs, a.k, static_cast<double*>(a.out), a.ld,
      a.unique_entries, a.pair_values, a.trial_lo, a.trial_hi);
  return cudaGetLastError();
}

template <int KER, int OP>
cudaError_t launch_nb(const CellSet& test, const int* tdofs, int nbt, const CellSet& trial,
                      const int* sdofs, int nbs, const SingularRules& rules,
                      const SingularPairs& pairs, const SingularArgs& a, cudaStream_t stream) {
  if (nbt == 1 && nbs == 1)
    return launch_one<KER, OP, 1, 1>(test, tdofs, trial, sdofs, rules, pairs, a, stream);
  if (nbt == 1 && nbs == 3)
    return launch_one<KER, OP, 1, 3>(test, tdofs, trial, sdofs, rules, pairs, a, stream);
  if (nbt == 3 && nbs == 1)
    return launch_one<KER, OP, 3, 1>(test, tdofs, trial, sdofs, rules, pairs, a, stream);
  if (nbt == 3 && nbs == 3)
    return launch_one<KER, OP, 3, 3>(test, tdofs, trial, sdofs, rules, pairs, a, stream);
  return cudaErrorInvalidValue;
}

template <int KER>
cudaError_t launch_op(const CellSet& test, const int* tdofs, int nbt, const CellSet& trial,
                      const int* sdofs, int nbs, const SingularRules& rules,
                      const SingularPairs& pairs, const SingularArgs& a, cudaStream_t stream) {
  switch (a.op) {
    case kSL: return launch_nb<KER, kSL>(test, tdofs, nbt, trial, sdofs, nbs, rules, pairs, a, stream);
    case kDL: return launch_nb<KER, kDL>(test, tdofs, nbt, trial, sdofs, nbs, rules, pairs, a, stream);
    case kADL: return launch_nb<KER, kADL>(test, tdofs, nbt, trial, sdofs, nbs, rules, pairs, a, stream);
    case kHS: return launch_nb<KER, kHS>(test, tdofs, nbt, trial, sdofs, nbs, rules, pairs, a, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_singular(const CellSet& test, const int* test_dofs, int nbt,
                            const CellSet& trial, const int* trial_dofs, int nbs,
                            const SingularRules& rules, const SingularPairs& pairs,
                            const SingularArgs& a, cudaStream_t stream) {
  if (pairs.npairs <= 0) return cudaSuccess;
  if (nbt > 3 || nbs > 3) {  // degree-2 spaces: the generic warp-per-pair kernel
    GenericPairArgs g;
    g.kernel = a.kernel;
    g.op = a.op;
    g.k = a.k;
    g.nbt = nbt;
    g.nbs = nbs;
    g.test = test;
    g.trial = trial;
    g.test_dofs = test_dofs;
    g.trial_dofs = trial_dofs;
    g.rule = RegularRule{};
    g.rules = rules;
    g.pairs = pairs;
    g.singular = true;
    g.same_grid = 1;
    g.out = a.out;
    g.ld = a.ld;
    g.trial_lo = a.trial_lo;
    g.trial_hi = a.trial_hi;
    g.pair_values = a.pair_values;
    return launch_generic_pairs(g, stream);
  }
  return a.kernel == kLaplace
             ? launch_op<kLaplace>(test, test_dofs, nbt, trial, trial_dofs, nbs, rules, pairs, a, stream)
             : launch_op<kHelmholtz>(test, test_dofs, nbt, trial, trial_dofs, nbs, rules, pairs, a, stream);
}

}  // namespace bempp_b200
