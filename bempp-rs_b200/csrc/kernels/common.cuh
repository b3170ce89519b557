// Device-side data layout and Green's-function math shared by the assembly kernels.
//
// Layout in HBM (one allocation per grid, field-major so that a warp reading 32
// consecutive cells of one field issues one 256-byte transaction).  Rows have the stride
// S = ncells rounded up to a multiple of 32 (cell_stride), so that every 32-cell tile of
// every row starts on a 256-byte boundary and can be staged by bulk (TMA) copies; the
// padding cells hold zero geometry and vertex ids -1, -2, -3:
//   geom[f * S + c], f in GeomField          per-cell FP64 geometry of a flat triangle
//   qpts[(p * 3 + d) * S + c]                physical regular quadrature point p of cell c
//   qrel[p * S + c]                          float4: FP32 offset of that point from the
//                                            centroid (x, y, z) and its squared length (w)
//   vids[i * S + c], i = 0..2                vertex (point) indices, for adjacency tests
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bempp_b200 {

enum GeomField : int {
  kV0x = 0, kV0y, kV0z,      // vertex 0
  kT0x, kT0y, kT0z,          // t0 = v1 - v0 (Jacobian column 0)
  kT1x, kT1y, kT1z,          // t1 = v2 - v0 (Jacobian column 1)
  kNx, kNy, kNz,             // unit normal (t0 x t1) / |t0 x t1|
  kJdet,                     // |t0 x t1| = 2 * area
  kCx, kCy, kCz,             // centroid
  kDiam,                     // element diameter (longest edge)
  kRad,                      // largest distance from the centroid to a vertex
  kH,                        // v0 . n (the plane's offset)
  kNumGeomFields
};

// Row stride of the per-cell arrays of a grid with n cells.
__host__ __device__ inline int cell_stride(int n) { return (n + 31) & ~31; }

constexpr int kMaxRegularPoints = 37;

// Rows of FP32 offsets of an npts-point rule: points in pairs (a zero point completes an
// odd rule), so that packed FP32x2 arithmetic reads two trial points per 128-bit load.
__host__ __device__ inline int qrel_rows(int npts) { return (npts + 1) & ~1; }
constexpr double kInv4Pi = 0.079577471545947667884;

// Regular (non-singular) rule on the reference triangle (0,0),(1,0),(0,1), passed by
// value so it sits in the kernel's constant parameter bank.
struct RegularRule {
  int npts;
  double w[kMaxRegularPoints];
  double xi[2 * kMaxRegularPoints];
  // FP32 copies for the mixed-precision kernels: weights, and the point offsets from
  // the centroid in reference coordinates, (u, v) = xi - (1/3, 1/3).
  float wf[kMaxRegularPoints];
  float uf[kMaxRegularPoints];
  float vf[kMaxRegularPoints];
  // P1 basis values phi_b(xi_q) = (1 - x - y, x, y) at each point, FP64 and FP32
  double phi[3][kMaxRegularPoints];
  float phif[3][kMaxRegularPoints];
  // FP64 offsets from the centroid in reference coordinates, (u, v) = xi - (1/3, 1/3),
  // and the weights times the P1 basis values, w_q phi_b(xi_q)
  double u[kMaxRegularPoints];
  double v[kMaxRegularPoints];
  double wphi[3][kMaxRegularPoints];
  // Lagrange degree 2 (vertices, then the midpoints of edges [1,2], [0,2], [0,1]) at each
  // point, and times the weights
  double phi2[6][kMaxRegularPoints];
  double wphi2[6][kMaxRegularPoints];
};

#ifdef __CUDACC__
// Basis value of function b at rule point q for a space of nb functions per cell (1, 3 or
// 6), plain or times the weight.
template <int NB>
__device__ __forceinline__ double rule_phi(const RegularRule& r, int b, int q) {
  if constexpr (NB == 6) return r.phi2[b][q];
  else if constexpr (NB == 3) return r.phi[b][q];
  else return 1.0;
}
template <int NB>
__device__ __forceinline__ double rule_wphi(const RegularRule& r, int b, int q) {
  if constexpr (NB == 6) return r.wphi2[b][q];
  else if constexpr (NB == 3) return r.wphi[b][q];
  else return r.w[q];
}
#endif

struct CellSet {
  int ncells;
  int stride;           // cell_stride(ncells)
  const double* geom;   // kNumGeomFields * stride
  const double* qpts;   // npts * 3 * stride
  const float4* qrel;   // qrel_rows(npts) * stride (mixed precision only), points in pairs:
                        // row 2j (x_2j, x_2j+1, y_2j, y_2j+1), row 2j+1 (z_2j, z_2j+1,
                        // |.|^2_2j, |.|^2_2j+1) of the FP32 offsets from the centroid
  const int* vids;      // 3 * stride
};

// Kernel families and operators (OperatorType values of the C-ABI).
enum KernelKind : int { kLaplace = 0, kHelmholtz = 1 };
enum OpKind : int { kSL = 0, kDL = 1, kADL = 2, kHS = 3 };

struct cdouble {
  double re, im;
};

#ifdef __CUDACC__
__device__ __forceinline__ double g(const double* geom, int field, int n, int c) {
  return __ldg(geom + static_cast<int64_t>(field) * n + c);
}

__device__ __forceinline__ bool share_vertex(int a0, int a1, int a2, int b0, int b1, int b2) {
  return a0 == b0 || a0 == b1 || a0 == b2 || a1 == b0 || a1 == b1 || a1 == b2 || a2 == b0 ||
         a2 == b1 || a2 == b2;
}

// 1/sqrt(a) for normal positive FP64 a without a special-case branch: the hardware
// approximation rsqrt.approx.ftz.f64 (PTX) refined by one step of the binomial series
// (1 - e)^(-1/2) = 1 + e/2 + 3e^2/8 + O(e^3) with e = 1 - a y^2, which cubes the
// relative error of the seed.  Only used for distances between distinct quadrature
// points (a > 0, far from the subnormal range).
__device__ __forceinline__ double rsqrt_refined(double a) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  const double e = fma(-a * y, y, 1.0);
  return fma(y * e, fma(e, 0.375, 0.5), y);
}

// sin(r) and cos(r) in FP64 for |r| <= pi/4: Taylor series up to r^17 and r^16
// (truncation below 1e-19).
__device__ __forceinline__ void sincos_taylor(double r, double& sr, double& cr) {
  const double z = r * r;
  cr = 1.0 / 20922789888000.0;  // 1/16!
  cr = fma(cr, z, -1.0 / 87178291200.0);
  cr = fma(cr, z, 1.0 / 479001600.0);
  cr = fma(cr, z, -1.0 / 3628800.0);
  cr = fma(cr, z, 1.0 / 40320.0);
  cr = fma(cr, z, -1.0 / 720.0);
  cr = fma(cr, z, 1.0 / 24.0);
  cr = fma(cr, z, -0.5);
  cr = fma(cr, z, 1.0);
  sr = 1.0 / 355687428096000.0;  // 1/17!
  sr = fma(sr, z, -1.0 / 1307674368000.0);
  sr = fma(sr, z, 1.0 / 6227020800.0);
  sr = fma(sr, z, -1.0 / 39916800.0);
  sr = fma(sr, z, 1.0 / 362880.0);
  sr = fma(sr, z, -1.0 / 5040.0);
  sr = fma(sr, z, 1.0 / 120.0);
  sr = fma(sr, z, -1.0 / 6.0);
  sr = r * fma(sr, z, 1.0);
}

// sin(t) and cos(t) in FP64 for |t| <= 0.8 (pair-referenced phases k (r - r0) of the
// FP64 regular kernels): cos t = 1 + z P(z), sin t = t + t z Q(z), z = t^2, with P and Q of
// degree 5 from a near-minimax fit at 50 digits (fit_phase_polys.py fp64); max abs
// errors 2.5e-16 (cos) and 1.9e-17 (sin) on |t| <= 0.8.
__device__ __forceinline__ void sincos_small(double t, double& s, double& c) {
  const double z = t * t;
  double p = 2.0657616391477202e-09;
  p = fma(p, z, -2.755574396426964e-07);
  p = fma(p, z, 2.4801582078024058e-05);
  p = fma(p, z, -0.0013888888881056654);
  p = fma(p, z, 0.04166666666662371);
  p = fma(p, z, -0.4999999999999996);
  c = fma(z, p, 1.0);
  double q = 1.5912864224903485e-10;
  q = fma(q, z, -2.5051057394492127e-08);
  q = fma(q, z, 2.7557315738586845e-06);
  q = fma(q, z, -0.00019841269836043575);
  q = fma(q, z, 0.008333333333330467);
  q = fma(q, z, -0.16666666666666663);
  s = fma(t * z, q, t);
}

// sin(t) and cos(t) in FP64 for moderate |t| (the phases k r of boundary-element
// kernels): Cody-Waite reduction r = t - n pi/2 with pi/2 split into two doubles (each
// step one fused multiply-add), sincos_taylor on |r| <= pi/4, and the quadrant's exchange
// of sine and cosine.  Absolute error about 1e-16 for |t| up to 1e5 (checked against libm
// on [-40, 40]).
__device__ __forceinline__ void sincos_cw(double t, double& s, double& c) {
  const double n = rint(t * 0.63661977236758134308);
  double r = fma(-n, 1.5707963267948966192, t);
  r = fma(-n, 6.1232339957367660359e-17, r);
  double sr, cr;
  sincos_taylor(r, sr, cr);
  const int q = static_cast<int>(static_cast<long long>(n) & 3);
  c = (q == 0) ? cr : (q == 1) ? -sr : (q == 2) ? -cr : sr;
  s = (q == 0) ? sr : (q == 1) ? cr : (q == 2) ? -sr : -cr;
}

// a^(-3/2) for normal positive FP64 a: the rsqrt.approx.ftz.f64 seed y refined by the
// series (1 - e)^(-3/2) = 1 + 3e/2 + 15e^2/8 + O(e^3) with e = 1 - a y^2 (the inverse cube
// of a distance from its square, for double-layer kernels).
__device__ __forceinline__ double rinv3_refined(double a) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  const double y2 = y * y;
  const double e = fma(-a, y2, 1.0);
  const double y3 = y2 * y;
  return fma(y3 * e, fma(e, 1.875, 1.5), y3);
}

// Lagrange basis of NB functions (1: degree 0, 3: degree 1, 6: degree 2 in ndelement's
// order: vertices 0, 1, 2, then the midpoints of edges [1,2], [0,2], [0,1]) at (x, y):
// values and derivatives along the two reference axes.
template <int NB>
__device__ __forceinline__ void lagrange_basis(double x, double y, double v[NB], double d0[NB],
                                      double d1[NB]) {
  if (NB == 1) {
    v[0] = 1.0;
    d0[0] = d1[0] = 0.0;
  } else {
    const double l[3] = {1.0 - x - y, x, y};
    const double g0[3] = {-1.0, 1.0, 0.0}, g1[3] = {-1.0, 0.0, 1.0};
    if (NB == 3) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        v[i] = l[i];
        d0[i] = g0[i];
        d1[i] = g1[i];
      }
    } else {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        v[i] = l[i] * (2.0 * l[i] - 1.0);
        d0[i] = (4.0 * l[i] - 1.0) * g0[i];
        d1[i] = (4.0 * l[i] - 1.0) * g1[i];
      }
      const int ea[3] = {1, 0, 0}, eb[3] = {2, 2, 1};
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        const int a = ea[e], b = eb[e];
        v[3 + e] = 4.0 * l[a] * l[b];
        d0[3 + e] = 4.0 * (l[a] * g0[b] + l[b] * g0[a]);
        d1[3 + e] = 4.0 * (l[a] * g1[b] + l[b] * g1[a]);
      }
    }
  }
}

// P1 basis on the reference triangle: phi0 = 1 - x - y, phi1 = x, phi2 = y.
__device__ __forceinline__ void p1_basis(double x, double y, double* phi) {
  phi[0] = 1.0 - x - y;
  phi[1] = x;
  phi[2] = y;
}
#endif  // __CUDACC__

}  // namespace bempp_b200
