// Device-side data layout and Green's-function math shared by the assembly kernels.
//
// Layout in HBM (one allocation per grid, field-major so that a warp reading 32
// consecutive cells of one field issues one 256-byte transaction):
//   geom[f * ncells + c], f in GeomField     per-cell FP64 geometry of a flat triangle
//   qpts[(p * 3 + d) * ncells + c]           physical regular quadrature point p of cell c
//   qrel[(p * 3 + d) * ncells + c]           FP32 offset of that point from the centroid
//   vids[i * ncells + c], i = 0..2           vertex (point) indices, for adjacency tests
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
  kNumGeomFields
};

constexpr int kMaxRegularPoints = 37;
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
};

struct CellSet {
  int ncells;
  const double* geom;   // kNumGeomFields * ncells
  const double* qpts;   // npts * 3 * ncells
  const float* qrel;    // npts * 3 * ncells (mixed precision only)
  const int* vids;      // 3 * ncells
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

// P1 basis on the reference triangle: phi0 = 1 - x - y, phi1 = x, phi2 = y.
__device__ __forceinline__ void p1_basis(double x, double y, double* phi) {
  phi[0] = 1.0 - x - y;
  phi[1] = x;
  phi[2] = y;
}
#endif  // __CUDACC__

}  // namespace bempp_b200
