// Shared-memory tiles of kTile consecutive cells, staged once per CTA by the regular and
// adjoint kernels: FP64 quadrature points (field-major per point coordinate), optional
// FP32 centroid offsets, per-cell geometry and vertex ids.
#pragma once

#include "launch.h"

namespace bempp_b200 {
namespace tiles {

constexpr int kTile = 32;
constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;

enum TileField : int {
  fJdet = 0, fNx, fNy, fNz, fH, fT0x, fT0y, fT0z, fT1x, fT1y, fT1z, fCx, fCy, fCz, fDiam,
  fRad, kTileFields
};

// Shared-memory image of a tile of kTile cells.
struct Tile {
  double* pts;  // [(q*3+d) * kTile + c] absolute FP64 points
  float4* rel;  // [q * kTile + c] FP32 offset from the centroid (x, y, z) and its
                //   squared length (w) (mixed only)
  double* geo;  // [f * kTile + c]
  int* vid;     // [v * kTile + c]
  int* ldof;    // [b * kTile + c]
  __device__ __forceinline__ double P(int q, int d, int c) const { return pts[(q * 3 + d) * kTile + c]; }
  __device__ __forceinline__ float4 R4(int q, int c) const { return rel[q * kTile + c]; }
  __device__ __forceinline__ float R(int q, int d, int c) const {
    return reinterpret_cast<const float*>(rel + q * kTile + c)[d];
  }
  __device__ __forceinline__ double G(int f, int c) const { return geo[f * kTile + c]; }
};

__host__ __device__ inline size_t tile_doubles(int q) { return (3 * q + kTileFields) * kTile; }
__host__ __device__ inline size_t tile_floats(int q, bool mixed) { return mixed ? 4 * q * kTile : 0; }
__host__ __device__ inline size_t tile_ints(int nb) { return (3 + nb) * kTile; }

// Carves a tile out of shared memory at *cursor rounded up to 16 bytes.
__device__ inline Tile carve_tile(unsigned char*& cursor, int q, bool mixed, int nb) {
  Tile t;
  cursor = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(cursor) + 15) & ~uintptr_t(15));
  t.pts = reinterpret_cast<double*>(cursor);
  t.geo = t.pts + 3 * q * kTile;
  cursor = reinterpret_cast<unsigned char*>(t.geo + kTileFields * kTile);  // 16-B multiple
  t.rel = reinterpret_cast<float4*>(cursor);
  cursor += sizeof(float) * tile_floats(q, mixed);
  t.vid = reinterpret_cast<int*>(cursor);
  t.ldof = t.vid + 3 * kTile;
  cursor += sizeof(int) * tile_ints(nb);
  cursor = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(cursor) + 15) & ~uintptr_t(15));
  return t;
}

__device__ inline void stage_geo(const Tile& t, int c, const CellSet& cs, int cell) {
  const int N = cs.ncells;
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
}

__device__ inline void load_tile(const Tile& t, const CellSet& cs, int c0, int n, int q, bool mixed,
                          const uint8_t* cell_ldof, int nb) {
  const int N = cs.ncells;
  for (int idx = threadIdx.x; idx < 3 * q * kTile; idx += kThreads) {
    const int c = idx % kTile, pd = idx / kTile;
    t.pts[idx] = __ldg(cs.qpts + static_cast<int64_t>(pd) * N + c0 + min(c, n - 1));
  }
  if (mixed)
    for (int idx = threadIdx.x; idx < q * kTile; idx += kThreads) {
      const int c = idx % kTile, p = idx / kTile;
      const float* src = cs.qrel + static_cast<int64_t>(3 * p) * N + c0 + min(c, n - 1);
      const float x = __ldg(src), y = __ldg(src + N), z = __ldg(src + 2 * N);
      t.rel[p * kTile + c] = make_float4(x, y, z, fmaf(x, x, fmaf(y, y, z * z)));
    }
  for (int c = threadIdx.x; c < kTile; c += kThreads) {
    const int cell = c0 + min(c, n - 1);
    stage_geo(t, c, cs, cell);
    for (int v = 0; v < 3; ++v) t.vid[v * kTile + c] = c < n ? __ldg(cs.vids + v * N + cell) : -1 - v;
    for (int b = 0; b < nb; ++b) t.ldof[b * kTile + c] = cell_ldof ? cell_ldof[cell * nb + b] : 0;
  }
}

// One cell's FP64 quadrature points and geometry into column c of a tile (the staging of
// a single lane).
__device__ inline void stage_cell(const Tile& t, int c, const CellSet& cs, int cell, int q) {
  const int N = cs.ncells;
  for (int pd = 0; pd < 3 * q; ++pd)
    t.pts[pd * kTile + c] = __ldg(cs.qpts + static_cast<int64_t>(pd) * N + cell);
  stage_geo(t, c, cs, cell);
}


// ---- FP32 helpers of the mixed-precision paths ----

__device__ __forceinline__ void kahan_add(float& sum, float& comp, float v) {
  const float y = v - comp;
  const float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

// cos(t), sin(t) for |t| <= 0.8: polynomials in z = t^2 of degree 8 (cos) and 7 (sin)
// with the leading coefficient fixed to 1, fitted by minimising the maximum error on
// [-0.8, 0.8] (discrete minimax over 6001 points, a linear program); approximation
// errors 6.5e-11 (cos) and 3.3e-9 (sin), below FP32 rounding.
__device__ __forceinline__ void poly_cos_sin(float t, float& c, float& s) {
  const float z = t * t;
  c = fmaf(z, fmaf(z, fmaf(z, fmaf(z, 2.43751438e-5f, -1.38866017e-3f), 4.16666195e-2f), -0.5f),
           1.0f);
  s = t * fmaf(z, fmaf(z, fmaf(z, -1.95052402e-4f, 8.33209045e-3f), -0.166666538f), 1.0f);
}

__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// cos and sin of an argument of any moderate size: Cody-Waite reduction by multiples of
// pi/2 (two-part constant) to |r| <= pi/4, the polynomials above there, and the
// quadrant's exchange of sine and cosine.  FP32 arguments up to a few hundred.
__device__ __forceinline__ void reduced_cos_sin(float t, float& c, float& s) {
  const float n = rintf(t * 0.636619772f);
  float r = fmaf(-n, 1.57079637f, t);
  r = fmaf(-n, -4.37113883e-8f, r);
  float cr, sr;
  poly_cos_sin(r, cr, sr);
  const int q = static_cast<int>(n) & 3;
  c = (q == 0) ? cr : (q == 1) ? -sr : (q == 2) ? -cr : sr;
  s = (q == 0) ? sr : (q == 1) ? cr : (q == 2) ? -sr : -cr;
}

// e^{i theta} for an FP64 angle: the reduction by pi/2 in FP64 (two-part constant), the
// series and the quadrant in FP32; absolute error ~1e-7.
__device__ __forceinline__ void phase_cos_sin(double theta, float& c, float& s) {
  const double n = rint(theta * 0.63661977236758134308);
  double r = fma(-n, 1.5707963267948966192, theta);
  r = fma(-n, 6.1232339957367660359e-17, r);
  float cr, sr;
  poly_cos_sin(static_cast<float>(r), cr, sr);
  const int q = static_cast<int>(static_cast<long long>(n) & 3);
  c = (q == 0) ? cr : (q == 1) ? -sr : (q == 2) ? -cr : sr;
  s = (q == 0) ? sr : (q == 1) ? cr : (q == 2) ? -sr : -cr;
}

}  // namespace tiles
}  // namespace bempp_b200
