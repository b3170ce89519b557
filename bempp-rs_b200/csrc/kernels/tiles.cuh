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
__device__ inline Tile carve_tile(unsigned char*& cursor, int q, bool mixed, int nb) {
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

__device__ inline void load_tile(const Tile& t, const CellSet& cs, int c0, int n, int q, bool mixed,
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


}  // namespace tiles
}  // namespace bempp_b200
