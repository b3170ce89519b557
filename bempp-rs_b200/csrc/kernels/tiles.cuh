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

// Geometry rows of a tile: the grid's rows kT0x .. kH, in the same order, so that a tile
// is staged by copying whole rows.
enum TileField : int {
  fT0x = 0, fT0y, fT0z, fT1x, fT1y, fT1z, fNx, fNy, fNz, fJdet, fCx, fCy, fCz, fDiam, fRad,
  fH, kTileFields
};
static_assert(kH - kT0x + 1 == kTileFields && kNx - kT0x == fNx && kJdet - kT0x == fJdet &&
                  kCx - kT0x == fCx && kDiam - kT0x == fDiam && kRad - kT0x == fRad,
              "tile rows mirror the grid's geometry rows");

// Shared-memory image of a tile of kTile cells.
struct Tile {
  double* pts;  // [(q*3+d) * kTile + c] absolute FP64 points
  float4* rel;  // [r * kTile + c], r < qrel_rows(q): FP32 offsets from the centroid and
                //   their squared lengths, points in pairs (CellSet::qrel; mixed only)
  double* geo;  // [f * kTile + c]
  int* vid;     // [v * kTile + c]
  int* ldof;    // [b * kTile + c]
  __device__ __forceinline__ double P(int q, int d, int c) const { return pts[(q * 3 + d) * kTile + c]; }
  // point q of cell c: (x, y, z, squared length)
  __device__ __forceinline__ float4 R4(int q, int c) const {
    const float* a = reinterpret_cast<const float*>(rel + (q & ~1) * kTile + c);
    const float* b = reinterpret_cast<const float*>(rel + ((q & ~1) + 1) * kTile + c);
    const int h = q & 1;
    return make_float4(a[h], a[2 + h], b[h], b[2 + h]);
  }
  __device__ __forceinline__ float R(int q, int d, int c) const {
    return reinterpret_cast<const float*>(rel + ((q & ~1) + (d >> 1)) * kTile + c)[2 * (d & 1) + (q & 1)];
  }
  // points 2j, 2j+1 of cell c: (x, x', y, y') and (z, z', |.|^2, |.|^2')
  __device__ __forceinline__ float4 RA(int j, int c) const { return rel[2 * j * kTile + c]; }
  __device__ __forceinline__ float4 RB(int j, int c) const { return rel[(2 * j + 1) * kTile + c]; }
  __device__ __forceinline__ double G(int f, int c) const { return geo[f * kTile + c]; }
};

// pts: the tile holds the FP64 quadrature points (every kernel but the masked mixed ones,
// whose FP64 near pairs are integrated by another kernel)
__host__ __device__ inline size_t tile_doubles(int q, bool pts = true) {
  return ((pts ? 3 * q : 0) + kTileFields) * kTile;
}
__host__ __device__ inline size_t tile_floats(int q, bool mixed) { return mixed ? 4 * qrel_rows(q) * kTile : 0; }
__host__ __device__ inline size_t tile_ints(int nb) { return (3 + nb) * kTile; }
// Bytes of one tile staged by bulk copies (points, geometry, FP32 offsets, vertex ids).
__host__ __device__ inline unsigned bulk_tile_bytes(int q, bool mixed, bool pts = true) {
  return static_cast<unsigned>(sizeof(double) * tile_doubles(q, pts) +
                               sizeof(float) * tile_floats(q, mixed) + sizeof(int) * 3 * kTile);
}

// Carves a tile out of shared memory at *cursor rounded up to 16 bytes.  Every row of
// the tile starts on a 16-byte boundary (the bulk copies' requirement).
__device__ inline Tile carve_tile(unsigned char*& cursor, int q, bool mixed, int nb,
                                  bool pts = true) {
  Tile t;
  cursor = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(cursor) + 15) & ~uintptr_t(15));
  t.pts = reinterpret_cast<double*>(cursor);
  t.geo = t.pts + (pts ? 3 * q * kTile : 0);
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
  for (int f = 0; f < kTileFields; ++f) t.geo[f * kTile + c] = g(cs.geom, kT0x + f, cs.stride, cell);
}

// Local DOF indices of the tile's cells (scatter kernels), by plain loads.
__device__ inline void load_ldof(const Tile& t, int c0, int n, const uint8_t* cell_ldof, int nb) {
  for (int idx = threadIdx.x; idx < nb * kTile; idx += kThreads) {
    const int c = idx % kTile, b = idx / kTile;
    t.ldof[idx] = cell_ldof ? cell_ldof[(c0 + min(c, n - 1)) * nb + b] : 0;
  }
}

// Whole tile by plain loads from all threads (rows of the padded grid arrays; the
// padding cells of the last tile come along and are never used).
__device__ inline void load_tile(const Tile& t, const CellSet& cs, int c0, int n, int q, bool mixed,
                          const uint8_t* cell_ldof, int nb) {
  const int64_t S = cs.stride;
  for (int idx = threadIdx.x; idx < 3 * q * kTile; idx += kThreads) {
    const int c = idx % kTile, pd = idx / kTile;
    t.pts[idx] = __ldg(cs.qpts + pd * S + c0 + c);
  }
  if (mixed)
    for (int idx = threadIdx.x; idx < qrel_rows(q) * kTile; idx += kThreads) {
      const int c = idx % kTile, r = idx / kTile;
      t.rel[idx] = __ldg(cs.qrel + r * S + c0 + c);
    }
  for (int idx = threadIdx.x; idx < kTileFields * kTile; idx += kThreads) {
    const int c = idx % kTile, f = idx / kTile;
    t.geo[idx] = __ldg(cs.geom + (kT0x + f) * S + c0 + c);
  }
  for (int idx = threadIdx.x; idx < 3 * kTile; idx += kThreads) {
    const int c = idx % kTile, v = idx / kTile;
    t.vid[idx] = __ldg(cs.vids + v * S + c0 + c);
  }
  load_ldof(t, c0, n, cell_ldof, nb);
}

// One cell's FP64 quadrature points and geometry into column c of a tile (the staging of
// a single lane).
__device__ inline void stage_cell(const Tile& t, int c, const CellSet& cs, int cell, int q) {
  const int64_t S = cs.stride;
  for (int pd = 0; pd < 3 * q; ++pd) t.pts[pd * kTile + c] = __ldg(cs.qpts + pd * S + cell);
  stage_geo(t, c, cs, cell);
}

// ---- tile staging by bulk (TMA) copies, completed on a shared-memory mbarrier ----

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* m, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(m)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* m, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(m)), "r"(parity)
      : "memory");
  return done != 0;
}

constexpr int kStagePolls = 1 << 22;

// Waits for the mbarrier phase with the given parity, giving up after `polls` polls (each
// poll suspends for a hardware-defined interval): true when it completed.
__device__ inline bool mbar_wait_bounded(uint64_t* m, unsigned parity, int polls = kStagePolls) {
  for (int i = 0; i < polls; ++i)
    if (mbar_try_wait(m, parity)) return true;
  return false;
}

// One 1-D bulk copy global -> shared; both addresses 16-byte aligned, size a multiple of
// 16 bytes; its bytes complete a transaction on the mbarrier.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, uint64_t* m) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(m))
      : "memory");
}

// Issues the bulk copies of one tile (one thread): every row is 32 cells starting at a
// multiple of 32 of a padded grid array, so sources are 256-byte aligned.
__device__ inline void stage_tile_bulk(const Tile& t, const CellSet& cs, int c0, int q, bool mixed,
                                       uint64_t* m, bool pts = true) {
  const int64_t S = cs.stride;
  if (pts)
    for (int pd = 0; pd < 3 * q; ++pd)
      bulk_copy(t.pts + pd * kTile, cs.qpts + pd * S + c0, sizeof(double) * kTile, m);
  for (int f = 0; f < kTileFields; ++f)
    bulk_copy(t.geo + f * kTile, cs.geom + (kT0x + f) * S + c0, sizeof(double) * kTile, m);
  if (mixed)
    for (int r = 0; r < qrel_rows(q); ++r)
      bulk_copy(t.rel + r * kTile, cs.qrel + r * S + c0, sizeof(float4) * kTile, m);
  for (int v = 0; v < 3; ++v) bulk_copy(t.vid + v * kTile, cs.vids + v * S + c0, sizeof(int) * kTile, m);
}

// ---- FP32 helpers of the mixed-precision paths ----

__device__ __forceinline__ void kahan_add(float& sum, float& comp, float v) {
  const float y = v - comp;
  const float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

// cos(t), sin(t) for |t| <= 0.8: cos t ~ 1 + z P(z) of degree 8 and sin t ~ t (1 + z R(z))
// of degree 7 in t (z = t^2), discrete minimax fits (fit_phase_polys.py); approximation
// errors 6.5e-11 (cos) and 2.1e-9 (sin), below FP32 rounding.
__device__ __forceinline__ void poly_cos_sin(float t, float& c, float& s) {
  const float z = t * t;
  c = fmaf(z, fmaf(z, fmaf(z, fmaf(z, 2.437514408e-5f, -1.388660219e-3f), 4.166661828e-2f),
                   -4.999999968e-1f), 1.0f);
  s = t * fmaf(z, fmaf(z, fmaf(z, -1.948277516e-4f, 8.331875683e-3f), -1.666664881e-1f), 1.0f);
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

// Packed FP32x2 arithmetic (sm_100): one instruction, two independently rounded results,
// the same values as the scalar fmaf / + / *.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 rsqrt_approx2(float2 x) {
  return make_float2(rsqrt_approx(x.x), rsqrt_approx(x.y));
}
__device__ __forceinline__ float2 rcp_approx2(float2 x) {
  return make_float2(rcp_approx(x.x), rcp_approx(x.y));
}
// cos(t), sin(t) for |t| <= 1.6 on two arguments: cos of degree 8 and sin of degree 9 in
// t, discrete minimax fits (fit_phase_polys.py 1.6 4 4; errors 6.3e-8 and 5.7e-9, FP32
// rounding), for pairs whose phases exceed the range of poly_cos_sin2 by at most 2x.
__device__ __forceinline__ void poly_cos_sin_wide2(float2 t, float2& c, float2& s) {
  const float2 z = fmul2(t, t);
  c = ffma2(z, ffma2(z, ffma2(z, ffma2(z, f2(2.313598054e-5f), f2(-1.385346181e-3f)),
                              f2(4.166368189e-2f)), f2(-4.999992169e-1f)), f2(1.0f));
  s = fmul2(t, ffma2(z, ffma2(z, ffma2(z, ffma2(z, f2(2.594375954e-6f), f2(-1.980401633e-4f)),
                                       f2(8.332980908e-3f)), f2(-1.666665560e-1f)), f2(1.0f)));
}

// poly_cos_sin on two arguments
__device__ __forceinline__ void poly_cos_sin2(float2 t, float2& c, float2& s) {
  const float2 z = fmul2(t, t);
  // cos of degree 6 here (fit_phase_polys.py 0.8 3 3: max error 3.7e-8, FP32 rounding)
  c = ffma2(z, ffma2(z, ffma2(z, f2(-1.358700830e-3f), f2(4.165550692e-2f)),
                     f2(-4.999988255e-1f)), f2(1.0f));
  s = fmul2(t, ffma2(z, ffma2(z, ffma2(z, f2(-1.948277516e-4f), f2(8.331875683e-3f)),
                              f2(-1.666664881e-1f)), f2(1.0f)));
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
