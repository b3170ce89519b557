// Order of the tile pairs of a lower-triangle launch (a symmetric operator on one space,
// the adjoint gradient, the batched sweep): block b -> (test tile tx, trial tile sy) with
// tx >= sy, sy in [ty0, ty1), tx in [sy, ntt).  Shared by the kernels and the host (the
// C-ABI exports the host copy for a self-check).
//
// The trial tiles are cut into bands of kTileBand rows; a band's pairs run test tile by
// test tile, its rows fastest.  The CTAs resident at one time (about 740 on a B200) then
// cover ~46 test tiles x 16 trial tiles, so both the direct and the mirrored blocks they
// write fall in a few hundred 2 MB pages of the output.  Row by row (all test tiles of one
// trial tile), the mirrored blocks spread over every column of the matrix: on a 6.7 GB
// output that touched every page at once.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define BEMPP_HD __host__ __device__ __forceinline__
#else
#define BEMPP_HD inline
#endif

namespace bempp_b200 {

constexpr int kTileBand = 16;

// Pairs of a lower-triangle launch over trial tiles [ty0, ty1) of ntt test tiles.
BEMPP_HD long long lower_tile_pair_count(int ntt, int ty0, int ty1) {
  const long long r = ty1 - ty0;
  return r * ntt - (r * ty0 + r * (r - 1) / 2);
}

BEMPP_HD void lower_tile_pair(long long b, int ntt, int ty0, int ty1, int& tx, int& sy) {
  const long long N = ntt, a = ty0, H = kTileBand, rows = ty1 - ty0;
  // pairs with sy in [a, a + r)
  auto before = [&](long long r) { return r * N - (r * a + r * (r - 1) / 2); };
  long long lo = 0, hi = (rows + H - 1) / H - 1;  // the last band starting at or before b
  while (lo < hi) {
    const long long mid = (lo + hi + 1) / 2;
    if (before(mid * H) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  const long long r0 = a + lo * H, h = rows - lo * H < H ? rows - lo * H : H;
  long long l = b - before(lo * H);
  const long long tri = h * (h + 1) / 2;  // test tiles r0 .. r0 + h - 1: 1, 2, .., h rows
  if (l < tri) {
    long long m = static_cast<long long>((::sqrt(8.0 * static_cast<double>(l) + 1.0) - 1.0) * 0.5);
    while (m > 0 && m * (m + 1) / 2 > l) --m;
    while ((m + 1) * (m + 2) / 2 <= l) ++m;
    tx = static_cast<int>(r0 + m);
    sy = static_cast<int>(r0 + l - m * (m + 1) / 2);
  } else {
    l -= tri;
    tx = static_cast<int>(r0 + h + l / h);
    sy = static_cast<int>(r0 + l % h);
  }
}

}  // namespace bempp_b200
