// Per-cell geometry of flat triangles: the affine map x(xi) = v0 + xi0 t0 + xi1 t1, its
// Jacobian columns, unit normal, Jacobian determinant |t0 x t1|, centroid, diameter and
// the physical regular quadrature points (FP64, plus FP32 offsets from the centroid for
// the mixed-precision kernels, stored in pairs of points: CellSet::qrel).  Restates the ndgrid geometry map that bempp-rs calls at
// src/boundary_assemblers/cell_pair_assemblers.rs:87-108,224-236 for degree-1 cells.
#include "launch.h"

namespace bempp_b200 {

__global__ void geometry_kernel(const double* __restrict__ points, const int* __restrict__ cells,
                                const int* __restrict__ topo, int n, RegularRule rule,
                                double* __restrict__ geom,
                                double* __restrict__ qpts, float4* __restrict__ qrel,
                                int* __restrict__ vids) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int S = cell_stride(n);
  if (c >= S) return;
  if (c >= n) {  // padding of the last tile
    for (int f = 0; f < kNumGeomFields; ++f) geom[static_cast<int64_t>(f) * S + c] = 0.0;
    for (int p = 0; p < rule.npts; ++p)
      for (int k = 0; k < 3; ++k) qpts[static_cast<int64_t>(p * 3 + k) * S + c] = 0.0;
    if (qrel)
      for (int r = 0; r < qrel_rows(rule.npts); ++r)
        qrel[static_cast<int64_t>(r) * S + c] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = 0; i < 3; ++i) vids[i * S + c] = -1 - i;
    return;
  }
  int i0 = cells[3 * c], i1 = cells[3 * c + 1], i2 = cells[3 * c + 2];
  double a[3], b[3], d[3];
  for (int k = 0; k < 3; ++k) {
    a[k] = points[3 * i0 + k];
    b[k] = points[3 * i1 + k];
    d[k] = points[3 * i2 + k];
  }
  double t0[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double t1[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
  double cr[3] = {t0[1] * t1[2] - t0[2] * t1[1], t0[2] * t1[0] - t0[0] * t1[2],
                  t0[0] * t1[1] - t0[1] * t1[0]};
  double jdet = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  double cen[3] = {(a[0] + b[0] + d[0]) / 3.0, (a[1] + b[1] + d[1]) / 3.0,
                   (a[2] + b[2] + d[2]) / 3.0};
  auto dist = [](const double* p, const double* q) {
    double x = p[0] - q[0], y = p[1] - q[1], z = p[2] - q[2];
    return sqrt(x * x + y * y + z * z);
  };
  double diam = fmax(dist(a, b), fmax(dist(a, d), dist(b, d)));
  double rad = fmax(dist(a, cen), fmax(dist(b, cen), dist(d, cen)));
  const double nrm[3] = {cr[0] / jdet, cr[1] / jdet, cr[2] / jdet};
  double vals[kNumGeomFields] = {a[0], a[1], a[2], t0[0], t0[1], t0[2], t1[0], t1[1], t1[2],
                                 nrm[0], nrm[1], nrm[2], jdet,
                                 cen[0], cen[1], cen[2], diam, rad,
                                 a[0] * nrm[0] + a[1] * nrm[1] + a[2] * nrm[2]};
  for (int f = 0; f < kNumGeomFields; ++f) geom[static_cast<int64_t>(f) * S + c] = vals[f];
  for (int p = 0; p < qrel_rows(rule.npts); ++p) {
    float r[4] = {0.f, 0.f, 0.f, 0.f};  // the zero point completing an odd rule
    if (p < rule.npts) {
      const double x0 = rule.xi[2 * p], x1 = rule.xi[2 * p + 1];
      for (int k = 0; k < 3; ++k) {
        qpts[static_cast<int64_t>(p * 3 + k) * S + c] = a[k] + x0 * t0[k] + x1 * t1[k];
        r[k] = static_cast<float>(x0 * t0[k] + x1 * t1[k] + (a[k] - cen[k]));
      }
      r[3] = fmaf(r[0], r[0], fmaf(r[1], r[1], r[2] * r[2]));
    }
    if (qrel) {
      // point p is half (p & 1) of the pair rows 2 (p / 2), 2 (p / 2) + 1
      float* row0 = reinterpret_cast<float*>(qrel + static_cast<int64_t>(p & ~1) * S + c);
      float* row1 = reinterpret_cast<float*>(qrel + static_cast<int64_t>((p & ~1) + 1) * S + c);
      row0[p & 1] = r[0];
      row0[2 + (p & 1)] = r[1];
      row1[p & 1] = r[2];
      row1[2 + (p & 1)] = r[3];
    }
  }
  // vertex ids for adjacency tests: the topology's when it has its own numbering
  vids[c] = topo ? topo[3 * c] : i0;
  vids[S + c] = topo ? topo[3 * c + 1] : i1;
  vids[2 * S + c] = topo ? topo[3 * c + 2] : i2;
}

cudaError_t launch_geometry(const double* points, const int* cells, const int* topo,
                            int ncells, const RegularRule& rule, double* geom, double* qpts,
                            float4* qrel, int* vids, cudaStream_t stream) {
  if (ncells <= 0) return cudaSuccess;
  int threads = 128;
  int blocks = (cell_stride(ncells) + threads - 1) / threads;
  geometry_kernel<<<blocks, threads, 0, stream>>>(points, cells, topo, ncells, rule, geom,
                                                  qpts, qrel, vids);
  return cudaGetLastError();
}

}  // namespace bempp_b200
