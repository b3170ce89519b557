// Batched Helmholtz single-layer DP0 frequency sweep: one persistent, CUDA-graph-captured
// launch over many wavenumbers and meshes of uneven size (the regular.cu kernel
// sweep_sl_dp0), with a small autotuner.
//
// Plan.  Work items are (mesh, chunk of wavenumbers, tile pair test tile >= trial tile:
// the kernel mirrors the symmetric single layer), the largest mesh's items first so the
// dynamic item counter ends with short items.  The launch is
// captured once per plan (counter reset + kernel) and replayed with cudaGraphLaunch.
//
// Autotuner.  The free parameters are the tile shape of a work item (1 x 1 or 2 x 2 pairs
// of 32-cell tiles staged together: reuse of staged tiles versus shared memory per CTA),
// the wavenumbers per work item (k-chunk: more reuse of a staged tile pair versus finer
// load balance) and the CTAs per SM of the persistent grid (which also sets the register
// cap of the kernel: 4 or fewer CTAs allow 128 registers, 5 or 6 allow 80).  Each
// candidate runs the kernel on a leading slice of the work items (the first 1/16th, at
// least 148 x 8 items) timed with CUDA events; the fastest is kept per (device, mesh
// sizes, number of wavenumbers) for the life of the process.  The quadrature order is not
// a parameter: the 6-point rule is part of the problem (another order gives another
// matrix).
#include <algorithm>
#include <cstring>
#include <map>
#include <tuple>

#include "core.h"

namespace bempp_b200 {

namespace {

struct SweepPlan {
  std::vector<uint64_t> grids;
  std::vector<void*> outs;
  std::vector<double> ks;
  int device = -1;
  DeviceBuffer d_ks, d_counter;
  SweepArgs args{};
  SweepTuning tuning;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  ~SweepPlan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

std::mutex g_sweep_mu;
std::unique_ptr<SweepPlan> g_plan;  // the most recent plan (replayed while inputs repeat)
std::map<std::tuple<int, std::vector<int64_t>, int>, SweepTuning> g_tuned;
SweepTuning g_last;
SweepTuning g_forced{0, 4, 1, 0.0};  // kchunk > 0: parameters fixed by the caller (no autotuning)

int sm_count(int device) {
  int sms = 0;
  BEMPP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  return sms;
}

long long count_items(SweepArgs& a, int kchunk, int tile_shape) {
  a.kchunk = kchunk;
  a.tile_shape = tile_shape;
  const int nchunks = (a.nk + kchunk - 1) / kchunk;
  long long total = 0;
  for (int m = 0; m < a.nmesh; ++m) {
    a.mesh[m].item_begin = total;
    // super-tile pairs (test >= trial): the kernel mirrors the single layer
    const long long nt = (a.mesh[m].ntiles + tile_shape - 1) / tile_shape;
    total += nt * (nt + 1) / 2 * nchunks;
  }
  a.nitems = total;
  return total;
}

}  // namespace

// Defined in assembler.cpp.
const GridGeometry& sweep_geometry(GridT& g, int device, const RegularRule& rule);
SingularRules sweep_rules(int device, int order);
SingularPairList& sweep_pairs(GridT& g, int device);

void helmholtz_sl_sweep_device(GridT* const* grids, size_t ngrids, const double* ks, size_t nk,
                               const Options& opts, void* const* outs, cudaStream_t stream) {
  if (ngrids == 0 || nk == 0) return;
  if (ngrids > static_cast<size_t>(kMaxSweepMeshes))
    throw Error(kUnsupported, "at most 8 meshes per sweep");
  for (size_t i = 0; i < ngrids; ++i)
    if (grids[i]->quads()) throw Error(kUnsupported, "the sweep needs triangle grids");
  const auto qit = opts.regular.find(kTriangle);
  const auto sit = opts.singular.find({kTriangle, kTriangle});
  if (qit == opts.regular.end() || qit->second != 6)
    throw Error(kUnsupported, "the sweep kernel uses the 6-point regular rule");
  if (sit == opts.singular.end()) throw Error(kInvalidArgument, "no singular quadrature order");
  int device = 0;
  BEMPP_CUDA(cudaGetDevice(&device));
  const RegularRule rule = simplex_rule(6);
  const SingularRules rules = sweep_rules(device, static_cast<int>(sit->second));

  // meshes ordered largest first (their items come first)
  std::vector<size_t> order(ngrids);
  for (size_t i = 0; i < ngrids; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return grids[a]->ncells > grids[b]->ncells; });

  std::lock_guard<std::mutex> lock(g_sweep_mu);
  bool reuse = g_plan && g_plan->device == device && g_plan->grids.size() == ngrids &&
               g_plan->ks == std::vector<double>(ks, ks + nk);
  for (size_t i = 0; reuse && i < ngrids; ++i)
    reuse = g_plan->grids[i] == grids[i]->uid && g_plan->outs[i] == outs[i];
  if (!reuse) {
    auto plan = std::make_unique<SweepPlan>();
    plan->device = device;
    for (size_t i = 0; i < ngrids; ++i) plan->grids.push_back(grids[i]->uid);
    plan->outs.assign(outs, outs + ngrids);
    plan->ks.assign(ks, ks + nk);
    plan->d_ks.upload(plan->ks);
    plan->d_counter.alloc(sizeof(unsigned long long));
    SweepArgs& a = plan->args;
    std::vector<int64_t> sizes;
    for (size_t r = 0; r < ngrids; ++r) {
      const size_t i = order[r];
      if (!outs[i]) throw Error(kInvalidArgument, "null sweep output");
      const GridGeometry& geo = sweep_geometry(*grids[i], device, rule);
      SweepMesh& m = a.mesh[r];
      m.cells.ncells = static_cast<int>(grids[i]->ncells);
      m.cells.stride = cell_stride(m.cells.ncells);
      m.cells.geom = geo.geom.as<double>();
      m.cells.qpts = geo.qpts.as<double>();
      m.cells.qrel = geo.qrel.as<float4>();
      m.cells.vids = geo.vids.as<int>();
      m.out = static_cast<float2*>(outs[i]);
      m.ntiles = static_cast<int>((grids[i]->ncells + 31) / 32);
      // near field of the mesh with itself (the masks the far-pair kernel skips, the near
      // pairs) and its vertex-sharing pairs
      const NearField& nf = near_field(*grids[i], *grids[i]);
      m.tile_mask = nf.tile_mask.as<int>();
      m.masks = nf.masks.as<unsigned>();
      m.near_pairs = nf.pairs.as<int2>();
      m.nnear = nf.npairs;
      SingularPairList& pl = sweep_pairs(*grids[i], device);
      m.sing = SingularPairs{static_cast<int>(pl.test_cell.size()), pl.d_test.as<int>(),
                             pl.d_trial.as<int>(), pl.d_config.as<int>()};
      sizes.push_back(grids[i]->ncells);
    }
    a.nmesh = static_cast<int>(ngrids);
    a.near_begin[0] = a.sing_begin[0] = 0;
    for (size_t r = 0; r < ngrids; ++r) {
      a.near_begin[r + 1] = a.near_begin[r] + static_cast<long long>(a.mesh[r].nnear) * nk;
      a.sing_begin[r + 1] = a.sing_begin[r] + static_cast<long long>(a.mesh[r].sing.npairs) * nk;
    }
    a.ks = plan->d_ks.as<double>();
    a.nk = static_cast<int>(nk);
    a.counter = plan->d_counter.as<unsigned long long>();
    const int sms = sm_count(device);

    // autotune once per (device, mesh sizes, nk), unless the caller fixed the parameters
    const auto key = std::make_tuple(device, sizes, static_cast<int>(nk));
    auto it = g_tuned.find(key);
    if (g_forced.kchunk > 0) {
      g_tuned[key] = g_forced;
      it = g_tuned.find(key);
    } else if (it == g_tuned.end()) {
      cudaStream_t ts;
      BEMPP_CUDA(cudaStreamCreateWithFlags(&ts, cudaStreamNonBlocking));
      cudaEvent_t e0, e1;
      BEMPP_CUDA(cudaEventCreate(&e0));
      BEMPP_CUDA(cudaEventCreate(&e1));
      SweepTuning best;
      best.probe_ms = 1e30;
      for (int shape : {1, 2}) {
        // CTAs per SM that fit the shape's shared memory (227 KB per SM)
        const int fit = static_cast<int>((227u << 10) / (sweep_smem_bytes(shape) + 1024));
        for (int kchunk : {1, 2, 4, 8, 16, 32}) {
          if (kchunk > static_cast<int>(nk) && kchunk != 1) continue;
          for (int bps : {2, 3, 4, 5, 6}) {
            if (bps > fit) continue;
            SweepArgs probe = a;
            const long long full = count_items(probe, kchunk, shape);
            // a leading slice: same per-item mix as the largest mesh, ~1/16 of the work
            probe.nitems = std::min<long long>(full, std::max<long long>(full / 16, 8LL * sms));
            BEMPP_CUDA(cudaMemsetAsync(probe.counter, 0, sizeof(unsigned long long), ts));
            BEMPP_CUDA(cudaEventRecord(e0, ts));
            BEMPP_CUDA(launch_sweep_sl(probe, rule, rules, bps, sms, ts));
            BEMPP_CUDA(cudaEventRecord(e1, ts));
            BEMPP_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            BEMPP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            // milliseconds per (tile pair, wavenumber)
            const double per_unit = ms / static_cast<double>(probe.nitems) / kchunk /
                                    (shape * shape);
            if (per_unit < best.probe_ms) {
              best.probe_ms = per_unit;
              best.kchunk = kchunk;
              best.blocks_per_sm = bps;
              best.tile_shape = shape;
            }
          }
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      cudaStreamDestroy(ts);
      it = g_tuned.emplace(key, best).first;
    }
    plan->tuning = it->second;
    count_items(a, plan->tuning.kchunk, plan->tuning.tile_shape);

    // capture: counter reset + the persistent far-pair launch on one branch, the FP64
    // near and vertex-sharing launches on a forked branch (they write disjoint entries)
    cudaStream_t cs, side;
    cudaEvent_t fork, join;
    BEMPP_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    BEMPP_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    BEMPP_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    BEMPP_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    BEMPP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaError_t e1 = cudaEventRecord(fork, cs);
    if (e1 == cudaSuccess) e1 = cudaStreamWaitEvent(side, fork, 0);
    if (e1 == cudaSuccess) e1 = launch_sweep_near_singular(a, rule, rules, side);
    if (e1 == cudaSuccess) e1 = cudaEventRecord(join, side);
    cudaError_t e2 = e1 == cudaSuccess ? cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), cs) : e1;
    if (e2 == cudaSuccess) e2 = launch_sweep_sl(a, rule, rules, plan->tuning.blocks_per_sm, sms, cs);
    if (e2 == cudaSuccess && e1 == cudaSuccess) e2 = cudaStreamWaitEvent(cs, join, 0);
    cudaError_t e3 = cudaStreamEndCapture(cs, &plan->graph);
    cudaStreamDestroy(cs);
    cudaStreamDestroy(side);
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
    BEMPP_CUDA(e1);
    BEMPP_CUDA(e2);
    BEMPP_CUDA(e3);
    BEMPP_CUDA(cudaGraphInstantiate(&plan->exec, plan->graph, 0));
    g_plan = std::move(plan);
  }
  g_last = g_plan->tuning;
  BEMPP_CUDA(cudaGraphLaunch(g_plan->exec, stream));
}

void set_sweep_tuning(int kchunk, int blocks_per_sm, int tile_shape) {
  std::lock_guard<std::mutex> lock(g_sweep_mu);
  g_plan.reset();  // the next sweep builds (and captures) a new plan
  if (kchunk <= 0) {
    g_forced = SweepTuning{};
    g_forced.kchunk = 0;
    g_tuned.clear();
    return;
  }
  if (blocks_per_sm < 1 || blocks_per_sm > 6 || (tile_shape != 1 && tile_shape != 2))
    throw Error(kInvalidArgument, "blocks per SM must be 1..6 and the tile shape 1 or 2");
  g_forced.kchunk = kchunk;
  g_forced.blocks_per_sm = blocks_per_sm;
  g_forced.tile_shape = tile_shape;
  g_forced.probe_ms = 0.0;
}

SweepTuning last_sweep_tuning() {
  std::lock_guard<std::mutex> lock(g_sweep_mu);
  return g_last;
}

}  // namespace bempp_b200
