"""Benchmark: dense boundary-operator assembly on B200.

Workload (default): Laplace double-layer, adjoint double-layer and hypersingular
operators, continuous P1 trial and test spaces, f64, on the unit icosphere refined 5
times (20,480 flat triangles, 10,242 vertices) with a seeded radial perturbation
U(-0.02, 0.02) (numpy default_rng(20480)); regular pairs use the 6-point symmetric rule,
singular pairs order-4 Duffy rules.  One step assembles all three 10,242 x 10,242
matrices (314.7 M entries).  The metric is dense entries per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value: device-resident assembly (geometry cached, output in HBM), max over ranks.
e2e:   the same step through the C-ABI host path a user calls (grid and spaces built
       from host arrays, assemble_into_memory into host numpy arrays).
--impl reference: the CPU FP64 oracle (a restatement of the bempp-rs algorithm, which
       cannot be compiled here: no Rust toolchain) timed on a bounded sample of the same
       workload on all host cores.
Multi-GPU (torchrun): every rank assembles its own copy of the workload (weak scaling,
no collective on the data path).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "bempp-rs_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

LEVEL = 5
SEED = 20480
Q_REGULAR = 6
ORDER = 4
OPERATORS = ["double_layer", "adjoint_double_layer", "hypersingular"]
# Algorithmic FLOPs per regular P1 x P1 cell pair at Q = 6 (36 point pairs): kernel +
# factorised basis accumulation, transcendental = 1, per-cell constants hoisted.
FLOPS_PER_PAIR = {"double_layer": 990, "adjoint_double_layer": 990, "hypersingular": 459}
METRIC = "dense entries/s (Laplace DL+ADL+HS, P1, f64, 20480-triangle icosphere)"


def workload_mesh():
    from bempp import shapes

    pts, cells = shapes.icosphere(LEVEL)
    return shapes.radial_perturbation(pts, SEED), cells


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_spaces(points, cells):
    from bempp.function_space import function_space
    from ndelement.ciarlet import Continuity, Family, create_family
    from ndgrid.grid import Grid

    grid = Grid(points, cells)
    p1 = function_space(grid, create_family(Family.Lagrange, 1, Continuity.Standard))
    return grid, p1


def make_assemblers(precision_name="FP64"):
    from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType, Precision,
                                         create_laplace_assembler)
    from ndelement.reference_cell import ReferenceCellType

    ops = {"double_layer": OperatorType.DoubleLayer,
           "adjoint_double_layer": OperatorType.AdjointDoubleLayer,
           "hypersingular": OperatorType.Hypersingular}
    out = []
    for name in OPERATORS:
        o = BoundaryAssemblerOptions()
        o.set_regular_quadrature_degree(ReferenceCellType.Triangle, Q_REGULAR)
        o.set_singular_quadrature_degree(ReferenceCellType.Triangle, ReferenceCellType.Triangle,
                                         ORDER)
        o.set_precision(getattr(Precision, precision_name))
        out.append((name, create_laplace_assembler(ops[name], o)))
    return out


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    from bempp import _lib

    points, cells = workload_mesh()
    grid, space = build_spaces(points, cells)
    n = space.global_size
    assemblers = make_assemblers("FP64")
    outs = [torch.empty((n, n), dtype=torch.float64, device="cuda") for _ in assemblers]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def step(timing=False):
        launches = 0
        for (name, a), out in zip(assemblers, outs):
            a.set_timing(timing)
            a.assemble_into_device(space, space, out, stream)
            launches += a.launch_count()
        flush.fill_(1.0)  # L2 flush between steps (256 MiB > 126 MB L2)
        return launches + 1

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # kernel-level timing of the regular (dominant) kernel, live, on the same stream
    regular_ms = {}
    for name, a in assemblers:
        a.set_timing(True)
    step(timing=True)
    torch.cuda.synchronize()
    for name, a in assemblers:
        ph = a.phase_times()  # geometry, clear, regular, singular
        regular_ms[name] = ph[2] if len(ph) > 2 else float("nan")
        a.set_timing(False)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    launches = 0
    for _ in range(args.steps):
        launches += step()
    t1.record()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = t0.elapsed_time(t1)
    if world > 1:
        import torch.distributed as dist

        tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    ms_per_step = ms / args.steps
    entries_per_step = len(assemblers) * n * n
    value = world * entries_per_step / (ms_per_step * 1e-3)

    # end-to-end through the public API with host buffers (one replica per rank)
    e2e = None
    if not args.skip_e2e:
        torch.cuda.synchronize()
        pts_h = np.ascontiguousarray(points)
        cells_h = np.ascontiguousarray(cells)
        e2e_steps = max(1, min(args.steps, 3))
        barrier()
        t = time.perf_counter()
        for _ in range(e2e_steps):
            g2, s2 = build_spaces(pts_h, cells_h)
            for name, a in assemblers:
                a.assemble(s2, s2)
            del s2, g2
        e2e_s = (time.perf_counter() - t) / e2e_steps
        if world > 1:
            import torch.distributed as dist

            tt = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_s = float(tt.item())
        e2e = {"value": world * entries_per_step / e2e_s, "unit": "entries/s",
               "h2d_bytes_per_step": int(pts_h.nbytes + cells_h.astype(np.uintp).nbytes),
               "d2h_bytes_per_step": int(entries_per_step * 8),
               "ms_per_step": e2e_s * 1e3,
               "path": "function_space(grid) + BoundaryAssembler.assemble x3 (C-ABI "
                       "boundary_assembler_assemble_into_memory, host numpy output)"}

    # roofline of the dominant kernel (regular tile-scatter kernel, FP64 CUDA cores)
    peak = ctypes_peak(_lib)
    from bempp._lib import ffi as _ffi  # noqa: F401

    nsing = singular_pair_count(cells)
    nregular = len(cells) ** 2 - nsing
    achieved = {k: FLOPS_PER_PAIR[k] * nregular / (v * 1e-3) / 1e12 for k, v in regular_ms.items()}
    dl = "double_layer"
    roofline = {
        "bound": "fp64",
        "kernel": "regular_scatter_fp64 (Laplace double layer, P1 x P1)",
        "achieved": achieved[dl], "peak": peak, "unit": "TFLOP/s",
        "frac": achieved[dl] / peak if peak else None,
        "traffic": None,
        "peak_source": "measured FP64 FMA-chain probe (bempp_measure_fma_peak) on this GPU",
        "per_operator_tflops": achieved, "regular_ms": regular_ms,
        "flops_per_regular_pair": FLOPS_PER_PAIR, "regular_pairs": nregular,
    }

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "entries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded perturbed icosphere)",
            "config": {"workload": "laplace_dl_adl_hs_p1_ico5_f64", "triangles": len(cells),
                       "dofs": n, "operators": OPERATORS, "regular_points": Q_REGULAR,
                       "duffy_order": ORDER, "entries_per_step": entries_per_step,
                       "parallelism": f"replicas{world}", "l2": "flushed between steps "
                       "(256 MiB write); outputs (3 x 839 MB) exceed L2"},
            "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "clocks": clocks,
        }
        if not args.skip_cpu:
            line["cpu_baseline"] = cpu_baseline(points, cells, n, args)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def ctypes_peak(_lib_mod):
    from bempp._lib import ffi, lib

    out = ffi.new("double*")
    st = lib.bempp_measure_fma_peak(1, 4096, 5, out)
    return float(out[0]) if st == 0 else None


def singular_pair_count(cells):
    """Ordered cell pairs sharing at least one vertex (handled by the Duffy kernel)."""
    cells = np.asarray(cells)
    nv = int(cells.max()) + 1
    vc = [[] for _ in range(nv)]
    for c, tri in enumerate(cells):
        for v in tri:
            vc[v].append(c)
    count = 0
    for c, tri in enumerate(cells):
        nb = set()
        for v in tri:
            nb.update(vc[v])
        count += len(nb)
    return count


def cpu_baseline(points, cells, n, args):
    """CPU FP64 oracle on a bounded sample: the regular part for a subset of test cells
    (all trial cells) plus the full singular part, scaled to the whole workload."""
    from oracle import oracle

    threads = os.cpu_count() or 1
    nsub = args.cpu_sample_cells
    rng = np.random.default_rng(0)
    subset = np.sort(rng.choice(len(cells), size=nsub, replace=False))
    t_reg = t_sing = 0.0
    for op in OPERATORS:
        t = time.perf_counter()
        oracle.assemble(points, cells, "laplace", op, test_degree=1, test_continuous=True,
                        trial_degree=1, trial_continuous=True, q_regular=Q_REGULAR,
                        q_singular=ORDER, nthreads=threads, parts=1, test_subset=subset)
        t_reg += time.perf_counter() - t
        t = time.perf_counter()
        oracle.assemble(points, cells, "laplace", op, test_degree=1, test_continuous=True,
                        trial_degree=1, trial_continuous=True, q_regular=Q_REGULAR,
                        q_singular=ORDER, nthreads=threads, parts=2)
        t_sing += time.perf_counter() - t
    est = t_reg * len(cells) / nsub + t_sing
    return {"value": len(OPERATORS) * n * n / est, "unit": "entries/s", "cores": threads,
            "kind": "port",
            "sample": f"regular part of all 3 operators for {nsub} of {len(cells)} test cells "
                      f"(x all trial cells) scaled by {len(cells) / nsub:.1f}, plus the full "
                      "singular part; CPU FP64 restatement of the bempp-rs algorithm "
                      "(OpenMP over 128x128 blocks, -O3 -march=native)",
            "seconds_estimated_full_step": est}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    points, cells = workload_mesh()
    from oracle import oracle

    n = oracle.space_size(points, cells, 1, True)
    for _ in range(args.warmup):
        pass  # the oracle has no warm-up state; warm-up steps are not timed anyway
    vals = []
    base = None
    for _ in range(args.steps):
        base = cpu_baseline(points, cells, n, args)
        vals.append(base["value"])
    value = statistics.median(vals)
    line = {
        "metric": METRIC, "value": value, "unit": "entries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": len(OPERATORS) * n * n / value * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded perturbed icosphere)", "impl": "reference",
        "config": {"workload": "laplace_dl_adl_hs_p1_ico5_f64", "triangles": len(cells),
                   "dofs": n, "operators": OPERATORS, "regular_points": Q_REGULAR,
                   "duffy_order": ORDER, "entries_per_step": len(OPERATORS) * n * n,
                   "parallelism": "host cores"},
        "cpu_baseline": {**base, "value": value},
        "e2e": {"value": value, "unit": "entries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-sample-cells", type=int, default=48)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
