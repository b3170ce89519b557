"""Benchmark: dense boundary-operator assembly on B200.

Headline workload (default, ``--workload p1``): Laplace double-layer, adjoint
double-layer and hypersingular operators, continuous P1 trial and test spaces, f64, on
the unit icosphere refined 5 times (20,480 flat triangles, 10,242 vertices) with a seeded
radial perturbation U(-0.02, 0.02) (numpy default_rng(20480)); regular pairs use the
6-point symmetric rule, singular pairs order-4 Duffy rules.  One step assembles all three
10,242 x 10,242 matrices (314.7 M entries).  The metric is dense entries per second.

Other workloads: ``helmholtz_sl`` (Helmholtz single layer, k = 8, DP0, complex128, same
perturbed 20,480-triangle sphere, 419 M entries), ``helmholtz_p1`` (Helmholtz double
layer, adjoint double layer and hypersingular, k = 8, P1, complex128, same sphere) and
``laplace_sl`` (Laplace single layer, DP0, f64, 1,280-triangle icosphere).  The default run also measures the Helmholtz
single-layer FP64 and mixed-precision assemblies and reports their speed ratio and the
mixed result's relative Frobenius error against the FP64 result (``helmholtz_sl_fp64_vs_mixed``
key, with the Helmholtz DL / ADL / HS P1 operators), the adjoint gradient against one
forward assembly (``adjoint``) and the batched wavenumber sweep (``sweep``).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload p1|helmholtz_sl|helmholtz_p1|laplace_sl]
                  [--precision fp64|mixed]
                  [--level L] [--once]

value: device-resident assembly (geometry cached, output in HBM), max over ranks.
e2e:   the same step through the C-ABI host path a user calls (grid and spaces built
       from host arrays, assemble_into_memory into host numpy arrays).
--impl reference: the CPU FP64 oracle (a restatement of the bempp-rs algorithm, which
       cannot be compiled here: no Rust toolchain) timed on a bounded sample of the same
       workload on all host cores.
--once: assemble each operator once and exit (the command used under ncu).
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

Q_REGULAR = 6
ORDER = 4
SEED = 20480

# Algorithmic FLOPs per regular cell pair at Q = 6 (36 point pairs): kernel evaluation
# plus basis accumulation, transcendental functions counted as 1, per-cell constants
# hoisted (P1 x P1 uses the factorised sum U_b(p) = sum_q K psi_b w_q).
FLOPS_PER_PAIR = {
    ("laplace", "single_layer", "dp0"): 396,
    ("laplace", "double_layer", "p1"): 990,
    ("laplace", "adjoint_double_layer", "p1"): 990,
    ("laplace", "hypersingular", "p1"): 459,
    ("helmholtz", "single_layer", "dp0"): 720,
}

# DRAM bytes (read + write) per launch of the dominant regular kernel, from one ncu capture
# of the full-size workload (profiles/dram_traffic_laplace_p1_ico5_fp64.md).
DRAM_TRAFFIC_PER_LAUNCH = {
    ("laplace", "double_layer", "p1", 20480): 1013.84e6 + 1021.62e6,
    ("laplace", "adjoint_double_layer", "p1", 20480): 1013.84e6 + 1018.73e6,
    ("laplace", "hypersingular", "p1", 20480): 1010.52e6 + 1001.86e6,
}

WORKLOADS = {
    "p1": dict(name="laplace_dl_adl_hs_p1_ico5_f64", kernel="laplace", space="p1", level=5,
               perturb=True, k=0.0,
               ops=["double_layer", "adjoint_double_layer", "hypersingular"],
               metric="dense entries/s (Laplace DL+ADL+HS, P1, f64, 20480-triangle icosphere)"),
    "helmholtz_sl": dict(name="helmholtz_sl_dp0_ico5_k8_c128", kernel="helmholtz", space="dp0",
                         level=5, perturb=True, k=8.0, ops=["single_layer"],
                         metric="dense entries/s (Helmholtz SL k=8, DP0, c128, 20480-triangle "
                                "icosphere)"),
    "helmholtz_p1": dict(name="helmholtz_dl_adl_hs_p1_ico5_k8_c128", kernel="helmholtz",
                         space="p1", level=5, perturb=True, k=8.0,
                         ops=["double_layer", "adjoint_double_layer", "hypersingular"],
                         metric="dense entries/s (Helmholtz DL+ADL+HS k=8, P1, c128, "
                                "20480-triangle icosphere)"),
    "laplace_sl": dict(name="laplace_sl_dp0_ico3_f64", kernel="laplace", space="dp0", level=3,
                       perturb=False, k=0.0, ops=["single_layer"],
                       metric="dense entries/s (Laplace SL, DP0, f64, 1280-triangle icosphere)"),
}


def workload_mesh(w, level=None):
    from bempp import shapes

    pts, cells = shapes.icosphere(w["level"] if level is None else level)
    if w["perturb"]:
        pts = shapes.radial_perturbation(pts, SEED)
    return pts, cells


def max_over_ranks(x: float, world: int) -> float:
    """The maximum of x over all ranks (device time of a multi-rank run is the slowest
    rank's); a no-op for one rank.  Works on NCCL (CUDA tensor) and gloo (CPU tensor)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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


def build_space(points, cells, space):
    from bempp.function_space import function_space
    from ndelement.ciarlet import Continuity, Family, create_family
    from ndgrid.grid import Grid

    grid = Grid(points, cells)
    if space == "p1":
        fam = create_family(Family.Lagrange, 1, Continuity.Standard)
    else:
        fam = create_family(Family.Lagrange, 0, Continuity.Discontinuous)
    return grid, function_space(grid, fam)


def make_assemblers(w, precision="fp64"):
    from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType, Precision,
                                         create_helmholtz_assembler, create_laplace_assembler)
    from ndelement.reference_cell import ReferenceCellType

    ops = {"single_layer": OperatorType.SingleLayer, "double_layer": OperatorType.DoubleLayer,
           "adjoint_double_layer": OperatorType.AdjointDoubleLayer,
           "hypersingular": OperatorType.Hypersingular}
    out = []
    for name in w["ops"]:
        o = BoundaryAssemblerOptions()
        o.set_regular_quadrature_degree(ReferenceCellType.Triangle, Q_REGULAR)
        o.set_singular_quadrature_degree(ReferenceCellType.Triangle, ReferenceCellType.Triangle,
                                         ORDER)
        o.set_precision(Precision.Mixed if precision == "mixed" else Precision.FP64)
        if w["kernel"] == "laplace":
            out.append((name, create_laplace_assembler(ops[name], o)))
        else:
            out.append((name, create_helmholtz_assembler(ops[name], w["k"], o)))
    return out


def singular_pair_count(cells):
    """Ordered cell pairs sharing at least one vertex (handled by the Duffy kernel)."""
    cells = np.asarray(cells)
    nv = int(cells.max()) + 1
    vc = [[] for _ in range(nv)]
    for c, tri in enumerate(cells):
        for v in tri:
            vc[v].append(c)
    count = 0
    for tri in cells:
        nb = set()
        for v in tri:
            nb.update(vc[v])
        count += len(nb)
    return count


def fma_peak(fp64=True):
    from bempp._lib import ffi, lib

    out = ffi.new("double*")
    st = lib.bempp_measure_fma_peak(1 if fp64 else 0, 4096, 5, out)
    return float(out[0]) if st == 0 else None


# operators assembled on one space object compute only the lower-triangle tile pairs and
# mirror them: half of the regular pairs are integrated (the diagonal tiles' own mirror
# pairs, 0.16 % at 20,480 cells, are ignored)
SYMMETRIC_OPS = ("single_layer", "hypersingular")


def integrated_pairs(name, nreg):
    return nreg / 2 if name in SYMMETRIC_OPS else nreg


class Workload:
    """Assemblers, device outputs and the step function of one workload on one GPU."""

    def __init__(self, w, precision, level=None):
        import torch

        self.w = w
        self.points, self.cells = workload_mesh(w, level)
        self.grid, self.space = build_space(self.points, self.cells, w["space"])
        self.n = self.space.global_size
        self.assemblers = make_assemblers(w, precision)
        dt = torch.complex128 if w["kernel"] == "helmholtz" else torch.float64
        self.outs = [torch.empty((self.n, self.n), dtype=dt, device="cuda")
                     for _ in self.assemblers]
        self.flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        self.stream = torch.cuda.current_stream().cuda_stream
        self.entries_per_step = len(self.assemblers) * self.n * self.n

    def step(self, flush=True):
        launches = 0
        for (_, a), out in zip(self.assemblers, self.outs):
            a.assemble_into_device(self.space, self.space, out, self.stream)
            launches += a.launch_count()
        if flush:
            self.flush.fill_(1.0)  # L2 flush between steps (256 MiB > 126 MB L2)
        return launches

    def phase_ms(self):
        import torch

        for _, a in self.assemblers:
            a.set_timing(True)
        self.step(flush=False)
        torch.cuda.synchronize()
        out = {}
        for name, a in self.assemblers:
            out[name] = a.phase_times()  # geometry, clear, regular, singular
            a.set_timing(False)
        return out

    def timed(self, steps, warmup, barrier=lambda: None):
        import torch

        for _ in range(warmup):
            self.step()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        launches = 0
        for _ in range(steps):
            launches += self.step()
        t1.record()
        torch.cuda.synchronize()
        barrier()
        return t0.elapsed_time(t1) / steps, launches


def helmholtz_sl_fp64_vs_mixed(args):
    """Helmholtz SL (k=8, DP0, 20,480 triangles): FP64 vs mixed assembly time and error."""
    import torch

    w = WORKLOADS["helmholtz_sl"]
    res = {}
    outs = {}
    sample = None
    for prec in ("fp64", "mixed"):
        wl = Workload(w, prec)
        if sample is None and not args.skip_cpu:  # CPU baseline leg: oracle rows (checker)
            sample = oracle_row_sample("helmholtz", w["ops"], w["k"], w["space"], wl.points,
                                       wl.cells, args.cpu_sample_cells, 160, 1)
            res["cpu_baseline"] = cpu_baseline(w, wl.points, wl.cells, wl.n, args, sample)
        ms, _ = wl.timed(max(3, args.steps), 2)
        ph = wl.phase_ms()["single_layer"]
        res[prec] = {"ms_per_assembly": ms, "entries_per_s": wl.entries_per_step / (ms * 1e-3),
                     "regular_ms": ph[2] if len(ph) > 2 else None, "phase_ms": ph}
        # algorithmic FLOPs of the integrated regular pairs over the phase time (mixed: the
        # FP32 far pairs, with the FP64 near and singular kernels of that phase in the time)
        nreg = len(wl.cells) ** 2 - singular_pair_count(wl.cells)
        fl = FLOPS_PER_PAIR[("helmholtz", "single_layer", "dp0")] * integrated_pairs("single_layer", nreg)
        peak = fma_peak(fp64=prec == "fp64")
        ach = fl / (res[prec]["regular_ms"] * 1e-3) / 1e12 if res[prec]["regular_ms"] else None
        res[prec]["roofline"] = {"bound": "fp64" if prec == "fp64" else "fp32", "achieved": ach,
                                 "peak": peak, "unit": "TFLOP/s",
                                 "frac": ach / peak if (ach and peak) else None,
                                 "peak_source": "bempp_measure_fma_peak (FMA chains on this GPU)"}
        outs[prec] = wl.outs[0]
        if sample is not None:
            res[prec]["rel_frobenius_error_vs_oracle_rows"] = rows_error(wl.outs[0], sample,
                                                                         "single_layer")
        del wl
        torch.cuda.empty_cache()
    err = (torch.linalg.norm(outs["mixed"] - outs["fp64"]) / torch.linalg.norm(outs["fp64"])).item()
    res["speedup_mixed_vs_fp64"] = res["fp64"]["ms_per_assembly"] / res["mixed"]["ms_per_assembly"]
    res["mixed_rel_frobenius_error_vs_fp64"] = err
    res["workload"] = w["name"]
    # the output is written once: 16 B per entry
    res["mixed_hbm_write_gbs"] = (16 * w_entries(w) / (res["mixed"]["regular_ms"] * 1e-3) / 1e9
                                  if res["mixed"]["regular_ms"] else None)
    del outs
    torch.cuda.empty_cache()
    res["helmholtz_p1_operators"] = helmholtz_p1_ops(args)
    return res


def w_entries(w):
    pts, cells = workload_mesh(w)
    return len(cells) ** 2


def helmholtz_p1_ops(args):
    """Helmholtz DL, ADL and HS (k = 8, P1 x P1, c128) on the 20,480-triangle perturbed
    sphere: FP64 vs mixed assembly time and the mixed result's error against FP64."""
    import torch

    w = dict(WORKLOADS["helmholtz_sl"])
    w.update(space="p1", ops=["double_layer", "adjoint_double_layer", "hypersingular"])
    out = {}
    wls = {prec: Workload(w, prec) for prec in ("fp64", "mixed")}
    sample = None
    if not args.skip_cpu:  # CPU baseline leg: oracle rows of each operator (checker)
        wl0 = wls["fp64"]
        sample = oracle_row_sample("helmholtz", w["ops"], w["k"], w["space"], wl0.points,
                                   wl0.cells, 256, 27, 2)
        out["cpu_baseline"] = cpu_baseline(w, wl0.points, wl0.cells, wl0.n, args, sample)
    for prec, wl in wls.items():
        wl.timed(1, 2)
        out[prec] = {name: ph[2] for name, ph in wl.phase_ms().items()}  # regular ms
        step_ms, _ = wl.timed(max(2, args.steps // 2), 1)
        out[prec]["ms_per_step"] = step_ms
    out["rel_frobenius_error_vs_fp64"] = {
        name: (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()
        for name, a, b in zip(w["ops"], wls["mixed"].outs, wls["fp64"].outs)}
    if sample is not None:
        out["rel_frobenius_error_vs_oracle_rows"] = {
            prec: {name: rows_error(o, sample, name) for name, o in zip(w["ops"], wl.outs)}
            for prec, wl in wls.items()}
    out["speedup_mixed_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["workload"] = "helmholtz_dl_adl_hs_p1_ico5_k8_c128"
    del wls
    torch.cuda.empty_cache()
    return out


def adjoint_timing(args):
    """Adjoint gradient of Re(lambda^H A mu) (Helmholtz SL, DP0, k = 5, perturbed
    5,120-triangle icosphere) against one FP64 forward assembly, device times."""
    import torch

    from bempp import shapes
    from bempp._lib import check, ffi, lib
    from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType,
                                         create_helmholtz_assembler)
    from bempp.function_space import grid_handle
    from ndelement.reference_cell import ReferenceCellType

    k = 5.0
    pts, cells = shapes.icosphere(4)
    pts = shapes.radial_perturbation(pts, 5120)
    rng = np.random.default_rng(5)
    n = len(cells)
    lam = torch.as_tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n), device="cuda")
    mu = torch.as_tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n), device="cuda")
    grid, space = build_space(pts, cells, "dp0")
    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, Q_REGULAR)
    a = create_helmholtz_assembler(OperatorType.SingleLayer, k, opts)
    out = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    gopts = BoundaryAssemblerOptions()
    gopts.set_regular_quadrature_degree(ReferenceCellType.Triangle, Q_REGULAR)
    g = grid_handle(grid).ptr  # the grid handle shared by the space
    tot = torch.zeros(2, dtype=torch.float64, device="cuda")
    grad = torch.zeros((len(pts), 3), dtype=torch.float64, device="cuda")

    def forward():
        a.assemble_into_device(space, space, out, stream)
        return torch.real(torch.vdot(lam, out.T @ mu))

    def gradient():
        check(lib.bempp_helmholtz_single_layer_dp0_gradient_device(
            g, gopts._rs_options, k, ffi.cast("void*", lam.data_ptr()),
            ffi.cast("void*", mu.data_ptr()), ffi.cast("double*", tot.data_ptr()),
            ffi.cast("double*", grad.data_ptr()), ffi.cast("void*", stream)), "gradient")

    def timed(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(reps):
            fn()
        t1.record()
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / reps

    gopts_m = BoundaryAssemblerOptions()
    gopts_m.set_regular_quadrature_degree(ReferenceCellType.Triangle, Q_REGULAR)
    from bempp.assembly.boundary import Precision

    gopts_m.set_precision(Precision.Mixed)
    grad_m = torch.zeros_like(grad)
    tot_m = torch.zeros_like(tot)

    def gradient_mixed():
        check(lib.bempp_helmholtz_single_layer_dp0_gradient_device(
            g, gopts_m._rs_options, k, ffi.cast("void*", lam.data_ptr()),
            ffi.cast("void*", mu.data_ptr()), ffi.cast("double*", tot_m.data_ptr()),
            ffi.cast("double*", grad_m.data_ptr()), ffi.cast("void*", stream)), "gradient")

    f_ms = timed(forward, 5)
    g_ms = timed(gradient, 5)
    gm_ms = timed(gradient_mixed, 5)
    mixed_err = ((grad_m - grad).abs().max() / grad.abs().max()).item()
    jf = forward().item()
    gradient()
    torch.cuda.synchronize()
    return {"workload": "helmholtz_sl_dp0_ico4_k5_gradient", "forward_ms": f_ms,
            "gradient_ms": g_ms, "gradient_over_forward": g_ms / f_ms,
            "gradient_mixed_ms": gm_ms, "gradient_mixed_over_forward": gm_ms / f_ms,
            "gradient_mixed_max_rel_err_vs_fp64": mixed_err,
            "J_forward": jf, "J_adjoint": tot[0].item(),
            "note": "forward = dense FP64 assembly into HBM + Re(lambda^H A mu); gradient = "
                    "one adjoint pass (all 7686 coordinates and k)"}


def sweep_timing(args):
    """Batched Helmholtz SL DP0 sweep, 32 wavenumbers in [1, 20], three stretched
    icospheres (1,280 / 5,120 / 20,480 triangles, axes U(0.8, 1.2) with seeds 1280 / 5120 /
    20480); complex64 outputs (114 GB) resident in HBM; one graph launch per sweep."""
    import torch

    from bempp import shapes
    from bempp.sweep import helmholtz_single_layer_sweep, last_tuning
    from ndgrid.grid import Grid

    ks = np.linspace(1.0, 20.0, 32)
    grids = []
    for level, seed in ((3, 1280), (4, 5120), (5, 20480)):
        pts, cells = shapes.icosphere(level)
        grids.append(Grid(shapes.ellipsoidal_stretch(pts, seed), cells))
    need = sum(len(ks) * len(g.cells) ** 2 * 8 for g in grids)
    free, _ = torch.cuda.mem_get_info()
    if free < need + (8 << 30):
        return {"skipped": f"needs {need / 1e9:.1f} GB of free device memory, {free / 1e9:.1f} GB free"}
    outs = [torch.empty((len(ks), len(g.cells), len(g.cells)), dtype=torch.complex64,
                        device="cuda") for g in grids]
    t = time.perf_counter()
    helmholtz_single_layer_sweep(grids, ks, outs)  # autotune + capture + first launch
    torch.cuda.synchronize()
    first_s = time.perf_counter() - t
    reps = 2
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        helmholtz_single_layer_sweep(grids, ks, outs)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    entries = sum(len(ks) * len(g.cells) ** 2 for g in grids)
    kc, bps, probe, shape = last_tuning()
    check = None
    if not args.skip_cpu:
        # CPU baseline leg as the checker: oracle rows (16 seeded rows per mesh) at the
        # smallest, a middle and the largest wavenumber of every mesh
        errs = {}
        for g, out in zip(grids, outs):
            pts = g.points
            cells = g.cells.astype(np.int64)
            for j in (0, len(ks) // 2, len(ks) - 1):
                smp = oracle_row_sample("helmholtz", ["single_layer"], float(ks[j]), "dp0", pts,
                                        cells, 128, 16, j)
                errs[f"{len(cells)}_k{ks[j]:.3f}"] = rows_error(out[j], smp, "single_layer")
        check = {"rel_frobenius_error_vs_oracle_rows": errs, "max": max(errs.values()),
                 "rows_per_matrix": 16}
    del outs
    torch.cuda.empty_cache()
    return {"workload": "helmholtz_sl_dp0_sweep_32k_ico3_4_5_c64", "entries": entries,
            "ms_per_sweep": ms, "entries_per_s": entries / (ms * 1e-3),
            "first_call_s": first_s, "tuning": {"k_per_item": kc, "ctas_per_sm": bps,
                                                "tile_shape": f"{shape}x{shape} tiles of 32 cells",
                                                "probe_ms_per_tile_pair_and_k": probe},
            "launches_per_sweep": 1, "parity": check}


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    w = dict(WORKLOADS[args.workload])
    if args.k is not None:
        w["k"] = args.k
    wl = Workload(w, args.precision, args.level)
    if args.once:
        wl.step(flush=False)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"once": w["name"], "precision": args.precision,
                              "cells": len(wl.cells), "n": wl.n}))
        return

    for _ in range(args.warmup):
        wl.step()
    phases = wl.phase_ms()  # live CUDA-event timing of each phase on the launching stream

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ms_per_step, launches = wl.timed(args.steps, 1, barrier)
    clocks = sampler.stop()
    ms_per_step = max_over_ranks(ms_per_step, world)
    value = world * wl.entries_per_step / (ms_per_step * 1e-3)

    # CPU baseline leg: oracle rows of a seeded DOF sample (timed), also the checker of the
    # GPU's rows of the same DOFs
    sample = parity = None
    if rank == 0 and not args.skip_cpu:
        sample = oracle_row_sample(w["kernel"], w["ops"], w["k"], w["space"], wl.points,
                                   wl.cells, args.cpu_sample_cells, 160, 0)
        parity = {"rel_frobenius_error_vs_oracle_rows": {
                      op: rows_error(out, sample, op) for op, out in zip(w["ops"], wl.outs)},
                  "rows": len(sample["rows"]),
                  "note": "complete rows of seeded test DOFs, GPU output of the timed run "
                          "against the CPU FP64 oracle"}

    mixed_same = None
    if rank == 0 and not args.skip_comparisons and args.precision == "fp64":
        # the same workload with FP32 far pairs: speed and error against the FP64 result
        ref = [o.clone() for o in wl.outs]
        wm = Workload(w, "mixed", args.level)
        ms_mixed, _ = wm.timed(max(2, args.steps // 2), 2)
        errs = [(torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()
                for a, b in zip(wm.outs, ref)]
        mixed_same = {"ms_per_step": ms_mixed, "entries_per_s": wm.entries_per_step / (ms_mixed * 1e-3),
                      "speedup_vs_fp64": ms_per_step / ms_mixed,
                      "rel_frobenius_error_vs_fp64": dict(zip(w["ops"], errs))}
        if sample is not None:
            mixed_same["rel_frobenius_error_vs_oracle_rows"] = {
                op: rows_error(out, sample, op) for op, out in zip(w["ops"], wm.outs)}
        del wm, ref
        torch.cuda.empty_cache()

    e2e = None
    if not args.skip_e2e:
        pts_h = np.ascontiguousarray(wl.points)
        cells_h = np.ascontiguousarray(wl.cells)
        e2e_steps = max(1, min(args.steps, 3))
        # one untimed step: first-use costs (page-locked output blocks, copy threads)
        _, s2 = build_space(pts_h, cells_h, w["space"])
        for _, a in wl.assemblers:
            a.assemble(s2, s2)
        del s2
        torch.cuda.synchronize()
        barrier()
        t = time.perf_counter()
        t_build = 0.0
        t_ops = [0.0] * len(wl.assemblers)
        copy_stats = [None] * len(wl.assemblers)
        t_free = 0.0
        steps_ms = []
        for _ in range(e2e_steps):
            t0 = t1 = time.perf_counter()
            _, s2 = build_space(pts_h, cells_h, w["space"])
            t_build += time.perf_counter() - t1
            for i, (_, a) in enumerate(wl.assemblers):
                t1 = time.perf_counter()
                a.assemble(s2, s2)
                t_ops[i] += time.perf_counter() - t1
                copy_stats[i] = a.host_copy_stats()
            t1 = time.perf_counter()
            del s2
            t_free += time.perf_counter() - t1
            steps_ms.append(1e3 * (time.perf_counter() - t0))
        e2e_s = (time.perf_counter() - t) / e2e_steps
        e2e_s = max_over_ranks(e2e_s, world)
        esize = 16 if w["kernel"] == "helmholtz" else 8
        e2e = {"value": world * wl.entries_per_step / e2e_s, "unit": "entries/s",
               "h2d_bytes_per_step": int(pts_h.nbytes + cells_h.astype(np.uintp).nbytes),
               "d2h_bytes_per_step": int(wl.entries_per_step * esize),
               "ms_per_step": e2e_s * 1e3,
               "breakdown_ms": {"steps": steps_ms, "grid_and_space": 1e3 * t_build / e2e_steps,
                                "free_grid_and_space": 1e3 * t_free / e2e_steps,
                                "assemble": {n: 1e3 * t / e2e_steps
                                             for (n, _), t in zip(wl.assemblers, t_ops)},
                                "host_copy_last": {n: c for (n, _), c in zip(wl.assemblers,
                                                                             copy_stats)}},
               "path": "function_space(grid) + BoundaryAssembler.assemble per operator (C-ABI "
                       "boundary_assembler_assemble_into_memory_ex, host numpy output)"}

    peak = fma_peak()
    nreg = len(wl.cells) ** 2 - singular_pair_count(wl.cells)
    per_op = {}
    for name, ph in phases.items():
        key = (w["kernel"], name, w["space"])
        reg_ms = ph[2] if len(ph) > 2 else float("nan")
        fl = FLOPS_PER_PAIR.get(key)
        per_op[name] = {"regular_ms": reg_ms, "phase_ms": ph,
                        "pairs_integrated": integrated_pairs(name, nreg),
                        "tflops": fl * integrated_pairs(name, nreg) / (reg_ms * 1e-3) / 1e12
                        if fl else None}
    dom = max(per_op, key=lambda n: per_op[n]["regular_ms"])
    ach = per_op[dom]["tflops"]
    roofline = {
        "bound": "fp64", "kernel": f"regular kernel, {w['kernel']} {dom} ({w['space']})",
        "achieved": ach, "peak": peak, "unit": "TFLOP/s",
        "frac": (ach / peak) if (ach and peak) else None,
        "traffic": DRAM_TRAFFIC_PER_LAUNCH.get((w["kernel"], dom, w["space"], len(wl.cells))),
        "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
        "peak_source": "measured FP64 FMA-chain probe (bempp_measure_fma_peak) on this GPU; "
                       "MEASURED_PEAKS.json has no FP64 CUDA-core figure",
        "regular_pairs": nreg, "per_operator": per_op,
    }

    ns = adj = swp = None
    if rank == 0 and args.workload == "p1" and not args.skip_comparisons:
        del wl.outs
        torch.cuda.empty_cache()
        ns = helmholtz_sl_fp64_vs_mixed(args)
        adj = adjoint_timing(args)
        torch.cuda.empty_cache()
        swp = None if args.skip_sweep else sweep_timing(args)

    if rank == 0:
        line = {
            "metric": w["metric"], "value": value, "unit": "entries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128" if w["kernel"] == "helmholtz" else "f64",
            "data": "synthetic (seeded icosphere)",
            "config": {"workload": w["name"], "triangles": len(wl.cells), "dofs": wl.n,
                       "operators": w["ops"], "precision": args.precision,
                       "regular_points": Q_REGULAR, "duffy_order": ORDER,
                       "entries_per_step": wl.entries_per_step,
                       "parallelism": f"replicas{world}",
                       "l2": "flushed between steps (256 MiB write); outputs exceed L2"},
            "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "clocks": clocks,
        }
        if parity is not None:
            line["parity"] = parity
        if mixed_same is not None:
            line["mixed_same_workload"] = mixed_same
        if ns is not None:
            line["helmholtz_sl_fp64_vs_mixed"] = ns
        if adj is not None:
            line["adjoint"] = adj
        if swp is not None:
            line["sweep"] = swp
        if sample is not None:
            line["cpu_baseline"] = cpu_baseline(w, wl.points, wl.cells, wl.n, args, sample)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ----------------------------------------------------------------- CPU baseline leg ---
# The only part of this file that runs the oracle (oracle/, the CPU FP64 restatement of the
# bempp-rs algorithm: OpenMP over 128 x 128 cell blocks, -O3 -march=native): it times the
# CPU on samples of the workloads and on one complete step (--impl reference), and the
# complete rows it computes are the checker of the GPU's rows (*_vs_oracle keys).

def _space_degree(space):
    return (1, True) if space == "p1" else (0, False)


def oracle_row_sample(kernel, ops, k, space, points, cells, window, nrows, seed):
    """Complete rows of at most ``nrows`` seeded test DOFs of each operator, from the
    oracle on all host threads: {"rows", "oracle_rows": {op: rows x n}, "seconds": {op: s},
    "regular_seconds", "singular_seconds", "test_cells", "threads"}.  The test cells are a
    seeded run of ``window`` consecutive cells starting at a multiple of the oracle's
    128-cell block (so its blocks are full); the rows are DOFs all of whose cells lie in
    that run (so its regular part completes them), and the singular part of the whole grid
    is added.  The regular time scales with the number of test cells; the singular time is
    that of the whole step."""
    from oracle import oracle

    deg, cont = _space_degree(space)
    threads = os.cpu_count() or 1
    dofs, n = oracle.cell_dofs(points, cells, deg, cont)
    ncells = len(cells)
    rng = np.random.default_rng(seed)
    window = min(window, ncells)
    c0 = int(rng.integers(0, max(1, (ncells - window) // 128 + 1))) * 128
    sub = np.arange(c0, min(ncells, c0 + window))
    inside = np.zeros(ncells, dtype=bool)
    inside[sub] = True
    # DOFs touched only by cells of the run
    touched_outside = np.zeros(n, dtype=bool)
    touched_outside[np.unique(dofs[~inside])] = True
    eligible = np.setdiff1d(np.unique(dofs[sub]), np.flatnonzero(touched_outside))
    rows = np.sort(rng.choice(eligible, size=min(nrows, len(eligible)), replace=False))
    out = {"rows": rows, "oracle_rows": {}, "seconds": {}, "regular_seconds": {},
           "singular_seconds": {}, "test_cells": int(len(sub)), "threads": threads, "n": n}
    kw = dict(k=k, test_degree=deg, test_continuous=cont, trial_degree=deg,
              trial_continuous=cont, q_regular=Q_REGULAR, q_singular=ORDER, nthreads=threads)
    for op in ops:
        t = time.perf_counter()
        reg = oracle.assemble(points, cells, kernel, op, parts=1, test_subset=sub, **kw)[rows]
        t1 = time.perf_counter()
        sing = oracle.assemble(points, cells, kernel, op, parts=2, **kw)[rows]
        t2 = time.perf_counter()
        out["regular_seconds"][op] = t1 - t
        out["singular_seconds"][op] = t2 - t1
        out["seconds"][op] = t2 - t
        out["oracle_rows"][op] = reg + sing
    return out


def rows_error(out_tensor, sample, op):
    """Relative Frobenius error of the GPU's rows (column-major device matrix held as a
    (n_trial, n_test) tensor) against the oracle's rows of the same DOFs."""
    import torch

    idx = torch.as_tensor(sample["rows"], device=out_tensor.device)
    got = out_tensor[:, idx].T.to(torch.complex128 if out_tensor.is_complex() else torch.float64)
    ref = sample["oracle_rows"][op]
    got = got.cpu().numpy()
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))


def cpu_rate(sample, ncells, nops, n):
    """CPU entries/s of the whole workload estimated from a row sample: the regular time
    scaled by (all cells / sampled test cells) plus the singular time of the whole grid."""
    est = (sum(sample["regular_seconds"].values()) * ncells / sample["test_cells"] +
           sum(sample["singular_seconds"].values()))
    return nops * n * n / est


def cpu_baseline(w, points, cells, n, args, sample=None):
    """CPU baseline of the headline workload on a bounded sample (about 10-30 s of CPU
    work): complete rows of a seeded DOF subset of every operator, scaled."""
    if sample is None:
        sample = oracle_row_sample(w["kernel"], w["ops"], w["k"], w["space"], points, cells,
                                   args.cpu_sample_cells, 160, 0)
    return {"value": cpu_rate(sample, len(cells), len(w["ops"]), n), "unit": "entries/s",
            "cores": sample["threads"], "kind": "port",
            "sample": f"regular part of {len(w['ops'])} operator(s) for a seeded run of "
                      f"{sample['test_cells']} of {len(cells)} consecutive test cells (x all "
                      f"trial cells), time scaled by {len(cells) / sample['test_cells']:.1f}, "
                      "plus the whole singular part; CPU FP64 restatement of the bempp-rs "
                      "algorithm (OpenMP over 128x128 blocks, -O3 -march=native)",
            "sample_seconds": sum(sample["seconds"].values())}


def run_reference(args):
    """The reference arm: the CPU FP64 restatement of the bempp-rs algorithm (the reference
    itself needs a Rust toolchain, absent here) on all host cores.  It times ONE complete
    step of the workload (every operator, every row: the value), then --steps sampled steps
    as a cross-check of the sample-based estimate; warm-up steps are sampled steps."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle

    w = WORKLOADS[args.workload]
    points, cells = workload_mesh(w, args.level)
    deg, cont = _space_degree(w["space"])
    threads = os.cpu_count() or 1
    n = oracle.space_size(points, cells, deg, cont)
    for i in range(args.warmup):  # untimed: small samples (library load, page-in, caches)
        oracle_row_sample(w["kernel"], w["ops"], w["k"], w["space"], points, cells, 128, 8, i)
    t = time.perf_counter()
    for op in w["ops"]:
        oracle.assemble(points, cells, w["kernel"], op, k=w["k"], test_degree=deg,
                        test_continuous=cont, trial_degree=deg, trial_continuous=cont,
                        q_regular=Q_REGULAR, q_singular=ORDER, nthreads=threads)
    full_s = time.perf_counter() - t
    eps = len(w["ops"]) * n * n
    value = eps / full_s
    est = []
    for i in range(min(args.steps, 2)):
        smp = oracle_row_sample(w["kernel"], w["ops"], w["k"], w["space"], points, cells,
                                args.cpu_sample_cells, 8, 100 + i)
        est.append(cpu_rate(smp, len(cells), len(w["ops"]), n))
    est_med = statistics.median(est) if est else None
    sample_desc = (f"one complete step timed: all {len(w['ops'])} operator(s), {n} x {n} each, "
                   f"{full_s:.1f} s on {threads} threads; cross-check: {len(est)} sampled steps "
                   f"(regular part of {args.cpu_sample_cells} consecutive test cells scaled, plus the "
                   f"singular part) estimate "
                   f"{est_med:.4g} entries/s, {est_med / value:.3f} x the measured full step"
                   if est_med else f"one complete step timed ({full_s:.1f} s)")
    line = {
        "metric": w["metric"], "value": value, "unit": "entries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": full_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128" if w["kernel"] == "helmholtz" else "f64",
        "data": "synthetic (seeded icosphere)", "impl": "reference",
        "config": {"workload": w["name"], "triangles": len(cells), "dofs": n,
                   "operators": w["ops"], "regular_points": Q_REGULAR, "duffy_order": ORDER,
                   "entries_per_step": eps, "parallelism": "host cores"},
        "full_steps_timed": 1,
        "sampled_estimate": {"median": est_med, "values": est,
                             "ratio_to_full_step": (est_med / value) if est_med else None},
        "cpu_baseline": {"value": value, "unit": "entries/s", "cores": threads, "kind": "port",
                         "sample": sample_desc},
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
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="p1")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--level", type=int, default=None, help="icosphere refinement override")
    ap.add_argument("--k", type=float, default=None, help="wavenumber override (Helmholtz)")
    ap.add_argument("--once", action="store_true")
    ap.add_argument("--cpu-sample-cells", type=int, default=640,
                    help="consecutive test cells of the CPU baseline samples")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-comparisons", action="store_true",
                    help="skip the mixed-precision, Helmholtz, adjoint and sweep measurements")
    ap.add_argument("--skip-sweep", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
