"""Benchmark driver: python bench.py --gpus N --steps K --warmup W [--impl ours|reference]

Prints ONE JSON line on rank 0. Workloads (--workload) are the hot-path
configurations with synthetic seeded inputs:

  clover   (default) 2D compressible ideal-gas Lagrangian-remap hydro
           (CloverLeaf) on 3840x3840 cells, FP64, gamma 1.4; background
           rho=0.2, e=1.0 plus 4 seeded rectangles; a step is one hydro
           cycle with CFL dt and a field summary read back every step.
  clover3d the 3D CloverLeaf hydro on 256^3 cells, FP64; background rho=0.2,
           e=1.0 plus 3 seeded cuboids; a step is one hydro cycle.
  laplace  2D Laplace Jacobi, single block 4096x4096 FP64, 5-point stencil,
           seeded U[0,1) Dirichlet ring, interior 0; a step is one iteration
           (apply_stencil + max|delta| reduction read back + copy).
  adi      batched tridiagonal x/y/z sweeps (ops_tridMultiDimBatch), one
           256^3 block or 64 uneven blocks, FP64 or FP32; a step is the three
           sweeps.
  learned  the same heat solve with the learned multigrid preconditioner in
           flexible CG (trained on the GPU first), next to plain Jacobi-PCG.
  mg       the same heat solve with the native FP32 aggregation-multigrid
           V-cycle as the flexible-CG preconditioner, next to plain Jacobi-PCG.
  tea      implicit heat conduction (TeaLeaf CG, Jacobi preconditioner) on
           4096x4096 with 16 seeded density rectangles; a step is one implicit
           timestep solved to residual 1e-10, FP64 PCG beside FP32-inner /
           FP64-refinement PCG; the metric is time to solution.

`value` is device-timed (CUDA events on the runtime stream) with inputs
resident in HBM; `e2e` times the same work through the public C-ABI call
from host buffers (field upload, per-step result read-back, field download)
by wall clock. With N > 1 (torchrun) every rank runs its own replica of the
workload (weak scaling, no data-path collective) and rank 0 reports the
whole-job rate over the slowest rank's time.

--impl reference times the reference's own OpenMP build (oracle/_ref) on the
host cores for the same workload and metric (rank 0 only).
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# device the timing collectives use: the rank's GPU under NCCL, the host
# under gloo (the reference arm, and the CPU tests of this path)
_DIST_DEVICE = "cpu"


def dist_setup(args):
    global _DIST_DEVICE
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
            _DIST_DEVICE = f"cuda:{local}"
        else:
            _DIST_DEVICE = "cpu"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, value, local):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=_DIST_DEVICE)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, local):
    if pg is None:
        return
    import torch
    if _DIST_DEVICE.startswith("cuda"):
        torch.cuda.synchronize(local)
    pg.barrier()
    if _DIST_DEVICE.startswith("cuda"):
        torch.cuda.synchronize(local)


# ---------------------------------------------------------------------------
# Laplace
# ---------------------------------------------------------------------------
LAP_N = 4096


def cpu_reference_laplace(iters, threads):
    import oracle
    exe = oracle.reference_binary("laplace2d_seeded")
    if exe is None:
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    with tempfile.TemporaryDirectory() as td:
        r = subprocess.run([exe, str(LAP_N), str(LAP_N), str(iters), "1"], cwd=td, capture_output=True, text=True,
                           env=env, timeout=600, check=True)
    secs = [float(l.split()[1]) for l in r.stdout.splitlines() if l.startswith("wall_seconds")][0]
    return LAP_N * LAP_N * iters / secs, secs


def bench_laplace(args, world, rank, local, pg):
    import numpy as np

    from ops_b200 import apps, seeded
    from ops_b200 import ops as O

    peaks, peak_kind = load_peaks()
    O.ops_init(local, 0)
    field = seeded.laplace_field(LAP_N, LAP_N, 1)
    cells = LAP_N * LAP_N
    K, W = args.steps, args.warmup

    # value: W untimed + K timed iterations, inputs resident, CUDA events.
    barrier(pg, local)
    O.reset_counters()
    with ClockSampler(local) as cs:
        _, errs, secs = apps.laplace2d(field, K, warmup=W)
    clocks = cs.summary()
    c = O.counters()
    launches_timed = int(round(c["kernels"] * K / max(1, K + W)))
    barrier(pg, local)
    secs = max_over_ranks(pg, secs, local)

    # roofline: per-kernel CUDA-event durations of the dominant kernel.
    O.set_kernel_timing(1)
    O.clear_kernel_timing()
    apps.laplace2d(field, K, warmup=0)
    n, ms = O.kernel_time("laplace2d/apply_stencil")
    O.set_kernel_timing(0)
    avg_s = ms * 1e-3 / max(n, 1)
    alg_bytes = 16.0 * cells  # read A, write Anew per cell-update
    achieved = alg_bytes / avg_s / 1e9

    # e2e: the public C-ABI call from pinned host buffers (field in, final
    # field out; both allocated before timing), wall clock.
    import torch
    pinned = torch.from_numpy(field).pin_memory().numpy()
    pinned_out = torch.empty(field.shape, dtype=torch.float64).pin_memory().numpy()
    barrier(pg, local)
    t0 = time.perf_counter()
    out, _, _ = apps.laplace2d(pinned, K, warmup=0, out=pinned_out)
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(pg, t1 - t0, local)

    value = world * cells * K / secs
    line = {
        "metric": "cell-updates/s",
        "value": value,
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": secs * 1e3 / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded SplitMix64 boundary ring, interior 0)",
        "config": {"workload": "laplace2d_jacobi_4096x4096_fp64", "grid": [LAP_N, LAP_N], "halo": 1,
                   "step": "apply_stencil + max|delta| readback + copy (elided by renaming)",
                   "l2": "inputs larger than L2 (two 134 MB fields)", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": TRAFFIC_PER_CELL["laplace"] * cells,
                     "traffic_source": "ncu capture at 4096^2 (profiles/laplace2d_4096_apply_stencil_dram.md)",
                     "kernel": "laplace2d/apply_stencil", "alg_bytes_per_launch": alg_bytes,
                     "avg_launch_ms": avg_s * 1e3, "peak_source": f"{peak_kind} hbm_gbs"},
        "e2e": {"value": world * cells * K / e2e_s, "unit": "cell-updates/s",
                "h2d_bytes_per_step": field.nbytes / K, "d2h_bytes_per_step": 8 + out.nbytes / K,
                "note": "one C-ABI call: field upload, K iterations each reading max|delta| back, field download"},
        "gpu_launches": launches_timed,
        "clocks": clocks,
        "final_error": float(errs[-1]),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        base = cpu_reference_laplace(args.cpu_iters, threads)
        if base:
            line["cpu_baseline"] = {"value": base[0], "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                                    "sample": f"reference laplace2d OpenMP build, {LAP_N}^2, {args.cpu_iters} iterations,"
                                              f" {base[1]:.2f} s"}
    return line


def reference_laplace(args, world, rank):
    threads = os.cpu_count() or 1
    iters = max(1, min(args.steps, 200))
    base = cpu_reference_laplace(iters, threads)
    if base is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/bin/laplace2d_seeded was not built"}
    v, secs = base
    return {
        "impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": world,
        "steps": iters, "warmup": 0, "ms_per_step": secs * 1e3 / iters, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded SplitMix64 boundary ring, interior 0)",
        "config": {"workload": "laplace2d_jacobi_4096x4096_fp64", "grid": [LAP_N, LAP_N]},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                         "sample": f"{iters} iterations of the reference OpenMP build on {threads} host threads"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# CloverLeaf 2D hydro
# ---------------------------------------------------------------------------
CL_N = 3840
# DRAM bytes per cell of one launch of a workload's dominant kernel, from one
# ncu capture each (dram__bytes_read.sum + dram__bytes_write.sum; the
# captures are summarised in profiles/, which names the command):
#   CloverLeaf 2D PdV_kernel_nopredict at 2560^2: 89.3 + 21.0 B
#     (profiles/cloverleaf2d_2560_dram_per_kernel.md)
#   CloverLeaf 3D PdV_kernel_nopredict at 160^3: 141.4 + 22.6 B
#     (profiles/cloverleaf3d_160_pdv_accelerate.md)
#   Laplace apply_stencil at 4096^2: 227.4 MB per launch / 4096^2
#     (profiles/laplace2d_4096_apply_stencil_dram.md)
#   ADI 256^3 FP64 x / y / z sweeps: 650.1 / 1144.0 / 1283.4 MB per sweep / 256^3
#     (profiles/adi_cube_256_fp64_dram.md)
# Traffic grows with the cells (or unknowns) a launch processes, so a
# launch's traffic is the figure times its cells.
TRAFFIC_PER_CELL = {"clover": 110.3, "clover3d": 164.0, "laplace": 227.4e6 / 4096 ** 2,
                    "adi_cube_fp64": (650.1e6 / 256 ** 3, 1144.0e6 / 256 ** 3, 1283.4e6 / 256 ** 3)}


def clover_deck(steps, n=CL_N):
    from ops_b200 import apps, seeded
    return apps.clover_deck(x_cells=n, y_cells=n, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0, initial_timestep=0.04,
                            timestep_rise=1.5, max_timestep=0.04, end_step=steps, summary_frequency=1,
                            states=seeded.clover_config2_states(n, n, 2))


def cpu_reference_clover(steps, threads, n=CL_N):
    import oracle
    from ops_b200 import apps
    exe = oracle.reference_binary("cloverleaf")
    if exe is None:
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    with tempfile.TemporaryDirectory() as td:
        with open(os.path.join(td, "clover.in"), "w") as f:
            f.write(apps.clover_deck_text(clover_deck(steps, n)))
        r = subprocess.run([exe], cwd=td, capture_output=True, text=True, env=env, timeout=900, check=True)
    secs = [float(l.split()[-1]) for l in r.stdout.splitlines() if l.strip().startswith("Total Wall time")][-1]
    return n * n * steps / secs, secs


def print_kernel_table(stats, steps, cells, peak_gbs):
    """Per-kernel CUDA-event timing of `steps` cycles on stderr: launches,
    ms per step, share, algorithmic bytes per cell and achieved GB/s."""
    tot = sum(v[1] for v in stats.values())
    print(f"{'kernel':56s} {'launch/step':>11s} {'ms/step':>8s} {'share':>6s} {'B/cell':>7s} {'GB/s':>7s} {'frac':>5s}",
          file=sys.stderr)
    for k, (n, ms, by) in sorted(stats.items(), key=lambda kv: -kv[1][1]):
        gbs = by / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        print(f"{k:56s} {n / steps:11.2f} {ms / steps:8.4f} {ms / tot:6.1%} {by / steps / cells:7.1f} {gbs:7.0f}"
              f" {gbs / peak_gbs:5.2f}", file=sys.stderr)
    print(f"{'total':56s} {sum(v[0] for v in stats.values()) / steps:11.2f} {tot / steps:8.4f}", file=sys.stderr)


def bench_clover(args, world, rank, local, pg):
    from ops_b200 import apps
    from ops_b200 import ops as O

    peaks, peak_kind = load_peaks()
    O.ops_init(local, 0)
    N = args.grid or CL_N
    cells = N * N
    K, W = args.steps, args.warmup

    # Untimed: the fused chains' tile shapes are tuned on their first
    # executions (both sweep orders) and kept in the tuning cache file, which
    # the timed call reads.
    apps.cloverleaf(clover_deck(24, N))
    barrier(pg, local)
    O.reset_counters()
    with ClockSampler(local) as cs:
        summ, secs = apps.cloverleaf(clover_deck(W + K, N), warmup_steps=W)
    clocks = cs.summary()
    c = O.counters()
    fs = O.fusion_stats()
    barrier(pg, local)
    secs = max_over_ranks(pg, secs, local)

    # Roofline: per-kernel CUDA-event durations and compulsory bytes.
    kp = min(K, 10)
    O.set_kernel_timing(1)
    O.clear_kernel_timing()
    apps.cloverleaf(clover_deck(kp, N))
    stats = O.kernel_stats()
    O.set_kernel_timing(0)
    launches_per_step = sum(v[0] for v in stats.values()) / kp
    if args.kernel_table and rank == 0:
        print_kernel_table(stats, kp, cells, peaks["hbm_gbs"])
    dom, (n, ms, by) = max(stats.items(), key=lambda kv: kv[1][1])
    achieved = (by / n) / (ms / n * 1e-3) / 1e9
    tot_ms = sum(v[1] for v in stats.values())
    tot_by = sum(v[2] for v in stats.values())

    # e2e: the public C-ABI call from the host deck to host summaries, wall clock.
    barrier(pg, local)
    t0 = time.perf_counter()
    summ_e2e, _ = apps.cloverleaf(clover_deck(K, N))
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(pg, t1 - t0, local)

    line = {
        "metric": "cell-updates/s",
        "value": world * cells * K / secs,
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": secs * 1e3 / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (background rho=0.2 e=1.0 + 4 SplitMix64-seeded rectangles, seed 2)",
        "config": {"workload": f"cloverleaf2d_{N}x{N}_fp64", "grid": [N, N], "gamma": 1.4,
                   "cell_update": "one cell advanced one hydro timestep",
                   "step": "timestep (ideal_gas, viscosity, CFL dt) + PdV + accelerate + flux_calc + advection"
                           " + reset_field + field_summary (5 FP64 sums read back)",
                   "l2": "inputs larger than L2 (about 30 fields of 118 MB)", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": TRAFFIC_PER_CELL["clover"] * cells
                     if dom == "cloverleaf/PdV_kernel_nopredict" else None,
                     "traffic_source": "ncu capture of PdV_kernel_nopredict at 2560^2, per cell x cells"
                                       " (profiles/cloverleaf2d_2560_dram_per_kernel.md)", "kernel": dom,
                     "alg_bytes_per_launch": by / n, "avg_launch_ms": ms / n, "peak_source": f"{peak_kind} hbm_gbs",
                     "step_effective_gbs": tot_by / (tot_ms * 1e-3) / 1e9,
                     "step_alg_bytes_per_cell": tot_by / kp / cells},
        "e2e": {"value": world * cells * K / e2e_s, "unit": "cell-updates/s", "h2d_bytes_per_step": 0.0,
                "d2h_bytes_per_step": 6 * 8 + 3 * 8,
                "note": "one C-ABI call: deck in, device set-up (generate), K cycles each reading dt and the"
                        " 5-value field summary back; the state is generated on the device from the deck, as the"
                        " reference app generates it, so no field crosses the boundary; the dats' storage comes"
                        " from the runtime's pool of storage kept from the bench's earlier calls (warm pool)"},
        "gpu_launches": int(round(launches_per_step * K)),
        "clocks": clocks,
        "fusion": {"chains_per_step": fs["chains"] / (W + K), "loops_fused_per_step": fs["loops"] / (W + K),
                   "chain_alg_bytes_per_cell": fs["fused_bytes"] / (W + K) / cells,
                   "same_loops_unfused_bytes_per_cell": fs["loop_bytes"] / (W + K) / cells,
                   "note": "loop chains of the lazy queue run as one tiled kernel each; chain bytes = each dat's"
                           " points read once and written once per chain (the step's other loops run unfused)"},
        "final_summary": {"vol": summ[-1, 2], "mass": summ[-1, 3], "ie": summ[-1, 4], "ke": summ[-1, 5],
                          "press": summ[-1, 6]},
    }
    if rank == 0 and world == 1 and not args.no_learned:
        line["learned_vs_pcg"] = learned_vs_pcg(args, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        base = cpu_reference_clover(args.cpu_clover_steps, threads)
        if base:
            line["cpu_baseline"] = {"value": base[0], "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                                    "sample": f"reference CloverLeaf OpenMP build, {CL_N}^2, {args.cpu_clover_steps}"
                                              f" steps (hydro loop wall time {base[1]:.2f} s)"}
    return line


def learned_vs_pcg(args, local):
    """The second half of the headline metric in the default line: time to
    the 1e-10 residual of the 4096^2 heat solve with the learned
    preconditioners against plain FP64 PCG, on this GPU in this run (the
    networks are trained first, as `--workload learned` does). Failures are
    reported in the object; they do not affect the CloverLeaf figures."""
    import copy
    try:
        a = copy.copy(args)
        a.steps, a.warmup, a.grid, a.no_cpu_baseline = 1, 3, None, True
        t0 = time.perf_counter()
        d = bench_learned(a, 1, 0, local, None)
        return {"grid": [TEA_N, TEA_N], "eps": 1e-10, "plain_pcg_s": d["plain_pcg"]["seconds"],
                "learned_fcg_s": d["learned_fcg"]["seconds"],
                "learned_fcg_over_pcg": d["learned_fcg"]["time_ratio_vs_plain"],
                "learned_mg_fcg_s": d["learned_mg_fcg"]["seconds"],
                "learned_mg_fcg_over_pcg": d["learned_mg_fcg"]["time_ratio_vs_plain"],
                "multigrid_fcg_s": d["multigrid_fcg"]["seconds"],
                "note": "median of the timed solves after training both networks (bench.py --workload learned has"
                        " the full record); not part of the CloverLeaf timing",
                "wall_s": time.perf_counter() - t0}
    except Exception as e:  # the headline line must survive
        return {"error": f"{type(e).__name__}: {e}"}


def reference_clover(args, world, rank):
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, args.cpu_clover_steps))
    base = cpu_reference_clover(steps, threads)
    if base is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/bin/cloverleaf was not built"}
    v, secs = base
    return {
        "impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": world,
        "steps": steps, "warmup": 0, "ms_per_step": secs * 1e3 / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (background rho=0.2 e=1.0 + 4 SplitMix64-seeded rectangles, seed 2)",
        "config": {"workload": "cloverleaf2d_3840x3840_fp64", "grid": [CL_N, CL_N]},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                         "sample": f"{steps} steps of the reference OpenMP build at {CL_N}^2 on {threads} threads"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# CloverLeaf 3D
# ---------------------------------------------------------------------------
CL3_N = 256


def clover3d_deck(steps, n=CL3_N):
    from ops_b200 import apps, seeded
    return apps.clover3d_deck(x_cells=n, y_cells=n, z_cells=n, xmax=10.0, ymax=10.0, zmax=10.0,
                              initial_timestep=0.04, timestep_rise=1.5, max_timestep=0.04, end_step=steps,
                              summary_frequency=1, states=seeded.clover3d_states(n, n, n, 6))


def cpu_reference_clover3d(steps, threads, n=CL3_N):
    import oracle
    from ops_b200 import apps
    exe = oracle.reference_binary("cloverleaf3d")
    if exe is None:
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    with tempfile.TemporaryDirectory() as td:
        with open(os.path.join(td, "clover.in"), "w") as f:
            f.write(apps.clover3d_deck_text(clover3d_deck(steps, n)))
        r = subprocess.run([exe], cwd=td, capture_output=True, text=True, env=env, timeout=900, check=True)
    secs = [float(l.split()[-1]) for l in r.stdout.splitlines() if l.strip().startswith("Total Wall time")][-1]
    return n ** 3 * steps / secs, secs


def bench_clover3d(args, world, rank, local, pg):
    from ops_b200 import apps
    from ops_b200 import ops as O

    peaks, peak_kind = load_peaks()
    O.ops_init(local, 0)
    N = args.grid or CL3_N
    cells = N ** 3
    K, W = args.steps, args.warmup

    barrier(pg, local)
    O.reset_counters()
    with ClockSampler(local) as cs:
        summ, secs = apps.cloverleaf3d(clover3d_deck(W + K, N), warmup_steps=W)
    clocks = cs.summary()
    barrier(pg, local)
    secs = max_over_ranks(pg, secs, local)

    kp = min(K, 10)
    O.set_kernel_timing(1)
    O.clear_kernel_timing()
    apps.cloverleaf3d(clover3d_deck(kp, N))
    stats = O.kernel_stats()
    O.set_kernel_timing(0)
    launches_per_step = sum(v[0] for v in stats.values()) / kp
    if args.kernel_table and rank == 0:
        print_kernel_table(stats, kp, cells, peaks["hbm_gbs"])
    dom, (n, ms, by) = max(stats.items(), key=lambda kv: kv[1][1])
    achieved = (by / n) / (ms / n * 1e-3) / 1e9
    tot_ms = sum(v[1] for v in stats.values())
    tot_by = sum(v[2] for v in stats.values())

    barrier(pg, local)
    t0 = time.perf_counter()
    apps.cloverleaf3d(clover3d_deck(K, N))
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(pg, t1 - t0, local)

    line = {
        "metric": "cell-updates/s",
        "value": world * cells * K / secs,
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": secs * 1e3 / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (background rho=0.2 e=1.0 + 3 SplitMix64-seeded cuboids, seed 6)",
        "config": {"workload": f"cloverleaf3d_{N}^3_fp64", "grid": [N, N, N], "gamma": 1.4,
                   "cell_update": "one cell advanced one hydro timestep",
                   "step": "timestep + PdV + accelerate + flux_calc + 3 advection sweeps + reset_field"
                           " + field_summary (5 FP64 sums read back)",
                   "l2": "inputs larger than L2 (about 40 fields of 140 MB)", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": TRAFFIC_PER_CELL["clover3d"] * cells
                     if dom == "cloverleaf3d/PdV_kernel_nopredict" else None,
                     "traffic_source": "ncu capture of PdV_kernel_nopredict at 160^3, per cell x cells"
                                       " (profiles/cloverleaf3d_160_pdv_accelerate.md)", "kernel": dom,
                     "alg_bytes_per_launch": by / n, "avg_launch_ms": ms / n, "peak_source": f"{peak_kind} hbm_gbs",
                     "step_effective_gbs": tot_by / (tot_ms * 1e-3) / 1e9,
                     "step_alg_bytes_per_cell": tot_by / kp / cells},
        "e2e": {"value": world * cells * K / e2e_s, "unit": "cell-updates/s", "h2d_bytes_per_step": 0.0,
                "d2h_bytes_per_step": 6 * 8 + 3 * 8,
                "note": "one C-ABI call: deck in, device set-up (generate), K cycles each reading dt and the"
                        " 5-value field summary back"},
        "gpu_launches": int(round(launches_per_step * K)),
        "clocks": clocks,
        "final_summary": {"vol": summ[-1, 2], "mass": summ[-1, 3], "ie": summ[-1, 4], "ke": summ[-1, 5],
                          "press": summ[-1, 6]},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        base = cpu_reference_clover3d(args.cpu_clover_steps, threads, N)
        if base:
            line["cpu_baseline"] = {"value": base[0], "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                                    "sample": f"reference CloverLeaf 3D OpenMP build, {N}^3, {args.cpu_clover_steps}"
                                              f" steps (hydro loop wall time {base[1]:.2f} s)"}
    return line


def reference_clover3d(args, world, rank):
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, args.cpu_clover_steps))
    N = args.grid or CL3_N
    base = cpu_reference_clover3d(steps, threads, N)
    if base is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/bin/cloverleaf3d was not built"}
    v, secs = base
    return {
        "impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": world,
        "steps": steps, "warmup": 0, "ms_per_step": secs * 1e3 / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (background rho=0.2 e=1.0 + 3 SplitMix64-seeded cuboids, seed 6)",
        "config": {"workload": f"cloverleaf3d_{N}^3_fp64", "grid": [N, N, N]},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                         "sample": f"{steps} steps of the reference OpenMP build at {N}^3 on {threads} threads"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# Batched tridiagonal ADI sweeps (ops_tridMultiDimBatch)
# ---------------------------------------------------------------------------
ADI_N = 256


def adi_batch_shapes(seed=3, nblocks=64, lo=32, hi=192):
    """64 blocks, each edge log-uniform in [32, 192] (numpy order z, y, x)."""
    import numpy as np

    from ops_b200 import seeded
    u = seeded.u01(seed, np.arange(3 * nblocks, dtype=np.uint64)).reshape(nblocks, 3)
    return [tuple(int(round(lo * (hi / lo) ** v)) for v in row) for row in u]


def bench_adi(args, world, rank, local, pg):
    import numpy as np
    import torch

    from ops_b200 import ops as O
    from ops_b200 import seeded

    peaks, peak_kind = load_peaks()
    O.ops_init(local, 0)
    dt = np.float64 if args.precision == "fp64" else np.float32
    es = np.dtype(dt).itemsize
    all_shapes = [(ADI_N,) * 3] if args.adi_case == "cube" else adi_batch_shapes()
    # the batch's blocks are independent units: over N GPUs each rank solves
    # its share, assigned by cost (unknowns), with no collective; the 256^3
    # cube runs as N replicas
    shard = args.adi_case == "batch" and world > 1
    owned = list(range(len(all_shapes)))
    if shard:
        from ops_b200.dist import assign_by_cost
        owned = assign_by_cost([int(np.prod(s)) for s in all_shapes], world)[rank]
    shapes = [all_shapes[i] for i in owned]
    total_unknowns = sum(int(np.prod(s)) for s in all_shapes)
    sets = []
    for i, shp in zip(owned, shapes):
        a, b, c, d = seeded.trid_system(shp, 0, 3 + i, dt)
        t = [torch.from_numpy(v).cuda(local) for v in (a, b, c, d)] + [torch.zeros(shp, dtype=torch.from_numpy(a).dtype,
                                                                               device=f"cuda:{local}")]
        sets.append((shp, t))
    unknowns = sum(int(np.prod(s)) for s, _ in sets)

    def systems(inc):
        out = []
        for shp, t in sets:
            out.append(dict(a=t[0].data_ptr(), b=t[1].data_ptr(), c=t[2].data_ptr(), d=t[3].data_ptr(),
                            u=t[4].data_ptr() if inc else None, dims=list(reversed(shp)), pads=list(reversed(shp))))
        return out

    sx, sy, sz = systems(False), systems(False), systems(True)
    stream = torch.cuda.current_stream(local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    sweep_ms = [0.0, 0.0, 0.0]

    def step(timed=False):
        if timed:
            ev[0].record(stream)
        O.trid_batch(es, 0, sx, stream.cuda_stream)
        if timed:
            ev[1].record(stream)
        O.trid_batch(es, 1, sy, stream.cuda_stream)
        if timed:
            ev[2].record(stream)
        O.trid_batch(es, 2, sz, stream.cuda_stream)
        if timed:
            ev[3].record(stream)

    K, W = args.steps, args.warmup
    for _ in range(W):
        step()
    torch.cuda.synchronize(local)
    barrier(pg, local)
    O.reset_counters()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as cs:
        t0.record(stream)
        for _ in range(K):
            step()
        t1.record(stream)
        torch.cuda.synchronize(local)
    clocks = cs.summary()
    launches = O.counters()["kernels"]
    secs = max_over_ranks(pg, t0.elapsed_time(t1) * 1e-3, local)
    # per-sweep event timing (separate pass)
    for _ in range(min(K, 5)):
        step(timed=True)
        torch.cuda.synchronize(local)
        for j in range(3):
            sweep_ms[j] += ev[j].elapsed_time(ev[j + 1]) / min(K, 5)
    dom = int(np.argmax(sweep_ms))
    byt = [40.0 * es / 8, 40.0 * es / 8, 48.0 * es / 8]
    achieved = byt[dom] * unknowns / (sweep_ms[dom] * 1e-3) / 1e9
    # e2e: every step copies a, b, c, d and u of every block in from pinned
    # host memory, runs the three sweeps through the C-ABI and copies u back
    # to pinned host memory (device buffers allocated once, before timing)
    host = [(shp, [x.cpu().pin_memory() for x in t]) for shp, t in sets]
    devs = [[torch.empty_like(h, device=f"cuda:{local}") for h in hv] for _, hv in host]
    outs = [torch.empty_like(hv[4]).pin_memory() for _, hv in host]
    e2e_sys = []
    for (shp, _), dev in zip(host, devs):
        s1 = [dict(a=dev[0].data_ptr(), b=dev[1].data_ptr(), c=dev[2].data_ptr(), d=dev[3].data_ptr(), u=None,
                   dims=list(reversed(shp)), pads=list(reversed(shp)))]
        e2e_sys.append((s1, [dict(s1[0], u=dev[4].data_ptr())]))

    def e2e_step():
        for (_, hv), dev, out, (s1, s3) in zip(host, devs, outs, e2e_sys):
            for dv, h in zip(dev, hv):
                dv.copy_(h, non_blocking=True)
            O.trid_batch(es, 0, s1, stream.cuda_stream)
            O.trid_batch(es, 1, s1, stream.cuda_stream)
            O.trid_batch(es, 2, s3, stream.cuda_stream)
            out.copy_(dev[4], non_blocking=True)
        torch.cuda.synchronize(local)

    e2e_step()
    KE = 3
    barrier(pg, local)
    te0 = time.perf_counter()
    for _ in range(KE):
        e2e_step()
    e2e_s = max_over_ranks(pg, (time.perf_counter() - te0) / KE, local)
    h2d = sum(5 * int(np.prod(s)) * es for s, _ in host)
    name = f"adi_{args.adi_case}_{args.precision}"
    line = {
        "metric": "cell-solves/s", "value": (total_unknowns if shard else world * unknowns) * 3 * K / secs,
        "unit": "unknowns solved/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": secs * 1e3 / K, "higher_is_better": True,
        "scaling": "strong" if shard else "weak", "vs_baseline": None, "dtype": args.precision.replace("fp", "f"),
        "data": "synthetic (a=c=-lam, b=1+2lam, lam~U[0.1,1] per line, d~N(0,1))",
        "config": {"workload": name, "blocks": len(all_shapes), "unknowns": total_unknowns,
                   "step": "x sweep + y sweep + z sweep (_Inc into u)", "l2": "inputs larger than L2"
                   if unknowns * es * 4 > 126e6 else "inputs fit in L2 (batch case)",
                   "parallelism": (f"{len(all_shapes)} blocks by cost over {world} GPUs (rank 0: {len(owned)})"
                                   if shard else f"replicas x{world}")},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "kernel": f"sweep {'xyz'[dom]}",
                     "traffic": TRAFFIC_PER_CELL["adi_cube_fp64"][dom] * unknowns
                     if name == "adi_cube_fp64" else None,
                     "traffic_source": "ncu capture of one x, y and z sweep at 256^3 FP64"
                                       " (profiles/adi_cube_256_fp64_dram.md); other cases not captured",
                     "sweep_ms": sweep_ms, "alg_bytes_per_unknown": byt, "peak_source": f"{peak_kind} hbm_gbs"},
        "e2e": {"value": (total_unknowns if shard else world * unknowns) * 3 / e2e_s, "unit": "unknowns solved/s",
                "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": unknowns * es},
        "gpu_launches": launches, "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import ctypes

        import oracle
        L = oracle.lib()
        f = L.oracle_trid_batch_d if dt == np.float64 else L.oracle_trid_batch_s
        tc = time.perf_counter()
        for shp, hv in host:
            dims = (ctypes.c_int * 3)(*reversed(shp))
            a, b, c, d, u = [np.ascontiguousarray(v) for v in hv]
            for sd, uu in ((0, None), (1, None), (2, u)):
                f(a.ctypes.data, b.ctypes.data, c.ctypes.data, d.ctypes.data, None if uu is None else uu.ctypes.data,
                  3, sd, dims, dims)
        cs_ = time.perf_counter() - tc
        line["cpu_baseline"] = {"value": 3 * unknowns / cs_, "unit": "unknowns solved/s", "cores": os.cpu_count(),
                                "kind": "port", "sample": f"oracle Thomas (OpenMP over lines), one x+y+z step, {cs_:.2f} s"}
    return line


def reference_adi(args, world, rank):
    """The reference's tridiagonal solver is the external Tridsolver library,
    not vendored with the reference, so its CPU path cannot be built: the
    oracle's Thomas restatement (OpenMP over lines, all host threads) stands
    in for it, on the same seeded systems and the same x + y + z(_Inc) step."""
    import ctypes

    import numpy as np

    import oracle
    from ops_b200 import seeded
    threads = os.cpu_count() or 1
    dt = np.float64 if args.precision == "fp64" else np.float32
    shapes = [(ADI_N,) * 3] if args.adi_case == "cube" else adi_batch_shapes()
    L = oracle.lib()
    f = L.oracle_trid_batch_d if dt == np.float64 else L.oracle_trid_batch_s
    sets = []
    for i, shp in enumerate(shapes):
        a, b, c, d = seeded.trid_system(shp, 0, 3 + i, dt)
        sets.append((shp, a, b, c, d, np.zeros(shp, dtype=dt)))
    unknowns = sum(int(np.prod(t[0])) for t in sets)

    def step():
        for shp, a, b, c, d, u in sets:
            dims = (ctypes.c_int * 3)(*reversed(shp))
            for sd, uu in ((0, None), (1, None), (2, u)):
                f(a.ctypes.data, b.ctypes.data, c.ctypes.data, d.ctypes.data, None if uu is None else uu.ctypes.data,
                  3, sd, dims, dims)

    step()
    K = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(K):
        step()
    secs = time.perf_counter() - t0
    v = 3 * unknowns * K / secs
    name = f"adi_{args.adi_case}_{args.precision}"
    return {
        "impl": "reference", "metric": "cell-solves/s", "value": v, "unit": "unknowns solved/s", "n_gpus": world,
        "steps": K, "warmup": 1, "ms_per_step": secs * 1e3 / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.precision.replace("fp", "f"),
        "data": "synthetic (a=c=-lam, b=1+2lam, lam~U[0.1,1] per line, d~N(0,1))",
        "config": {"workload": name, "blocks": len(shapes), "unknowns": unknowns,
                   "step": "x sweep + y sweep + z sweep (_Inc into u)"},
        "cpu_baseline": {"value": v, "unit": "unknowns solved/s", "cores": threads, "kind": "port",
                         "sample": f"{K} steps of the oracle Thomas (OpenMP over lines) on {threads} host threads;"
                                   " Tridsolver, the reference's solver, is not vendored"},
        "e2e": {"value": v, "unit": "unknowns solved/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# Implicit heat conduction (TeaLeaf CG, jac_diag), 4096^2, eps 1e-10
# ---------------------------------------------------------------------------
TEA_N = 4096
TEA_BYTES_FP64 = 120.0   # per cell-iteration: k_w 32 + k_ur 64 + k_p 24 (FP64 words)
TEA_BYTES_FP32 = 60.0


def tea_deck(steps, n=TEA_N, max_iters=200000, **kw):
    from ops_b200 import apps, seeded
    return apps.tea_deck(x_cells=n, y_cells=n, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0, initial_timestep=0.004,
                         end_step=steps, summary_frequency=0, max_iters=max_iters, eps=1e-10, solver=1,
                         preconditioner=1, states=seeded.tea_config4_states(n, n, 4), **kw)


def cpu_reference_tea_converged(threads, n=TEA_N):
    """The reference OpenMP TeaLeaf's Jacobi-PCG on the same deck run to its
    own stopping test (eps 1e-10): (solve seconds, iterations). The solve time
    is the wall-time difference to the same run capped at 2 iterations (its
    set-up), plus those 2 iterations at the run's own mean rate."""
    import oracle
    from ops_b200 import apps
    exe = oracle.reference_binary("tealeaf")
    if exe is None:
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    wall, iters = [], []
    for m in (2, 200000):
        with tempfile.TemporaryDirectory() as td:
            with open(os.path.join(td, "tea.in"), "w") as f:
                f.write(apps.tea_deck_text(tea_deck(1, n, max_iters=m)))
            r = subprocess.run([exe], cwd=td, capture_output=True, text=True, env=env, timeout=1800, check=True)
        wall.append([float(l.split()[-1]) for l in r.stdout.splitlines() if l.strip().startswith("Total Wall time")][-1])
        iters.append([int(l.split()[-1]) for l in r.stdout.splitlines() if l.strip().startswith("Iteration count")][-1])
    n_it = iters[1]
    per_it = (wall[1] - wall[0]) / max(1, n_it - 2)
    return (wall[1] - wall[0]) + 2 * per_it, n_it


def cpu_reference_tea(iters, threads, n=TEA_N):
    """Seconds per CG iteration of the reference OpenMP TeaLeaf on the same
    deck: two runs capped at 2 and 2 + iters iterations, wall-time difference."""
    import oracle
    from ops_b200 import apps
    exe = oracle.reference_binary("tealeaf")
    if exe is None:
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    wall = []
    for m in (2, 2 + iters):
        with tempfile.TemporaryDirectory() as td:
            with open(os.path.join(td, "tea.in"), "w") as f:
                f.write(apps.tea_deck_text(tea_deck(1, n, max_iters=m)))
            r = subprocess.run([exe], cwd=td, capture_output=True, text=True, env=env, timeout=1800, check=True)
        wall.append([float(l.split()[-1]) for l in r.stdout.splitlines() if l.strip().startswith("Total Wall time")][-1])
    return (wall[1] - wall[0]) / iters, wall


def bench_tea(args, world, rank, local, pg):
    import numpy as np

    from ops_b200 import apps
    from ops_b200 import ops as O

    peaks, peak_kind = load_peaks()
    O.ops_init(local, 0)
    N = args.grid or TEA_N
    cells = N * N
    K, W = args.steps, args.warmup
    td = tempfile.mkdtemp(prefix="tea_bench_")
    barrier(pg, local)

    def run(tag, **kw):
        O.reset_counters()
        with ClockSampler(local) as cs:
            _, sv, _ = apps.tealeaf(tea_deck(W + K, N, **kw), dump_dir=os.path.join(td, tag))
        return sv[W:], cs.summary(), O.counters()["kernels"]

    os.makedirs(os.path.join(td, "plain"))
    os.makedirs(os.path.join(td, "mixed"))
    sp, clk_p, launches_p = run("plain", fused=1, true_residual_stop=1)
    sm, clk_m, launches_m = run("mixed", fused=1, mixed=1, reliable_delta=args.reliable_delta)
    up = np.fromfile(os.path.join(td, "plain", "u.bin"))
    um = np.fromfile(os.path.join(td, "mixed", "u.bin"))
    err_vs_fp64 = float(np.linalg.norm(um - up) / np.linalg.norm(up))
    shutil.rmtree(td, ignore_errors=True)

    t_plain = max_over_ranks(pg, float(np.median(sp[:, 6])), local)
    t_mixed = max_over_ranks(pg, float(np.median(sm[:, 6])), local)
    it_p = float(np.mean(sp[:, 0]))
    it_m = float(np.mean(sm[:, 0]))
    # roofline of the dominant chain: the FP32 inner iteration (k_w + k_ur + k_p)
    per_it_m = t_mixed / max(it_m, 1.0)
    per_it_p = t_plain / max(it_p, 1.0)
    ach_m = TEA_BYTES_FP32 * cells / per_it_m / 1e9
    ach_p = TEA_BYTES_FP64 * cells / per_it_p / 1e9

    # e2e: one public C-ABI call (deck in, device set-up, one solve, summaries back), wall clock
    barrier(pg, local)
    te0 = time.perf_counter()
    _, sv_e2e, _ = apps.tealeaf(tea_deck(1, N, fused=1, mixed=1, reliable_delta=args.reliable_delta))
    e2e_s = max_over_ranks(pg, time.perf_counter() - te0, local)

    line = {
        "metric": "time to 1e-10 residual",
        "value": t_mixed,
        "unit": "s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": t_mixed * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 outer / f32 inner",
        "data": "synthetic (rho=1 background + 16 SplitMix64-seeded rectangles, rho log-uniform [0.1,100],"
                " energy U[0,1], seed 4)",
        "config": {"workload": f"tealeaf2d_cg_jacdiag_{N}x{N}", "grid": [N, N], "eps": 1e-10,
                   "step": "one implicit timestep: coefficient set-up + solve to ||u0 - A u|| < 1e-10 ||r0|| +"
                           " finalise", "l2": "inputs larger than L2 (fields of 134 MB FP64 / 67 MB FP32 x 8)",
                   "reliable_delta": args.reliable_delta, "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": ach_m, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": ach_m / peaks["hbm_gbs"], "traffic": None,
                     "kernel": "FP32 inner PCG iteration (k_w + k_ur + k_p)",
                     "alg_bytes_per_cell_iteration": TEA_BYTES_FP32, "avg_iteration_ms": per_it_m * 1e3,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "fp64_iteration": {"achieved": ach_p, "frac": ach_p / peaks["hbm_gbs"],
                                        "alg_bytes_per_cell_iteration": TEA_BYTES_FP64,
                                        "avg_iteration_ms": per_it_p * 1e3}},
        "plain_fp64_pcg": {"seconds": t_plain, "iterations": it_p,
                           "tealeaf_stop_ratio": float(np.max(sp[:, 2])), "true_residual_ratio": float(np.max(sp[:, 4])),
                           "cell_iterations_per_s": cells * it_p / t_plain, "gpu_launches": launches_p},
        "mixed_pcg": {"seconds": t_mixed, "inner_iterations": it_m, "reliable_updates": float(np.mean(sm[:, 5])),
                      "true_residual_ratio": float(np.max(sm[:, 4])), "rel_l2_error_vs_fp64_solution": err_vs_fp64,
                      "speedup_vs_plain": t_plain / t_mixed},
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 13 * 8,
                "note": "one C-ABI call: deck in, device set-up (generate), one mixed-precision solve, summaries back",
                "solve_seconds": float(sv_e2e[0, 6])},
        "gpu_launches": int(round(launches_m / (W + K))),
        "clocks": clk_m,
        "clocks_plain": clk_p,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        base = cpu_reference_tea(args.cpu_tea_iters, threads, N)
        if base:
            per_it = base[0]
            line["cpu_baseline"] = {
                "value": cells / per_it, "unit": "cell-iterations/s", "cores": threads, "kind": "reference",
                "sample": f"reference TeaLeaf OpenMP build, same {N}^2 deck, CG capped at 2 and"
                          f" {2 + args.cpu_tea_iters} iterations (wall {base[1][0]:.2f} s / {base[1][1]:.2f} s)",
                "est_time_to_solution_s": per_it * it_p}
    return line


def reference_tea(args, world, rank):
    threads = os.cpu_count() or 1
    N = args.grid or TEA_N
    base = cpu_reference_tea_converged(threads, N)
    if base is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/bin/tealeaf was not built"}
    v, iters = base
    return {
        "impl": "reference",
        "metric": {"learned": "time to 1e-10 residual (learned FCG)",
                   "mg": "time to 1e-10 residual (multigrid FCG)"}.get(args.workload, "time to 1e-10 residual"),
        "value": v, "unit": "s", "n_gpus": world,
        "steps": 1, "warmup": 0, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (rho=1 background + 16 SplitMix64-seeded rectangles, seed 4)",
        "config": {"workload": {"learned": f"tealeaf2d_learned_fcg_{N}x{N}",
                                "mg": f"tealeaf2d_multigrid_fcg_{N}x{N}"}.get(args.workload,
                                                                             f"tealeaf2d_cg_jacdiag_{N}x{N}"),
                   "grid": [N, N], "eps": 1e-10},
        "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "reference",
                         "sample": f"reference OpenMP TeaLeaf Jacobi-PCG run to its own stopping test"
                                   f" (sqrt|r.z| < 1e-10 ||r0||, {iters} iterations), one timestep; solve"
                                   f" time = wall time minus the same run capped at 2 iterations, plus 2"
                                   f" iterations"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# Learned multigrid preconditioner in flexible CG vs plain Jacobi-PCG
# ---------------------------------------------------------------------------
def bench_learned(args, world, rank, local, pg):
    import numpy as np
    import torch

    from ops_b200 import cnn, lmg
    from ops_b200 import ops as O

    peaks, peak_kind = load_peaks()
    O.ops_init(local, 0)
    N = args.grid or TEA_N
    rx = 0.004 / (10.0 / N) ** 2          # the implicit timestep of the 4096^2 heat problem (dt = 0.004)
    K, W = args.steps, args.warmup

    # training on the GPU: PCG pairs + three on-policy rounds on 64^2 fields
    t0 = time.perf_counter()
    net = lmg.Net(seed=5)
    hists = lmg.fit(net, n=64, nfields=300, steps=1500, rounds=3)
    torch.cuda.synchronize(local)
    train_s = time.perf_counter() - t0
    # the learned correction of the native V-cycle: PCG pairs retargeted to
    # e - V-cycle(r), one on-policy round
    t0 = time.perf_counter()
    net_mg = lmg.Net(seed=5)
    hists_mg = lmg.fit(net_mg, n=64, nfields=300, steps=1500, rounds=1, base="mg")
    torch.cuda.synchronize(local)
    train_mg_s = time.perf_counter() - t0

    rho, en = lmg.density_field(N, 4)
    Kx, Ky, u0 = lmg.padded_problem(rho, en)
    kx, ky, b = (torch.from_numpy(a).cuda(local) for a in (Kx, Ky, u0))
    u = torch.empty_like(b)

    def run(method, window=40):
        u.copy_(b)
        h = net_mg.h if method == lmg.FCG_LEARNED_MG else net.h
        return lmg.solve(kx, ky, b, u, rx, rx, method=method, net=h, eps=1e-10, window=window, max_iters=20000)

    for _ in range(W):
        run(lmg.PCG_TRUE)
        run(lmg.FCG_LEARNED)
        run(lmg.FCG_MG)
        run(lmg.FCG_LEARNED_MG)
    barrier(pg, local)
    with ClockSampler(local) as cs:
        plain = [run(lmg.PCG_TRUE) for _ in range(K)]
        learned = [run(lmg.FCG_LEARNED) for _ in range(K)]
        multigrid = [run(lmg.FCG_MG) for _ in range(K)]
        learned_mg = [run(lmg.FCG_LEARNED_MG) for _ in range(K)]
    clocks = cs.summary()
    u_lmg = u.clone()
    t_lmg = max_over_ranks(pg, float(np.median([s["seconds"] for s in learned_mg])), local)
    u_mg = u.clone()
    run(lmg.FCG_LEARNED)
    u_learned = u.clone()
    run(lmg.PCG_TRUE)
    err = float(torch.linalg.norm(u_learned - u) / torch.linalg.norm(u))
    err_mg = float(torch.linalg.norm(u_mg - u) / torch.linalg.norm(u))
    err_lmg = float(torch.linalg.norm(u_lmg - u) / torch.linalg.norm(u))
    t_mg = max_over_ranks(pg, float(np.median([s["seconds"] for s in multigrid])), local)
    t_plain = max_over_ranks(pg, float(np.median([s["seconds"] for s in plain])), local)
    t_learned = max_over_ranks(pg, float(np.median([s["seconds"] for s in learned])), local)

    # the dominant kernel: the full-resolution 16 -> 16 channel tcgen05 convolution
    x = torch.zeros((1, N, N, 16), dtype=torch.bfloat16, device=f"cuda:{local}")
    y = torch.empty_like(x)
    wt = torch.zeros((9, 16, 16), dtype=torch.bfloat16, device=f"cuda:{local}")
    bias = torch.zeros(16, dtype=torch.float32, device=f"cuda:{local}")
    stream = torch.cuda.current_stream(local)
    for _ in range(3):
        cnn.conv3x3(x, wt, y, bias=bias, mode=cnn.CONV_BIAS_RELU, stream=stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(10):
        cnn.conv3x3(x, wt, y, bias=bias, mode=cnn.CONV_BIAS_RELU, stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize(local)
    conv_ms = e0.elapsed_time(e1) / 10
    conv_bytes = 2.0 * N * N * 16 * 2          # read x, write y (BF16, 16 channels)
    conv_gbs = conv_bytes / (conv_ms * 1e-3) / 1e9
    conv_tflops = 2.0 * 9 * 16 * 16 * N * N / (conv_ms * 1e-3) / 1e12

    # the gain on the training scale: held-out 64^2 fields, rx = 400
    small = []
    for seed in (90001, 90002, 90003):
        r_, e_ = lmg.density_field(64, seed)
        a, c, d = lmg.padded_problem(r_, e_)
        skx, sky, sb = (torch.from_numpy(v).cuda(local) for v in (a, c, d))
        row = {}
        for name, m, h in (("pcg", lmg.PCG_TRUE, net.h), ("learned_fcg", lmg.FCG_LEARNED, net.h),
                           ("multigrid_fcg", lmg.FCG_MG, net.h), ("learned_mg_fcg", lmg.FCG_LEARNED_MG, net_mg.h)):
            su = sb.clone()
            st = lmg.solve(skx, sky, sb, su, 400.0, 400.0, method=m, net=h, eps=1e-10, window=40)
            row[name] = {"iterations": st["iterations"], "seconds": st["seconds"], "fallbacks": st["fallbacks"]}
        small.append(row)

    # the network's gain as the grid grows (one seeded field per size, rx 400,
    # the middle of the training range): iterations and time of plain PCG and
    # of the learned FCG on the same problem
    sweep = []
    for n_ in (64, 128, 256, 512, 1024):
        r_, e_ = lmg.density_field(n_, 91000 + n_)
        a, c, d = lmg.padded_problem(r_, e_)
        skx, sky, sb = (torch.from_numpy(v).cuda(local) for v in (a, c, d))
        row = {"n": n_}
        for name, m in (("pcg", lmg.PCG_TRUE), ("learned_fcg", lmg.FCG_LEARNED)):
            su = sb.clone()
            lmg.solve(skx, sky, sb, su, 400.0, 400.0, method=m, net=net.h, eps=1e-10, window=40)  # untimed
            su = sb.clone()
            st = lmg.solve(skx, sky, sb, su, 400.0, 400.0, method=m, net=net.h, eps=1e-10, window=40)
            row[name] = {"iterations": st["iterations"], "seconds": st["seconds"], "fallbacks": st["fallbacks"]}
        row["iteration_ratio"] = row["learned_fcg"]["iterations"] / max(1, row["pcg"]["iterations"])
        row["time_ratio"] = row["learned_fcg"]["seconds"] / max(1e-12, row["pcg"]["seconds"])
        sweep.append(row)

    # e2e: Kx, Ky, u0 in from pinned host memory, one solve through the C-ABI,
    # the solution out to pinned host memory (buffers allocated before timing;
    # one untimed call first, as the timed solves above had)
    hk = [torch.from_numpy(a).pin_memory() for a in (Kx, Ky, u0)]
    dk = [torch.empty_like(t, device=f"cuda:{local}") for t in hk]
    du = torch.empty_like(dk[2])
    host_u = torch.empty_like(hk[2]).pin_memory()

    def e2e_solve():
        for d_, h_ in zip(dk, hk):
            d_.copy_(h_, non_blocking=True)
        du.copy_(dk[2])
        st_ = lmg.solve(dk[0], dk[1], dk[2], du, rx, rx, method=lmg.FCG_LEARNED, net=net.h, eps=1e-10, window=40)
        host_u.copy_(du, non_blocking=True)
        torch.cuda.synchronize(local)
        return st_

    e2e_solve()
    barrier(pg, local)
    te = time.perf_counter()
    st_e2e = e2e_solve()
    e2e_s = max_over_ranks(pg, time.perf_counter() - te, local)
    net.close()
    net_mg.close()

    line = {
        "metric": "time to 1e-10 residual (learned FCG)", "value": t_learned, "unit": "s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": t_learned * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 solve / bf16 network",
        "data": "synthetic (rho=1 background + 16 SplitMix64-seeded rectangles, rho log-uniform [0.1,100], seed 4);"
                " network trained on 300 + 3 x 150 seeded 64^2 fields",
        "config": {"workload": f"tealeaf2d_learned_fcg_{N}x{N}", "grid": [N, N], "rx": rx, "eps": 1e-10,
                   "network": "4-level U-Net 16/32/64/64 ch, 3x3 tcgen05 BF16 convs, FP32 accumulation",
                   "training": "A-norm loss, PCG pairs + 3 on-policy rounds, 64^2 fields, 1500 Adam steps each",
                   "fallback": "Jacobi-PCG when ||r|| has not halved in 40 iterations",
                   "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"},
        "plain_pcg": {"seconds": t_plain, "iterations": plain[0]["iterations"],
                      "final_residual_ratio": plain[0]["final_residual"] / plain[0]["initial_residual"]},
        "learned_fcg": {"seconds": t_learned, "iterations": learned[0]["iterations"],
                        "fallbacks": learned[0]["fallbacks"],
                        "final_residual_ratio": learned[0]["final_residual"] / learned[0]["initial_residual"],
                        "rel_l2_vs_fp64_pcg_solution": err, "time_ratio_vs_plain": t_learned / t_plain},
        "multigrid_fcg": {"seconds": t_mg, "iterations": multigrid[0]["iterations"],
                          "fallbacks": multigrid[0]["fallbacks"], "launches": int(multigrid[0]["launches"]),
                          "final_residual_ratio": multigrid[0]["final_residual"] / multigrid[0]["initial_residual"],
                          "rel_l2_vs_fp64_pcg_solution": err_mg, "time_ratio_vs_plain": t_mg / t_plain,
                          "note": "native FP32 aggregation V-cycle (2+2 damped-Jacobi sweeps) per FCG iteration,"
                                  " hierarchy setup inside the timed solve"},
        "learned_mg_fcg": {"seconds": t_lmg, "iterations": learned_mg[0]["iterations"],
                           "fallbacks": learned_mg[0]["fallbacks"],
                           "final_residual_ratio": learned_mg[0]["final_residual"] / learned_mg[0]["initial_residual"],
                           "rel_l2_vs_fp64_pcg_solution": err_lmg, "time_ratio_vs_plain": t_lmg / t_plain,
                           "time_ratio_vs_multigrid_alone": t_lmg / t_mg, "training_seconds": train_mg_s,
                           "final_loss_per_round": [float(np.mean(h[-50:])) for h in hists_mg],
                           "note": "M(r) = V-cycle(r) + the network's correction, trained on e - V-cycle(r)"},
        "training": {"seconds": train_s, "final_loss_per_round": [float(np.mean(h[-50:])) for h in hists]},
        "small_scale_gain_64x64_rx400": small,
        "grid_sweep_rx400": sweep,
        "roofline": {"bound": "hbm", "achieved": conv_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": conv_gbs / peaks["hbm_gbs"], "traffic": None,
                     "kernel": "conv3x3_tc_kernel<16,16> (full-resolution layer)", "avg_launch_ms": conv_ms,
                     "alg_bytes_per_launch": conv_bytes, "tensor_tflops": conv_tflops,
                     "peak_source": f"{peak_kind} hbm_gbs"},
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 3 * (N + 2) ** 2 * 8,
                "d2h_bytes_per_step": (N + 2) ** 2 * 8, "solve_seconds": st_e2e["seconds"],
                "note": "Kx, Ky, u0 from pinned host memory, one learned-FCG solve through ops_b200_heat_solve,"
                        " solution back to the host"},
        "gpu_launches": int(learned[0]["launches"]), "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        base = cpu_reference_tea(args.cpu_tea_iters, threads, N)
        if base:
            line["cpu_baseline"] = {
                "value": base[0] * plain[0]["iterations"], "unit": "s", "cores": threads, "kind": "reference",
                "sample": f"reference TeaLeaf OpenMP build, same {N}^2 deck, seconds per CG iteration from runs"
                          f" capped at 2 and {2 + args.cpu_tea_iters} iterations, times the FP64 PCG count"}
    del host_u
    return line


# ---------------------------------------------------------------------------
# Native multigrid preconditioner in flexible CG vs plain Jacobi-PCG
# ---------------------------------------------------------------------------
def bench_mg(args, world, rank, local, pg):
    import numpy as np
    import torch

    from ops_b200 import lmg
    from ops_b200 import ops as O

    peaks, peak_kind = load_peaks()
    O.ops_init(local, 0)
    N = args.grid or TEA_N
    rx = 0.004 / (10.0 / N) ** 2          # the implicit timestep of the 4096^2 heat problem (dt = 0.004)
    K, W = args.steps, args.warmup
    rho, en = lmg.density_field(N, 4)
    Kx, Ky, u0 = lmg.padded_problem(rho, en)
    kx, ky, b = (torch.from_numpy(a).cuda(local) for a in (Kx, Ky, u0))
    u = torch.empty_like(b)

    def run(method):
        u.copy_(b)
        return lmg.solve(kx, ky, b, u, rx, rx, method=method, eps=1e-10, window=40, max_iters=20000)

    for _ in range(W):
        run(lmg.FCG_MG)
    barrier(pg, local)
    with ClockSampler(local) as cs:
        mg = [run(lmg.FCG_MG) for _ in range(K)]
    clocks = cs.summary()
    u_mg = u.clone()
    plain = [run(lmg.PCG_TRUE) for _ in range(max(1, min(K, 2)))]
    err = float(torch.linalg.norm(u_mg - u) / torch.linalg.norm(u))
    t_mg = max_over_ranks(pg, float(np.median([s["seconds"] for s in mg])), local)
    t_plain = max_over_ranks(pg, float(np.median([s["seconds"] for s in plain])), local)
    it = mg[0]["iterations"]
    # algorithmic bytes of one iteration, per cell: the FP64 flexible-CG
    # kernels (w = A p with p.w, p.r: Kx Ky p r w 40; u, r update: 48; z.w: 16;
    # p = z + beta p: 24) and the FP32 V-cycle's fine level (106: r in FP64 and
    # its FP32 copy, five streaming passes, z out in FP64) plus its coarse
    # levels (a third of the fine level's 5 x 20 bytes in FP32)
    per_cell = 128 + 106 + 100 / 3
    alg = per_cell * N * N * it
    ach = alg / t_mg / 1e9

    # e2e: Kx, Ky, u0 in from pinned host memory, one solve through the C-ABI,
    # the solution out to pinned host memory (buffers allocated before timing;
    # one untimed call first, as the timed solves above had)
    hk = [torch.from_numpy(a).pin_memory() for a in (Kx, Ky, u0)]
    dk = [torch.empty_like(t, device=f"cuda:{local}") for t in hk]
    du = torch.empty_like(dk[2])
    host_u = torch.empty_like(hk[2]).pin_memory()

    def e2e_solve():
        for d_, h_ in zip(dk, hk):
            d_.copy_(h_, non_blocking=True)
        du.copy_(dk[2])
        st_ = lmg.solve(dk[0], dk[1], dk[2], du, rx, rx, method=lmg.FCG_MG, eps=1e-10, window=40)
        host_u.copy_(du, non_blocking=True)
        torch.cuda.synchronize(local)
        return st_

    e2e_solve()
    barrier(pg, local)
    te = time.perf_counter()
    st_e2e = e2e_solve()
    e2e_s = max_over_ranks(pg, time.perf_counter() - te, local)
    del host_u
    line = {
        "metric": "time to 1e-10 residual (multigrid FCG)", "value": t_mg, "unit": "s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": t_mg * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 solve / f32 V-cycle",
        "data": "synthetic (rho=1 background + 16 SplitMix64-seeded rectangles, rho log-uniform [0.1,100], seed 4)",
        "config": {"workload": f"tealeaf2d_multigrid_fcg_{N}x{N}", "grid": [N, N], "rx": rx, "eps": 1e-10,
                   "preconditioner": "2x2 aggregation, coarse faces x 1/2, 2+2 damped-Jacobi sweeps (0.8),"
                                     " 16x16 coarsest level, one V-cycle per FCG iteration",
                   "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"},
        "multigrid_fcg": {"seconds": t_mg, "iterations": it, "fallbacks": mg[0]["fallbacks"],
                          "final_residual_ratio": mg[0]["final_residual"] / mg[0]["initial_residual"],
                          "rel_l2_vs_fp64_pcg_solution": err},
        "plain_pcg": {"seconds": t_plain, "iterations": plain[0]["iterations"],
                      "time_ratio_mg_vs_plain": t_mg / t_plain},
        "roofline": {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": ach / peaks["hbm_gbs"], "traffic": None,
                     "kernel": "whole solve (every kernel of the FCG iterations and V-cycles)",
                     "alg_bytes_per_cell_iteration": per_cell, "peak_source": f"{peak_kind} hbm_gbs"},
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 3 * (N + 2) ** 2 * 8,
                "d2h_bytes_per_step": (N + 2) ** 2 * 8, "solve_seconds": st_e2e["seconds"],
                "note": "Kx, Ky, u0 from pinned host memory, one multigrid-FCG solve through ops_b200_heat_solve,"
                        " solution back to the host"},
        "gpu_launches": int(mg[0]["launches"]), "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        base = cpu_reference_tea(args.cpu_tea_iters, threads, N)
        if base:
            line["cpu_baseline"] = {
                "value": base[0] * plain[0]["iterations"], "unit": "s", "cores": threads, "kind": "reference",
                "sample": f"reference TeaLeaf OpenMP build, same {N}^2 deck, seconds per CG iteration from runs"
                          f" capped at 2 and {2 + args.cpu_tea_iters} iterations, times the FP64 PCG count"}
    return line


# ---------------------------------------------------------------------------
# 3D heat solve: the 7-point operator at 512^3, FP64 Jacobi-PCG to 1e-10
# ---------------------------------------------------------------------------
H3_N = 512
HEAT3D_BYTES = 128.0  # FP64 per cell-iteration: w = A p (p, Kx, Ky, Kz, w: 40) + u, r, z updates (64) + p (24)
# DRAM bytes per cell of one iteration (k_w3 + k_ur + k_p) from one ncu capture
# at 256^3 (profiles/heat3d_256_pcg_iteration_dram.md); they scale with the cells
HEAT3D_TRAFFIC = 124.8


def heat3d_problem(n, seed, local):
    """16 seeded boxes of density log-uniform in [0.1, 100] over rho = 1 and
    energy U[0, 1] (the 2D heat configuration's recipe in 3D); face
    conductivities as ops_b200.lmg.faces3d, built on the device."""
    import numpy as np
    import torch
    rng = np.random.default_rng(seed)
    dev = f"cuda:{local}"
    rho = torch.ones((n, n, n), dtype=torch.float64, device=dev)
    for _ in range(16):
        lo = rng.integers(0, n - 1, 3)
        hi = np.minimum(n, lo + rng.integers(n // 16, n // 3, 3))
        rho[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = float(np.exp(rng.uniform(np.log(0.1), np.log(100.0))))
    g = torch.Generator(device=dev).manual_seed(seed)
    en = torch.rand((n, n, n), dtype=torch.float64, device=dev, generator=g)
    shape = (n + 2, n + 2, n + 2)
    Kx, Ky, Kz, u0 = (torch.zeros(shape, dtype=torch.float64, device=dev) for _ in range(4))
    w = rho
    Kx[1:-1, 1:-1, 2:-1] = (w[:, :, :-1] + w[:, :, 1:]) / (2.0 * w[:, :, :-1] * w[:, :, 1:])
    Ky[1:-1, 2:-1, 1:-1] = (w[:, :-1, :] + w[:, 1:, :]) / (2.0 * w[:, :-1, :] * w[:, 1:, :])
    Kz[2:-1, 1:-1, 1:-1] = (w[:-1, :, :] + w[1:, :, :]) / (2.0 * w[:-1, :, :] * w[1:, :, :])
    u0[1:-1, 1:-1, 1:-1] = en * rho
    del rho, en
    return Kx, Ky, Kz, u0


def bench_heat3d(args, world, rank, local, pg):
    import numpy as np
    import torch

    from ops_b200 import lmg
    from ops_b200 import ops as O

    peaks, peak_kind = load_peaks()
    O.ops_init(local, 0)
    N = args.grid or H3_N
    cells = N ** 3
    rxyz = 100.0
    Kx, Ky, Kz, u0 = heat3d_problem(N, 6, local)
    u = torch.empty_like(u0)
    K, W = args.steps, args.warmup
    barrier(pg, local)
    times, stats = [], None
    with ClockSampler(local) as cs:
        for it in range(W + K):
            u.copy_(u0)
            st = lmg.solve3d(Kx, Ky, Kz, u0, u, rxyz, rxyz, rxyz, method=lmg.PCG_TRUE, eps=1e-10)
            if it >= W:
                times.append(st["seconds"])
                stats = st
        # the mixed-precision solve of the same problem (FP32 inner PCG, FP64 reliable updates)
        mtimes, mstats = [], None
        for it in range(1 + K):
            u.copy_(u0)
            st = lmg.solve3d(Kx, Ky, Kz, u0, u, rxyz, rxyz, rxyz, method=lmg.MIXED, eps=1e-10)
            if it >= 1:
                mtimes.append(st["seconds"])
                mstats = st
    clocks = cs.summary()
    t = max_over_ranks(pg, float(np.median(times)), local)
    tm = max_over_ranks(pg, float(np.median(mtimes)), local)
    iters = stats["iterations"]
    achieved = HEAT3D_BYTES * cells * iters / t / 1e9
    # e2e: Kx, Ky, Kz, u0 in from pinned host memory, one solve through the
    # C-ABI, u out to pinned host memory (buffers allocated before timing)
    hk = [x.cpu().pin_memory() for x in (Kx, Ky, Kz, u0)]
    hu = torch.empty_like(hk[3]).pin_memory()
    barrier(pg, local)
    torch.cuda.synchronize(local)
    te0 = time.perf_counter()
    for d_, h_ in zip((Kx, Ky, Kz, u0), hk):
        d_.copy_(h_, non_blocking=True)
    u.copy_(u0)
    lmg.solve3d(Kx, Ky, Kz, u0, u, rxyz, rxyz, rxyz, method=lmg.PCG_TRUE, eps=1e-10)
    hu.copy_(u, non_blocking=True)
    torch.cuda.synchronize(local)
    e2e_s = max_over_ranks(pg, time.perf_counter() - te0, local)
    line = {
        "metric": "time to 1e-10 residual", "value": t, "unit": "s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (rho=1 background + 16 seeded boxes, rho log-uniform [0.1,100], energy U[0,1], seed 6)",
        "config": {"workload": f"heat3d_pcg_{N}^3", "grid": [N, N, N], "rx=ry=rz": rxyz, "eps": 1e-10,
                   "step": "one FP64 Jacobi-PCG solve of the 7-point operator to ||u0 - A u|| < 1e-10 ||r0||",
                   "l2": f"inputs larger than L2 (fields of {8 * (N + 2) ** 3 / 1e9:.2f} GB)",
                   "parallelism": f"replicas x{world}"},
        "iterations": iters, "final_residual_ratio": stats["final_residual"] / max(stats["initial_residual"], 1e-300),
        "mixed_pcg": {"seconds": tm, "inner_iterations": mstats["iterations"], "reliable_updates": mstats["updates"],
                      "final_residual_ratio": mstats["final_residual"] / max(mstats["initial_residual"], 1e-300),
                      "speedup_vs_fp64": t / tm},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": HEAT3D_TRAFFIC * cells,
                     "traffic_source": "ncu capture of one iteration at 256^3, per cell x cells"
                                       " (profiles/heat3d_256_pcg_iteration_dram.md)",
                     "kernel": "PCG iteration (k_w3 + k_ur + k_p)", "alg_bytes_per_cell_iteration": HEAT3D_BYTES,
                     "avg_iteration_ms": t * 1e3 / max(iters, 1), "peak_source": f"{peak_kind} hbm_gbs"},
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": sum(h.numel() * 8 for h in hk),
                "d2h_bytes_per_step": hu.numel() * 8},
        "gpu_launches": int(stats["launches"]), "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the same iteration in numpy on a 96^3 sample, one core (no 3D reference exists)
        n_ = 96
        rng = np.random.default_rng(7)
        sh = (n_ + 2,) * 3
        A = [np.zeros(sh) for _ in range(5)]
        for a in A:
            a[1:-1, 1:-1, 1:-1] = rng.uniform(0.1, 1.0, (n_,) * 3)
        kx, ky, kz, p_, r_ = A
        c = (slice(1, -1),) * 3
        nit = 10
        t0 = time.perf_counter()
        for _ in range(nit):
            w_ = np.zeros(sh)
            w_[c] = ((1.0 + rxyz * (kz[2:, 1:-1, 1:-1] + kz[c] + ky[1:-1, 2:, 1:-1] + ky[c]
                                    + kx[1:-1, 1:-1, 2:] + kx[c])) * p_[c]
                     - rxyz * (kz[2:, 1:-1, 1:-1] * p_[2:, 1:-1, 1:-1] + kz[c] * p_[:-2, 1:-1, 1:-1])
                     - rxyz * (ky[1:-1, 2:, 1:-1] * p_[1:-1, 2:, 1:-1] + ky[c] * p_[1:-1, :-2, 1:-1])
                     - rxyz * (kx[1:-1, 1:-1, 2:] * p_[1:-1, 1:-1, 2:] + kx[c] * p_[1:-1, 1:-1, :-2]))
            al = np.sum(r_ * r_) / max(np.sum(p_ * w_), 1e-300)
            r_ -= al * w_
            z_ = r_ / (1.0 + 6.0 * rxyz)
            p_ = z_ + 0.5 * p_
        secs = (time.perf_counter() - t0) / nit
        line["cpu_baseline"] = {"value": n_ ** 3 / secs, "unit": "cell-iterations/s", "cores": 1, "kind": "port",
                                "sample": f"{nit} iterations of the same 7-point PCG step in numpy on a {n_}^3 sample, one core"
                                          " (no 3D reference exists)",
                                "est_time_to_solution_s": iters * cells * secs / n_ ** 3}
    return line


def reference_heat3d(args, world, rank):
    return {"impl": "reference", "unavailable": "the reference has no 3D heat solve (OPS TeaLeaf is 2D)"}


WORKLOADS = {"laplace": (bench_laplace, reference_laplace), "clover": (bench_clover, reference_clover),
             "clover3d": (bench_clover3d, reference_clover3d),
             "adi": (bench_adi, reference_adi), "tea": (bench_tea, reference_tea),
             "learned": (bench_learned, reference_tea), "mg": (bench_mg, reference_tea),
             "heat3d": (bench_heat3d, reference_heat3d)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="clover")
    ap.add_argument("--cpu-iters", type=int, default=100)
    ap.add_argument("--cpu-clover-steps", type=int, default=40,
                    help="clover/clover3d: most steps the reference arm times (it times --steps, up to this)")
    ap.add_argument("--grid", type=int, default=None, help="clover grid edge (default 3840; smaller for profiling)")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64", help="adi workload precision")
    ap.add_argument("--adi-case", choices=["cube", "batch"], default="cube", help="adi: 256^3 block or 64 uneven blocks")
    ap.add_argument("--reliable-delta", type=float, default=0.1,
                    help="tea: FP32 residual decrease between FP64 reliable updates")
    ap.add_argument("--cpu-tea-iters", type=int, default=100, help="tea: CG iterations in the CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true",
                    help="clover: skip the learned-vs-PCG heat solve comparison in the line")
    ap.add_argument("--kernel-table", action="store_true",
                    help="clover, clover3d: print the per-kernel timing table of the roofline pass on stderr")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = {"laplace": 200, "clover": 200, "clover3d": 100, "adi": 50, "tea": 3,
                      "learned": 2, "mg": 10, "heat3d": 2}.get(args.workload, 20)
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local, pg = dist_setup(args)
    ours, ref = WORKLOADS[args.workload]
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(ref(args, world, rank)), flush=True)
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
        return
    line = ours(args, world, rank, local, pg)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
