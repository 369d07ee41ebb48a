#!/usr/bin/env python3
"""Steady solves per second on the drag-curve sweep, on N GPUs.

Workload (one step): the 16 cases of the drag curve - a tangent ogive of
fineness 3 on a 4-caliber cylinder at Mach 1.5, 1.6, ..., 3.0, 160 x 80 cells
each - every case marched from the free stream by LU-SGS at CFL 5 until its
RMS density residual d(rho)/dt (the reference's densityResidualNorm, FP64) is
at most 1e-6. The cases are independent: with N GPUs every rank solves its
own copy of the sweep (weak scaling, no data-path collective).

`value` is the device time of the solves (CUDA events on the library's
stream, inputs resident in HBM, L2 flushed between steps); `e2e` is the same
throughput through the public batch API with the host-to-device upload of the
starting field and the device-to-host read of each case's drag inside the
timed region. `--impl reference` times the CPU restatement of the reference's
FP64 engine (the oracle) on the host cores instead.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "steady solves/s to RMS density residual 1e-6 (drag curve, LU-SGS CFL 5)"
UNIT = "solves/s"
TOLERANCE = 1e-6
CFL = 5.0
OMEGA = 1.5
MAX_STEPS = 20000
CHECK_EVERY = 20
# Algorithmic bytes per cell of each LU-SGS kernel launch: every array
# element a pass reads or writes, counted once (FP64 state, FP32 sweep
# records, float4 face metrics), halo re-reads not counted (the records hold
# one slot per cell, no padding).
#   residual pass, with the previous step's update applied as it reads:
#                  state 32 + dQ 16 + i-face 16 + j-face 16 + cell 8
#                  + updated state 32 + forward record 80 (residual, 1/D,
#                  west and south neighbour terms) + backward record 64
#                  (1/D, east and north neighbour terms) = 264
#   sweeps: forward  record 80 + dQ* 16 = 96
#           backward record 80 (dQ*, 1/D, two neighbour terms) + dQ 16 = 96
#   closing update, once per run of up to 16 steps: state 32 + dQ 16 + state 32 = 80
BYTES_PREPARE = 264
BYTES_SWEEP = 192
BYTES_UPDATE = 80
# FP64 operations per cell of the residual pass (DADD + DMUL + 2 DFMA,
# thread instructions counted by ncu on the drag curve's residual pass with
# the update fused in, halo cells' updates and conversions included, divided
# by its 204,800 cells: (30.11 M + 48.97 M + 2 x 106.89 M) / 204,800; the
# summary in profiles/ names the capture).
FLOPS_PREPARE = 1430


def workload_config() -> dict:
    return {
        "workload": "drag curve: tangent ogive fineness 3 + 4-caliber cylinder, "
                    "Mach 1.5..3.0 step 0.1 (16 cases), 160x80 cells each, "
                    "LU-SGS CFL 5 omega 1.5 from free stream to RMS d(rho)/dt <= 1e-6",
        "cases_per_gpu": 16,
        "grid": "160x80",
        "precision": "FP64 state and residual; FP32 metrics and LU-SGS operator",
        "l2": "flushed between timed steps (512 MiB device write)",
        "scheme": "HLLC, van Albada with scaled shared factor (MUSCL), axisymmetric",
    }


def dist_env() -> tuple[int, int, int]:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float, world: int, device: str) -> float:
    """The largest `value` over the ranks of the job; every rank calls it at
    the same point (the job's time is its slowest rank's)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_solves_per_s(world: int, cases_per_rank: int, steps: int, job_ms: float) -> float:
    """Whole-job throughput: every rank solves its own cases (weak scaling)."""
    return world * cases_per_rank * steps / (job_ms / 1000)


class Clocks:
    """nvidia-smi clock and throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def cpu_solve(cases, threads: int) -> tuple[float, list[float], list[int]]:
    """The FP64 oracle (CPU restatement of the reference engine) on the same
    cases, one case per host thread; returns (seconds, drags, steps)."""
    from oracle.oracle import OracleEuler2D, parallel_solve

    engines = []
    for c in cases:
        o = OracleEuler2D(c.config)
        o.set_uniform(c.free.state)
        engines.append(o)
    t0 = time.perf_counter()
    status, steps, res, init = parallel_solve(engines, "lusgs", TOLERANCE, MAX_STEPS, CHECK_EVERY,
                                              cfl=CFL, omega=OMEGA, relative=False, threads=threads)
    dt = time.perf_counter() - t0
    drags = [o.forebody_drag(c.free.pressure, c.free.dynamic_pressure, c.body.nose.base_radius)
             for o, c in zip(engines, cases)]
    return dt, drags, [int(s) for s in steps]


def run_reference(args, world, rank) -> None:
    if rank != 0:
        return
    from bowshock_b200.workloads import drag_sweep_cases

    cases = drag_sweep_cases()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_solve(cases, threads)
    times = []
    for _ in range(args.steps):
        dt, _, _ = cpu_solve(cases, threads)
        times.append(dt)
    total = sum(times)
    value = len(cases) * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "the full 16-case sweep per step, one case per host thread "
                                   "(C++ FP64 restatement of src/engine-cpu/euler2d.ts)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


TRAIN_MACHS = 48  # seeded Mach numbers of the drag-curve body that train the warm start


def warm_start_target(cases) -> dict:
    """The north-star comparison on the drag curve: the warm-started batch
    against the plain cold-started single-case GPU path.

    Setup, untimed: the drag curve's body at TRAIN_MACHS seeded Mach numbers
    (SplitMix64 seeds 1.., uniform in [1.5, 3.0]) is solved cold in one
    batch at 160 x 80, and the 5 x 256 network trains (3,000 Adam steps) on
    4,096 random cells of each converged field. Timed, on the 16 cases:
    (a) each case alone from the free stream, one after another - the device
    time of each solve; (b) the 16 cases in one batch from the network's
    fields - device time plus the prediction's wall time, a case whose warm
    start fails solved again from the free stream (its time added)."""
    from bowshock_b200.warmstart import solve_cases, train_on_solves, warm_solve
    from bowshock_b200.workloads import SplitMix64, ogive_case

    machs = [SplitMix64(s).uniform(1.5, 3.0) for s in range(1, TRAIN_MACHS + 1)]
    tr = train_on_solves([ogive_case(m) for m in machs], cells_per_case=4096, train_steps=3000,
                         max_steps=MAX_STEPS)
    single_ms, single_steps = [], []
    for c in cases:
        r = solve_cases([c], max_steps=MAX_STEPS)
        assert r.status[0] == 0, c.name
        single_ms.append(r.device_ms)
        single_steps.append(r.steps[0])
    warm, fell_back = warm_solve(tr.net, cases, max_steps=MAX_STEPS)
    tr.net.destroy()
    n = len(cases)
    cold_rate = n / (sum(single_ms) / 1000)
    warm_s = warm.device_ms / 1000 + warm.predict_s
    warm_rate = sum(1 for s in warm.status if s == 0) / warm_s
    return {
        "single_cold_solves_per_s": cold_rate,
        "warm_batch_solves_per_s": warm_rate,
        "ratio": warm_rate / cold_rate,
        "target_ratio": 5.0,
        "fell_back": len(fell_back),
        "fell_back_fraction": len(fell_back) / n,
        "converged": sum(1 for s in warm.status if s == 0),
        "single_cold_steps_median": int(statistics.median(single_steps)),
        "warm_steps_median": int(statistics.median(warm.steps)),
        "warm_device_ms": warm.device_ms, "predict_s": warm.predict_s,
        "single_cold_device_ms": sum(single_ms),
        "train": {"cases": len(machs), "converged": tr.solved, "samples": tr.samples,
                  "adam_steps": tr.steps, "seconds": tr.seconds, "loss_last": tr.loss_last},
        "drags": warm.drags,
    }


def run_gpu(args, world, rank, local) -> None:
    import torch
    import torch.distributed as dist

    from bowshock_b200 import _native
    from bowshock_b200.batch import CudaBatch
    from bowshock_b200.workloads import drag_sweep_cases

    torch.cuda.set_device(local)
    lib = _native.load()
    _native.check(lib.bs_set_device(local), lib)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    cases = drag_sweep_cases()
    n = len(cases)
    batch = CudaBatch([c.config for c in cases], precision=64)
    # Setup, untimed: the autotuner picks the number of lanes and the tile shape.
    batch.set_free_stream()
    batch.autotune("lusgs", 40, CFL, OMEGA)
    tuning = batch.tuning()
    flush = torch.empty(512 * 2**20 // 4, dtype=torch.int32, device=f"cuda:{local}")
    start_fields = [np.tile(np.array([c.free.state.rho, c.free.state.u, c.free.state.v,
                                      c.free.state.p]), c.config.grid.ni * c.config.grid.nj)
                    for c in cases]

    def one_step() -> tuple[float, int, list]:
        batch.set_free_stream()
        res = batch.solve("lusgs", TOLERANCE, relative=False, max_steps=MAX_STEPS,
                          check_every=CHECK_EVERY, cfl=CFL, omega=OMEGA)
        ms, launches = batch.last_solve_timing()
        return ms, launches, res

    for _ in range(args.warmup):
        one_step()
    # Timed region: device time of each solve, L2 flushed between steps.
    clocks = Clocks(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    device_ms = []
    launches = 0
    results = None
    for _ in range(args.steps):
        flush.fill_(0)
        torch.cuda.synchronize()
        ms, nl, results = one_step()
        device_ms.append(ms)
        launches += nl
    torch.cuda.synchronize()
    barrier()
    clock_info = clocks.stop()
    total_ms = max_over_ranks(sum(device_ms), world, f"cuda:{local}")
    value = job_solves_per_s(world, n, args.steps, total_ms)
    converged = all(r.status == 0 for r in results)
    steps_taken = [r.steps for r in results]

    # End to end through the public API: upload the starting field from host
    # memory, solve, read back every case's drag.
    h2d = sum(f.nbytes for f in start_fields)
    d2h = n * 8 + n * 32
    barrier()
    torch.cuda.synchronize()
    e2e_times = []
    drags = []
    for _ in range(args.steps):
        flush.fill_(0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k, f in enumerate(start_fields):
            batch.set_primitives(k, f)
        batch.solve("lusgs", TOLERANCE, relative=False, max_steps=MAX_STEPS,
                    check_every=CHECK_EVERY, cfl=CFL, omega=OMEGA)
        drags = [batch.forebody_drag(k, c.free, c.body.nose.base_radius) for k, c in enumerate(cases)]
        e2e_times.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(sum(e2e_times), world, f"cuda:{local}")
    e2e_value = job_solves_per_s(world, n, args.steps, 1000 * e2e_total)

    # Rank 0 alone (no collective follows before its line is printed).
    target = warm_start_target(cases) if rank == 0 and not args.no_target else None

    # Roofline of the dominant kernel, timed with CUDA events on the
    # library's stream over the same solve from the free stream.
    batch.set_free_stream()
    prep_ms, sweep_ms, update_ms = batch.kernel_times("lusgs", CFL, OMEGA, iterations=50)
    cells = sum(c.config.grid.ni * c.config.grid.nj for c in cases)
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    kernels = {
        "lusgs_sweep": (sweep_ms, BYTES_SWEEP * cells),
        "lusgs_prepare": (prep_ms, BYTES_PREPARE * cells),
        "lusgs_update": (update_ms, BYTES_UPDATE * cells),
    }
    dominant = max(kernels, key=lambda k: kernels[k][0])
    kms, kbytes = kernels[dominant]
    achieved = kbytes / (kms / 1000) / 1e9
    # The residual pass is FP64 arithmetic: its rate against the measured
    # FP64 FMA rate of this GPU.
    fp64 = None
    rate = C.c_double()
    rate_ms = C.c_double()
    _native.check(lib.bs_fp64_fma_rate(200000, C.byref(rate), C.byref(rate_ms)), lib)
    if FLOPS_PREPARE is not None:
        tf = FLOPS_PREPARE * cells / (prep_ms / 1000) / 1e12
        fp64 = {"kernel": "lusgs_prepare", "achieved_tflops": tf, "peak_tflops": rate.value,
                "peak_source": "measured (bs_fp64_fma_rate)", "frac": tf / rate.value,
                "flops_per_cell": FLOPS_PREPARE}
    else:
        fp64 = {"peak_tflops": rate.value, "peak_source": "measured (bs_fp64_fma_rate)"}
    # The sweep is bound by its dependent diagonal steps, not by HBM: the
    # steps of one launch (forward and backward over ni + nj - 1 diagonals
    # of the widest case) and the SM cycles each took, at the median SM clock
    # sampled during the timed region.
    g0 = cases[0].config.grid
    diag_steps = 2 * (g0.ni + g0.nj - 1)
    latency = {"kernel": "lusgs_sweep", "diagonal_steps_per_launch": diag_steps,
               "ns_per_diagonal_step": 1e6 * sweep_ms / diag_steps}
    mhz = (clock_info or {}).get("sm_mhz")
    if mhz:
        latency["cycles_per_diagonal_step"] = latency["ns_per_diagonal_step"] * mhz / 1000
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        try:
            traffic = json.loads(tfile.read_text()).get(dominant)
        except ValueError:
            traffic = None

    if rank == 0:
        cpu = None
        cd_err = None
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            sec, cpu_drags, cpu_steps = cpu_solve(cases, threads)
            cpu = {"value": n / sec, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"the full 16-case sweep once ({sum(cpu_steps)} LU-SGS steps), one "
                             "case per host thread (C++ FP64 restatement of the reference engine)"}
            cd_err = max(abs(a / b - 1) for a, b in zip(drags, cpu_drags))
            if target is not None:
                target["cd_max_rel_err_vs_fp64_oracle"] = max(
                    abs(a / b - 1) for a, b in zip(target["drags"], cpu_drags))
        if target is not None:
            del target["drags"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(), "tuning": tuning,
            "target": target,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": hbm,
                         "peak_source": peak_src, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic,
                         "kernel_ms": {k: v[0] for k, v in kernels.items()},
                         "bytes_per_cell": {"lusgs_sweep": BYTES_SWEEP, "lusgs_prepare": BYTES_PREPARE,
                                            "lusgs_update": BYTES_UPDATE},
                         "fp64": fp64, "latency": latency},
            "cpu_baseline": cpu,
            "clocks": clock_info,
            "accuracy": {"converged": converged, "lusgs_steps": steps_taken,
                         "cd_max_rel_err_vs_fp64_oracle": cd_err},
        }
        print(json.dumps(line), flush=True)
    batch.destroy()
    del flush
    if world > 1:
        dist.destroy_process_group()


def run_probe(args) -> None:
    """A few LU-SGS steps of the benchmark's batch, each kernel timed with CUDA
    events: a short command for profilers (ncu) to capture."""
    from bowshock_b200.batch import CudaBatch
    from bowshock_b200.workloads import drag_sweep_cases

    cases = drag_sweep_cases()
    batch = CudaBatch([c.config for c in cases], precision=64)
    batch.set_free_stream()
    prep, sweep, update = batch.kernel_times("lusgs", CFL, OMEGA, iterations=args.probe)
    print(json.dumps({"probe_iterations": args.probe, "lusgs_prepare_ms": prep,
                      "lusgs_sweep_ms": sweep, "lusgs_update_ms": update}), flush=True)
    batch.destroy()


def run_seeded(args) -> None:
    """The batched uneven workload: `--cases` seeded cases (nose family,
    fineness, body length, Mach number and grid level drawn from SplitMix64
    seeds; 40x20 to 320x160 cells), solved in one batch by LU-SGS CFL 5 to
    RMS d(rho)/dt <= 1e-6 within `--max-steps` steps each. `value` counts the
    converged solves per second of device time; cases that do not converge
    within the budget (the FP64 oracle does not converge on them either: the
    residual stalls near 1) use their whole budget and are listed. The
    `--check` smallest cases' drags are checked against the FP64 oracle."""
    import torch

    from bowshock_b200.batch import CudaBatch
    from bowshock_b200.workloads import seeded_cases

    torch.cuda.set_device(0)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    cases, refused = seeded_cases(args.cases, first_seed=1, threads=threads)
    grid_s = time.perf_counter() - t0
    n = len(cases)
    cells = [c.config.grid.ni * c.config.grid.nj for c in cases]
    batch = CudaBatch([c.config for c in cases], precision=64)
    batch.set_free_stream()
    batch.autotune("lusgs", 40, CFL, OMEGA)
    tuning = batch.tuning()
    flush = torch.empty(512 * 2**20 // 4, dtype=torch.int32, device="cuda:0")

    def one_step():
        """The batch from the free stream; then, with --rescue D > 0, the
        cases it did not converge solved again from the free stream by
        Anderson-accelerated steps (D differences), whose time counts too."""
        batch.set_free_stream()
        res = batch.solve("lusgs", TOLERANCE, relative=False, max_steps=args.max_steps,
                          check_every=CHECK_EVERY, cfl=CFL, omega=OMEGA)
        ms, launches = batch.last_solve_timing()
        stuck = [k for k, r in enumerate(res) if r.status != 0]
        rescued: dict[int, float] = {}
        if stuck and args.rescue > 0:
            rb = CudaBatch([cases[k].config for k in stuck], precision=64)
            try:
                rb.set_free_stream()
                rb.set_anderson(args.rescue, 30)
                rres = rb.solve("lusgs", TOLERANCE, relative=False, max_steps=args.max_steps,
                                check_every=CHECK_EVERY, cfl=CFL, omega=OMEGA)
                rms, rl = rb.last_solve_timing()
                ms += rms
                launches += rl
                for j, k in enumerate(stuck):
                    rres[j].steps += res[k].steps
                    res[k] = rres[j]
                    if rres[j].status == 0:
                        rescued[k] = rb.forebody_drag(j, cases[k].free, cases[k].body.nose.base_radius)
            finally:
                rb.destroy()
        return ms, launches, res, rescued

    for _ in range(args.warmup):
        one_step()
    clocks = Clocks(0)
    clocks.start()
    device_ms, launches, results, rescued = [], 0, None, {}
    for _ in range(args.steps):
        flush.fill_(0)
        torch.cuda.synchronize()
        ms, nl, results, rescued = one_step()
        device_ms.append(ms)
        launches += nl
    clock_info = clocks.stop()
    total_ms = sum(device_ms)
    converged = [k for k, r in enumerate(results) if r.status == 0]
    steps_taken = [results[k].steps for k in converged]
    check = None
    if args.check > 0:
        # The plain-stepping oracle cycles on the rescued cases: they are not checked.
        pick = sorted((k for k in converged if k not in rescued), key=lambda k: (cells[k], k))[: args.check]
        sec, cpu_drags, _ = cpu_solve([cases[k] for k in pick], threads)
        gpu_drags = [batch.forebody_drag(k, cases[k].free, cases[k].body.nose.base_radius) for k in pick]
        errs = [abs(g - d) / max(abs(d), 1e-12) for g, d in zip(gpu_drags, cpu_drags)]
        check = {"cases": len(pick), "cd_max_rel_err_vs_fp64_oracle": max(errs),
                 "oracle_seconds": sec, "oracle_threads": threads}
    cell_steps = sum(c * r.steps for c, r in zip(cells, results))
    print(json.dumps({
        "metric": "steady solves/s to RMS density residual 1e-6 (seeded uneven batch, LU-SGS CFL 5)",
        "value": len(converged) * args.steps / (total_ms / 1000), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{n} seeded cases (seeds 1..{args.cases}, {len(refused)} refused by "
                               "the grid generator): nose conical/tangent ogive/parabolic/ellipsoid/"
                               "Von Karman, fineness U[1,5], body length U[2,8], Mach U[1.5,5], "
                               f"ni = 40*2^k (k in 0..3), nj = ni/2, at most {args.max_steps} steps each",
                   "cells_total": sum(cells), "grid_build_s": grid_s, "tuning": batch.tuning(),
                   "l2": "flushed between timed steps (512 MiB device write)"},
        "gpu_launches": launches,
        "converged": len(converged),
        "rescued_by_anderson": len(rescued),
        "not_converged": [cases[k].name for k in range(n) if results[k].status != 0],
        "lusgs_steps_converged": {"min": min(steps_taken), "median": int(statistics.median(steps_taken)),
                                  "max": max(steps_taken)},
        "cell_steps_per_s": cell_steps * args.steps / (total_ms / 1000),
        "accuracy": check, "clocks": clock_info,
    }), flush=True)
    batch.destroy()


def run_warmstart(args) -> None:
    """The learned warm start: `--train-cases` seeded 160x80 cases are solved
    cold in one batch and their fields train the network (5 x 256 GELU, Adam,
    tcgen05 GEMMs); `--eval-cases` held-out seeds are then solved in one batch
    from the free stream and from the network's fields. One JSON line: the
    warm-started batch's solves/s, its LU-SGS steps against the cold batch's,
    the drag difference, and the plain cold single-case solve rate."""
    import torch

    from bowshock_b200.warmstart import solve_cases, train_on_solves, warm_solve
    from bowshock_b200.workloads import seeded_cases

    torch.cuda.set_device(0)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    train, _ = seeded_cases(args.train_cases, first_seed=1, threads=threads, levels=(2,))
    held, _ = seeded_cases(args.eval_cases, first_seed=1_000_001, threads=threads, levels=(2,))
    grid_s = time.perf_counter() - t0

    tr = train_on_solves(train, args.cells_per_case, args.train_steps, args.max_steps)
    net = tr.net

    t0 = time.perf_counter()
    cold = solve_cases(held, max_steps=args.max_steps)
    cold_wall_s = time.perf_counter() - t0
    good = [k for k, s in enumerate(cold.status) if s == 0]
    t0 = time.perf_counter()
    warm, fell_back = warm_solve(net, held, max_steps=args.max_steps)
    warm_wall_s = time.perf_counter() - t0
    single = solve_cases(held[good[0]:good[0] + 1], max_steps=args.max_steps)
    cd_diff = max(abs(warm.drags[k] - cold.drags[k]) / abs(cold.drags[k]) for k in good)
    n = len(held)
    print(json.dumps({
        "metric": "warm-started steady solves/s to RMS density residual 1e-6 (seeded 160x80 batch, LU-SGS CFL 5)",
        "value": sum(1 for s in warm.status if s == 0) / (warm.device_ms / 1000), "unit": UNIT,
        "n_gpus": 1, "higher_is_better": True, "dtype": "f64 solve, bf16/fp32 network", "data": "synthetic",
        "config": {"workload": f"train on {tr.solved} converged of {len(train)} seeded 160x80 cases "
                               f"({args.cells_per_case} random cells each, {tr.samples} samples), "
                               f"evaluate on {n} held-out cases ({args.eval_cases} seeds, "
                               f"{args.eval_cases - n} refused by the grid generator)",
                   "network": "5 x 256 GELU, Fourier features",
                   "train_steps": tr.steps, "batch": 16384, "grid_build_s": grid_s},
        "train": {"solve_device_ms": tr.solve_device_ms, "seconds": tr.seconds,
                  "loss_first": tr.loss_first, "loss_last": tr.loss_last},
        "cold": {"solves_per_s": len(good) / (cold.device_ms / 1000), "device_ms": cold.device_ms,
                 "wall_s": cold_wall_s,
                 "steps_median": int(statistics.median([cold.steps[k] for k in good])),
                 "steps_total": int(sum(cold.steps[k] for k in good)),
                 "initial_residual_median": float(statistics.median([cold.initial_residual[k] for k in good]))},
        "warm": {"device_ms": warm.device_ms, "wall_s_with_prediction": warm_wall_s,
                 "steps_median": int(statistics.median([warm.steps[k] for k in good])),
                 "steps_total": int(sum(warm.steps[k] for k in good)), "fell_back": len(fell_back),
                 "initial_residual_median": float(statistics.median([warm.initial_residual[k] for k in good]))},
        "step_ratio_cold_over_warm": sum(cold.steps[k] for k in good) / max(1, sum(warm.steps[k] for k in good)),
        "cd_max_rel_diff_warm_vs_cold": cd_diff,
        "single_case_cold_solves_per_s": 1000.0 / single.device_ms,
        "warm_batch_over_single_cold": (sum(1 for s in warm.status if s == 0) / (warm.device_ms / 1000))
                                       / (1000.0 / single.device_ms),
    }), flush=True)
    net.destroy()


def run_stream(args) -> None:
    """The combined warm-started stream: the network is trained as in the
    warm-start workload (`--train-cases` seeded 160x80 solves), then
    `--geometries` held-out seeded geometries, each at Mach 1.5, 2, 3 and 4
    on grids ni = 80 2^k (80x40 to 640x320, k drawn per geometry), are
    solved wave by wave within `--wave-gb` of device memory, each wave
    warm-started by the network, its grids made on the host while the wave
    before it solves. `value` counts converged solves per second of solve
    device time plus prediction wall time; beside it the fraction of warm
    starts that fell back, the algorithmic HBM rate, the drag error against
    the FP64 oracle on the `--check` smallest converged cases, and the plain
    cold single-case solve of one case per grid level."""
    import torch

    from bowshock_b200.stream import by_grid_size, plan_waves, run_stream as stream
    from bowshock_b200.warmstart import solve_cases, train_on_solves
    from bowshock_b200.workloads import seeded_cases, stream_specs

    torch.cuda.set_device(0)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    train, _ = seeded_cases(args.train_cases, first_seed=1, threads=threads, levels=(2,))
    train_grid_s = time.perf_counter() - t0
    tr = train_on_solves(train, args.cells_per_case, args.train_steps, args.max_steps)
    del train

    specs = stream_specs(args.geometries, first_seed=2_000_001)
    free_bytes, _ = torch.cuda.mem_get_info()
    budget = int(min(args.wave_gb * 2**30, 0.6 * free_bytes))
    levels = sorted({s.ni for s in specs})
    keep: set[int] = set()
    per_level: dict[int, int] = {}
    smallest = 0
    for k, s in enumerate(specs):
        if per_level.get(s.ni, 0) < 4:
            per_level[s.ni] = per_level.get(s.ni, 0) + 1
            keep.add(k)
        if s.ni == levels[0] and smallest < 4 * args.check:
            smallest += 1
            keep.add(k)
    clocks = Clocks(0)
    clocks.start()
    res = stream(tr.net, specs, budget, threads, args.stream_steps, args.warm_steps, 80, keep)
    clock_info = clocks.stop()
    tr.net.destroy()

    made = [k for k, st in enumerate(res.status) if st is not None]
    converged = [k for k in made if res.status[k] == 0]
    device_s = sum(w.device_ms for w in res.waves) / 1000
    predict_s = sum(w.predict_s for w in res.waves)
    cell_steps = sum(w.cell_steps for w in res.waves)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    hbm = cell_steps * (BYTES_PREPARE + BYTES_SWEEP + BYTES_UPDATE) / device_s / 1e9

    def q(v: list[float], f: float) -> float:
        return float(np.quantile(np.asarray(v), f)) if v else float("nan")

    by_level = {}
    for ni in levels:
        ks = [k for k in made if specs[k].ni == ni]
        ok = [res.steps[k] for k in ks if res.status[k] == 0]
        by_level[f"{ni}x{ni // 2}"] = {
            "cases": len(ks), "converged": len(ok), "fell_back": sum(1 for k in res.fell_back if specs[k].ni == ni),
            "steps_median": int(statistics.median(ok)) if ok else None, "steps_max": max(ok) if ok else None}

    check = None
    pick = [k for k in sorted(res.kept) if specs[k].ni == levels[0] and res.status[k] == 0][: args.check]
    if pick:
        sec, cpu_drags, _ = cpu_solve([res.kept[k] for k in pick], threads)
        errs = [abs(res.drags[k] - d) / max(abs(d), 1e-12) for k, d in zip(pick, cpu_drags)]
        check = {"cases": len(pick), "grid": f"{levels[0]}x{levels[0] // 2}", "median": q(errs, 0.5),
                 "p90": q(errs, 0.9), "max": max(errs), "oracle_seconds": sec, "oracle_threads": threads}

    single = {}
    for ni in levels:
        ks = [k for k in sorted(res.kept) if specs[k].ni == ni and res.status[k] == 0]
        if ks:
            one = solve_cases([res.kept[ks[0]]], max_steps=int(args.stream_steps * ni / 80))
            single[f"{ni}x{ni // 2}"] = {"device_ms": one.device_ms, "steps": one.steps[0],
                                         "converged": one.status[0] == 0}
    single_rate = (len(single) / (sum(v["device_ms"] for v in single.values()) / 1000)) if single else None
    value = len(converged) / (device_s + predict_s)
    print(json.dumps({
        "metric": "combined warm-started stream: steady solves/s to RMS density residual 1e-6 "
                  "(seeded geometries x Mach 1.5/2/3/4, 80x40..640x320, LU-SGS CFL 5)",
        "value": value, "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
        "dtype": "f64 solve, bf16/fp32 network", "data": "synthetic",
        "config": {"workload": f"{len(specs)} cases: {args.geometries} seeded geometries (seeds from 2000001) "
                               "x Mach 1.5, 2, 3, 4; nose conical/tangent ogive/parabolic/ellipsoid/Von Karman, "
                               "fineness U[1,5], body length U[2,8], ni = 80*2^k (k in 0..3 per geometry), "
                               f"nj = ni/2; waves smallest grids first; step budgets {args.warm_steps} "
                               f"(warm start) and {args.stream_steps} (from the free stream) at 80x40, "
                               "scaled with ni",
                   "cells_total": sum(s.ni * s.nj for s in specs), "waves": len(plan_waves(specs, budget, by_grid_size(specs))),
                   "wave_budget_gb": budget / 2**30,
                   "training": {"cases": args.train_cases, "converged": tr.solved, "samples": tr.samples,
                                "adam_steps": tr.steps, "seconds": tr.seconds, "loss_last": tr.loss_last,
                                "grid_build_s": train_grid_s, "solve_device_ms": tr.solve_device_ms}},
        "gpu_launches": sum(w.launches for w in res.waves),
        "converged": len(converged), "not_converged": len(made) - len(converged),
        "refused_by_grid_generator": len(specs) - len(made),
        "fell_back_fraction": len(res.fell_back) / max(1, len(made)),
        "solve_device_s": device_s, "predict_wall_s": predict_s,
        "solves_per_s_solve_only": len(converged) / device_s,
        "cell_steps": cell_steps,
        "hbm": {"achieved_gbs": hbm, "peak_gbs": hbm_peak, "frac": hbm / hbm_peak,
                "bytes_per_cell_step": BYTES_PREPARE + BYTES_SWEEP + BYTES_UPDATE,
                "peak_source": "measured" if peaks else "fallback"},
        "by_level": by_level,
        "cd_rel_err_vs_fp64_oracle": check,
        "single_case_cold": {"per_level": single, "solves_per_s": single_rate},
        "stream_over_single_cold": value / single_rate if single_rate else None,
        "wall_s": res.wall_s, "first_wave_grid_build_s": res.first_build_s,
        "waves": [w.__dict__ for w in res.waves],
        "clocks": clock_info,
    }), flush=True)


def run_fitted(args) -> None:
    """The fitted bow shock (bs_fit_*): the Mach 3, 20 deg cone on 4-caliber
    cylinder at nj = 10 refined 1, 2 and 4 times (drag against Taylor-Maccoll,
    observed order, the second-order extrapolation), and the Mach 2
    hemisphere-cylinder at nj = 20 (stagnation-point wall pressure against the
    pitot value), each settled as the reference's GPU fit settles; `value`
    counts fitted solves per second of wall time on the GPU. Beside it the
    oracle's restatement of the fitted iteration (FP64, one host thread) over
    a bounded sample of the nj = 10 cone's steps."""
    import math

    import torch

    from bowshock_b200.fitted import CudaFit, blunt_fit_problem, settle, sharp_fit_problem
    from bowshock_b200.grid import Body, Nose, NoseShape, normal_shock, taylor_maccoll
    from bowshock_b200.workloads import cone_body

    torch.cuda.set_device(0)
    exact = taylor_maccoll(3.0, 20 * math.pi / 180, 1.4).surface_pressure_coefficient
    rows, total_s, fits = [], 0.0, 0
    errors = []
    for r in (1, 2, 4):
        p = sharp_fit_problem(cone_body(20, 4.0), 3.0, nj=10, refinement=r)
        with CudaFit(p) as g:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            converged, it, speed, drag = settle(g, 60000 * r, check_every=250 * r)
            dt = time.perf_counter() - t0
        total_s += dt
        fits += 1
        errors.append(drag / exact - 1)
        rows.append({"case": f"cone 20 deg, Mach 3, refinement {r}", "cells": p.ni * p.nj, "converged": converged,
                     "steps": it, "max_speed": speed, "drag": drag, "rel_err_vs_taylor_maccoll": drag / exact - 1,
                     "wall_s": dt, "us_per_step": 1e6 * dt / max(1, it)})
    order = math.log(abs((errors[0] - errors[1]) / (errors[1] - errors[2]))) / math.log(2)
    hemi = blunt_fit_problem(Body(Nose(NoseShape("ellipsoid"), 0.5, 0.5), 4.0), 2.0, nj=20)
    with CudaFit(hemi) as g:
        t0 = time.perf_counter()
        converged, it, speed, drag = settle(g, 60000, check_every=250)
        dt = time.perf_counter() - t0
        face = g.wall_fluxes()[0]
    total_s += dt
    fits += 1
    s = normal_shock(2.0, 1.4)
    pitot = s.pressure_ratio * (1 + 0.2 * s.downstream_mach ** 2) ** 3.5
    rows.append({"case": "hemisphere-cylinder, Mach 2, nj 20", "cells": hemi.ni * hemi.nj, "converged": converged,
                 "steps": it, "max_speed": speed, "drag": drag,
                 "stagnation_pressure_rel_err_vs_pitot": (face.flux[1] * face.nx + face.flux[2] * face.ny) / pitot - 1,
                 "wall_s": dt, "us_per_step": 1e6 * dt / max(1, it)})
    from bowshock_b200.fitted import settle_many, verified_fitted_drag
    from bowshock_b200.workloads import drag_sweep_machs, ogive_body

    # The drag curve of the headline's tangent ogive, fitted: 16 Mach numbers
    # at once, one stream each, against the same fits one after another.
    curve_problems = [sharp_fit_problem(ogive_body(3.0, 4.0), m, nj=20) for m in drag_sweep_machs()]
    curve_fits = [CudaFit(p) for p in curve_problems]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    outs = settle_many(curve_fits, 60000, check_every=250)
    concurrent_s = time.perf_counter() - t0
    for f in curve_fits:
        f.destroy()
    one = CudaFit(curve_problems[0])
    t0 = time.perf_counter()
    settle(one, 60000, check_every=250)
    single_s = time.perf_counter() - t0
    one.destroy()
    curve = {"case": "tangent ogive fineness 3 + 4-caliber cylinder, Mach 1.5..3.0 (16), nj 20",
             "cells": curve_problems[0].ni * curve_problems[0].nj, "converged": sum(1 for o in outs if o[0]),
             "wall_s": concurrent_s, "solves_per_s": len(outs) / concurrent_s,
             "single_first_case_wall_s": single_s, "steps": [o[1] for o in outs],
             "drags": [o[3] for o in outs]}

    t0 = time.perf_counter()
    vf = verified_fitted_drag(cone_body(20, 4.0), 3.0, tolerance=1e-4, max_refinement=8)
    vdt = time.perf_counter() - t0
    verified = {"case": "cone 20 deg, Mach 3, base nj 20", "kind": vf.kind, "wall_s": vdt}
    if vf.result is not None:
        v = vf.result
        verified.update({"value": v.estimate.value, "band": v.uncertainty, "verified": v.verified,
                         "extrapolated": v.estimate.extrapolated, "order": v.estimate.order,
                         "exact_taylor_maccoll": exact, "exact_inside_band": abs(v.estimate.value - exact) <= v.uncertainty,
                         "levels": [{"refinement": rep.refinement, "cells": rep.ni * rep.nj, "steps": rep.iterations,
                                     "drag": rep.drag} for rep in vf.reports]})
    t0 = time.perf_counter()
    vb = verified_fitted_drag(Body(Nose(NoseShape("ellipsoid"), 0.5, 0.5), 4.0), 2.0, tolerance=1e-4,
                              max_refinement=8)
    verified_blunt = {"case": "hemisphere-cylinder, Mach 2, base nj 20", "kind": vb.kind,
                      "wall_s": time.perf_counter() - t0}
    if vb.result is not None:
        v = vb.result
        verified_blunt.update({"value": v.estimate.value, "band": v.uncertainty, "verified": v.verified,
                               "extrapolated": v.estimate.extrapolated, "order": v.estimate.order,
                               "levels": [{"refinement": rep.refinement, "cells": rep.ni * rep.nj,
                                           "steps": rep.iterations, "drag": rep.drag} for rep in vb.reports]})
    # A two-scale nose: the 1-caliber Von Karman nose with a caliber of body at
    # Mach 2 (the reference measured its fitted drags 0.42909806331 on nj = 20
    # and 0.42869653926 on nj = 40, tests/analysis/two-scale-fit.test.ts:29).
    t0 = time.perf_counter()
    vk = verified_fitted_drag(Body(Nose(NoseShape("haack", 0.0), 1.0, 0.5), 1.0), 2.0, tolerance=1e-3,
                              max_refinement=8)
    verified_two_scale = {"case": "Von Karman nose 1 caliber + 1 caliber of body, Mach 2, base nj 20",
                          "kind": vk.kind, "wall_s": time.perf_counter() - t0, "allowance": vk.floor,
                          "reference_drags_nj20_nj40": [0.42909806331220435, 0.42869653925562817]}
    if vk.result is not None:
        v = vk.result
        verified_two_scale.update({"value": v.estimate.value, "band": v.uncertainty, "verified": v.verified,
                                   "extrapolated": v.estimate.extrapolated, "order": v.estimate.order,
                                   "levels": [{"refinement": rep.refinement, "cells": rep.ni * rep.nj,
                                               "steps": rep.iterations, "drag": rep.drag} for rep in vk.reports]})
    cpu = None
    if not args.no_cpu_baseline:
        from oracle.shock_fitting import fit_shock

        p = sharp_fit_problem(cone_body(20, 4.0), 3.0, nj=10)
        sample = 400
        t0 = time.perf_counter()
        fit_shock(p, sample)
        sec = time.perf_counter() - t0
        cpu = {"value": sample / sec, "unit": "fitted steps/s", "cores": 1, "kind": "port",
               "sample": f"{sample} fitted steps of the nj = 10 cone (1,890 cells) by oracle/shock_fitting.py, "
                         "a Python-driven restatement on the FP64 oracle",
               "gpu_steps_per_s": rows[0]["steps"] / rows[0]["wall_s"]}
    print(json.dumps({
        "metric": "fitted bow-shock solves/s (drag settled, shock at rest), one case at a time",
        "value": fits / total_s, "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "cone 20 deg Mach 3 on 4-caliber cylinder at nj = 10, refined 1, 2, 4; "
                               "hemisphere-cylinder Mach 2 at nj = 20; SSP-RK2 CFL 0.8 local steps, HLLC, "
                               "van Albada (shared scaled), axisymmetric"},
        "fits": rows, "observed_order": order, "verified_fitted_drag": verified, "verified_fitted_drag_blunt": verified_blunt,
        "verified_fitted_drag_two_scale": verified_two_scale,
        "fitted_drag_curve": curve,
        "extrapolated_rel_err": errors[2] - (errors[1] - errors[2]) / 3,
        "cpu_baseline": cpu,
    }), flush=True)


def run_gemm(args) -> None:
    """Throughput of the warm-start network's tensor-core GEMM (tcgen05, bf16
    in, FP32 accumulate) on the network's layer shapes at large batches."""
    import ctypes as C

    import torch

    from bowshock_b200 import _native

    lib = _native.load()
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("bf16_tflops", 1590.0)
    rows = []
    for m, n, k in [(16384, 256, 256), (65536, 256, 256), (131072, 256, 256), (16384, 256, 4096),
                    (8192, 8192, 8192)]:
        a = torch.randn(m, k, device="cuda").to(torch.bfloat16)
        b = torch.randn(n, k, device="cuda").to(torch.bfloat16)
        c = torch.empty(m, n, device="cuda")
        ms = C.c_float()
        _native.check(lib.bs_gemm_bf16_time(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, n, k, 20, C.byref(ms)), lib)
        tf = 2.0 * m * n * k / (ms.value / 1000) / 1e12
        rows.append({"m": m, "n": n, "k": k, "ms": ms.value, "tflops": tf, "frac_of_measured_peak": tf / peak})
        del a, b, c
    print(json.dumps({"gemm": rows, "peak_tflops": peak, "peak_source": "measured" if peaks else "fallback"}),
          flush=True)


def run_stencil(args) -> None:
    """HBM throughput of the stencil kernels on a batch larger than L2:
    `--cases` copies of a 640x320 case (a 15 deg cone, explicit SSP-RK3 stages;
    the fineness-3 ogive, LU-SGS passes), each kernel timed with CUDA events
    over 20 launches against the algorithmic bytes per cell each kernel must
    move (BYTES_PREPARE, BYTES_SWEEP, BYTES_UPDATE and the stage figures)."""
    from bowshock_b200.batch import CudaBatch
    from bowshock_b200.workloads import cone_case, ogive_case

    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    n = args.stencil_cases
    out = {"cases": n, "grid": "640x320", "peak_gbs": peak, "peak_source": "measured" if peaks else "fallback"}
    cone = cone_case(640, 320)
    ogive = ogive_case(2.0, 640, 320)
    cells = 640 * 320 * n
    for name, case, method, kinds in (
            ("explicit", cone, "explicit", (("ssprk3_stage1", 108), ("ssprk3_stage2", 140))),
            ("lusgs", ogive, "lusgs", (("lusgs_prepare", BYTES_PREPARE), ("lusgs_sweep", BYTES_SWEEP),
                                       ("lusgs_update", BYTES_UPDATE)))):
        batch = CudaBatch([case.config] * n, precision=64)
        batch.set_free_stream()
        batch.kernel_times(method, CFL, OMEGA, iterations=3)
        ms = batch.kernel_times(method, CFL, OMEGA, iterations=20)
        for (kind, bytes_per_cell), t in zip(kinds, ms):
            gbs = bytes_per_cell * cells / (t / 1000) / 1e9
            out[kind] = {"ms": t, "bytes_per_cell": bytes_per_cell, "gbs": gbs, "frac_of_peak": gbs / peak}
        batch.destroy()
    print(json.dumps(out), flush=True)


def run_transonic(args) -> None:
    """Transonic flow (bowshock_b200.transonic): the 7 deg cone of NACA TN 4233
    (half-angle 6 deg 59 min) at Mach 1.2 in its far-field domain (100 radii,
    10 calibers of cylinder), LU-SGS at a CFL number ramped to 1000 with
    Anderson acceleration (depth 8 after 200 plain steps) and two-float
    metrics, on the base grid and two refinements, each finer grid started
    from the coarser solution, until the drag settles within 1e-7; `value`
    counts settled grids per second of wall time on the GPU. Beside it the
    oracle's FP64 restatement of the same steps on the base grid, one host
    thread."""
    import math

    import torch

    from bowshock_b200.grid import Body, Nose, NoseShape, taylor_maccoll
    from bowshock_b200.transonic import solve_transonic, transonic_problem

    torch.cuda.set_device(0)
    half = (6 + 59 / 60) * math.pi / 180
    cone = Body(Nose(NoseShape("conical"), 1 / math.tan(half), 1.0), 0.0)
    # The reference's FP64 CPU engine (tests/analysis/transonic-flow.test.ts:16-19).
    measured = (0.0832184, 0.0830547, 0.0830207)
    exact = taylor_maccoll(1.2, half, 1.4).surface_pressure_coefficient
    problems = [transonic_problem(cone, 1.2, refinement=r) for r in (1, 2, 4)]

    def family():
        rows, previous = [], None
        for k, p in enumerate(problems):
            t1 = time.perf_counter()
            out = solve_transonic(p, max_steps=4000 * p.refinement,
                                  known_rate=previous[1].rate if previous else math.nan,
                                  start=(previous[0], previous[1].primitives) if previous else None)
            rows.append({"refinement": p.refinement, "cells": p.grid.grid.ni * p.grid.grid.nj, "steps": out.steps,
                         "converged": out.converged, "wall_s": time.perf_counter() - t1, "drag": out.drag,
                         "reference_drag": measured[k], "abs_diff_vs_reference": out.drag - measured[k]})
            previous = (p, out)
        return rows

    family()      # warm-up: the library and each grid size's first use
    clocks = Clocks(0)
    clocks.start()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rows = family()
    wall = time.perf_counter() - t0
    clock_info = clocks.stop()
    from oracle.transonic import solve_transonic as oracle_solve

    t1 = time.perf_counter()
    ora = oracle_solve(problems[0])
    cpu_s = time.perf_counter() - t1
    print(json.dumps({
        "metric": "transonic solves/s (drag settled within 1e-7)", "value": len(problems) / wall, "unit": "solves/s",
        "n_gpus": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "7 deg cone (TN 4233) at Mach 1.2, far field 100 radii, 10 calibers of cylinder; "
                               "transonic H grids refined 1, 2, 4; LU-SGS CFL 1 x1.2 to 1000, Anderson depth 8 "
                               "after 200 plain steps; two-float metrics"},
        "wall_s": wall, "grids": rows, "taylor_maccoll": exact, "clocks": clock_info,
        "cpu_baseline": {"value": 1 / cpu_s, "unit": "solves/s", "cores": 1, "kind": "port",
                         "sample": f"the base grid solved by oracle/transonic.py (FP64, Python-driven): "
                                   f"{ora.steps} steps in {cpu_s:.2f} s, drag {ora.drag:.10f}",
                         "gpu_base_grid_s": rows[0]["wall_s"]}}), flush=True)


def run_verified(args) -> None:
    """Verified forebody drag (the reference's banded answer) for several
    bodies and Mach numbers at once: grid families nj = 20 .. 160, each grid
    iterated until its drag settles, one refinement level of every case per
    GPU batch; the error band from the grid convergence index plus the
    captured-shock floor (1e-3 of the value)."""
    import math

    import torch

    from bowshock_b200.verified_drag import DRAG_FLOOR, verified_forebody_drags
    from bowshock_b200.workloads import cone_body, ogive_body

    torch.cuda.set_device(0)
    cases = [(cone_body(20, 4.0), m) for m in (2.0, 2.5, 3.0, 3.5, 4.0)] + \
            [(ogive_body(3.0, 4.0), m) for m in (2.0, 2.5, 3.0)]
    names = [f"cone20-cyl4-M{m}" for m in (2.0, 2.5, 3.0, 3.5, 4.0)] + \
            [f"ogive3-cyl4-M{m}" for m in (2.0, 2.5, 3.0)]
    t0 = time.perf_counter()
    out = verified_forebody_drags(cases, tolerance=args.band, max_refinement=8)
    wall = time.perf_counter() - t0
    rows = []
    for name, o in zip(names, out):
        row = {"case": name, "kind": o.kind}
        if o.result is not None:
            e = o.result.estimate
            row.update({"levels": [round(v, 10) for _, v in o.result.levels], "estimate": e.kind,
                        "value": e.value, "extrapolated": e.extrapolated, "order": e.order,
                        "band": o.result.uncertainty, "verified": o.result.verified,
                        "iterations": [r.iterations for r in o.reports]})
        else:
            row["reason"] = o.reason
        rows.append(row)
    print(json.dumps({"metric": "verified forebody drags (banded) per second", "value": len(cases) / wall,
                      "unit": "cases/s", "wall_s": wall, "tolerance_abs": args.band, "floor_rel": DRAG_FLOOR,
                      "cases": rows}), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-target", action="store_true",
                    help="drag curve: leave out the warm-started batch against the single-case cold path")
    ap.add_argument("--probe", type=int, default=0,
                    help="run this many LU-SGS steps of the batch with per-kernel timing and exit")
    ap.add_argument("--workload", choices=["drag-curve", "seeded", "warmstart", "stream", "fitted", "gemm", "stencil", "verified",
                                                  "transonic"], default="drag-curve")
    ap.add_argument("--train-cases", type=int, default=4096, help="warm start: training seeds")
    ap.add_argument("--eval-cases", type=int, default=512, help="warm start: held-out seeds")
    ap.add_argument("--train-steps", type=int, default=3000, help="warm start: Adam steps")
    ap.add_argument("--cells-per-case", type=int, default=4096, help="warm start: cells sampled per case")
    ap.add_argument("--cases", type=int, default=2048, help="seeded workload: cases drawn")
    ap.add_argument("--stencil-cases", type=int, default=32, help="stencil workload: 640x320 cases")
    ap.add_argument("--band", type=float, default=2e-3, help="verified workload: largest band, absolute")
    ap.add_argument("--max-steps", type=int, default=5000, help="seeded workload: steps per case")
    ap.add_argument("--geometries", type=int, default=2000, help="stream: seeded geometries (4 Mach numbers each)")
    ap.add_argument("--wave-gb", type=float, default=48.0, help="stream: device memory per wave")
    ap.add_argument("--warm-steps", type=int, default=1250,
                    help="stream: steps before a warm start falls back, at 80x40 (scaled with ni)")
    ap.add_argument("--stream-steps", type=int, default=2500,
                    help="stream: steps from the free stream, at 80x40 (scaled with ni)")
    ap.add_argument("--rescue", type=int, default=0,
                    help="seeded workload: Anderson depth for the cases plain LU-SGS does not converge (0: none)")
    ap.add_argument("--check", type=int, default=16,
                    help="seeded workload: smallest converged cases checked against the FP64 oracle")
    args = ap.parse_args()
    world, rank, local = dist_env()
    if args.probe > 0:
        run_probe(args)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "seeded":
        run_seeded(args)
        return
    if args.workload == "warmstart":
        run_warmstart(args)
        return
    if args.workload == "stream":
        run_stream(args)
        return
    if args.workload == "fitted":
        run_fitted(args)
        return
    if args.workload == "gemm":
        run_gemm(args)
        return
    if args.workload == "stencil":
        run_stencil(args)
        return
    if args.workload == "transonic":
        run_transonic(args)
        return
    if args.workload == "verified":
        run_verified(args)
        return
    run_gpu(args, world, rank, local)


if __name__ == "__main__":
    main()
