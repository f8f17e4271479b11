#!/usr/bin/env python
"""D3Q19 lattice-Boltzmann throughput on one or more B200s.

Workload (the headline configuration): channel flow past 40 random spheres,
256 x 128 x 128 cells, tau = 0.56, uniform inflow u_x = 0.04 at x = 0,
zero-gradient outflow at x = nx-1, periodic y/z, sphere radii U[4, 10],
centres in the middle 60 % of x, seed 42, uint8 flag grid.  A step is one
lattice update of every cell (one fused stream + boundary + collide kernel).
The headline arm stores populations in f32; the same run is repeated with
f16 / bf16 deviation storage and with the f64 build, and each storage's
velocity error after the timed steps is stated against the f64 run.

value     whole-job GLUPS (cells x steps / s, summed over ranks), populations
          resident in HBM; CUDA events on the launching stream.
e2e       the same metric through the public API with host buffers: upload of
          the initial populations (pinned) and the flag grid, the steps with
          per-step FP64 mass/momentum sums returned to the host, and the final
          rho/u read back.
roofline  algorithmic bytes per cell update (f32: 19*4*2 + 1 = 153 B) x cells
          / average kernel time, against the measured HBM copy bandwidth.

--impl reference times the reference's CPU algorithm (the f64 CPU oracle that
reproduces it bit-exactly, all host threads) on a bounded sample.
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
from datetime import timedelta
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for _p in (ROOT / "bit-physics_b200", ROOT / "oracle"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

import numpy as np  # noqa: E402

METRIC = "D3Q19 GLUPS + %HBM peak: FP32 vs FP16-store at stated err; adjoint/fwd time"
SHAPE = (256, 128, 128)
TAU = 0.56
INFLOW_U = 0.04
N_SPHERES = 40
RADIUS = (4.0, 10.0)
SEED = 42
WORKLOAD = (
    f"sphere-channel {SHAPE[0]}x{SHAPE[1]}x{SHAPE[2]}, {N_SPHERES} spheres r~U[4,10] seed {SEED}, "
    f"tau {TAU}, inflow u_x {INFLOW_U}, zero-gradient outflow, periodic y/z"
)
# Algorithmic bytes per cell update: read + write 19 populations, 1 flag byte.
BYTES_PER_CELL = {"f64": 19 * 8 * 2 + 1, "f32": 19 * 4 * 2 + 1, "f16": 19 * 2 * 2 + 1, "bf16": 19 * 2 * 2 + 1}
FALLBACK_HBM_GBS = 6650.0
PROFILE_SUMMARY = ROOT / "profiles" / "step_kernels_sphere_channel.md"


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_cell(storage: str):
    """DRAM bytes per cell update of the step kernel from the committed ncu
    summary (lines 'TRAFFIC <storage> <bytes_per_cell>'), or None."""
    try:
        for line in PROFILE_SUMMARY.read_text().splitlines():
            parts = line.strip().strip("`").split()
            if len(parts) == 3 and parts[0] == "TRAFFIC" and parts[1] == storage:
                return float(parts[2])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi samples (100 ms) of the SM clock and throttle reasons; each
    row carries nvidia-smi's own timestamp and the GPU's UUID."""

    FIELDS = ("timestamp,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.rows: list[list[str]] = []
        self.proc = None
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    @staticmethod
    def _epoch(ts: str):
        from datetime import datetime

        try:
            return datetime.strptime(ts, "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def summary(self, t0: float, t1: float):
        rows = [r for r in self.rows if len(r) == 9]
        if self.uuid:
            mine = [r for r in rows if r[1] == self.uuid]
            rows = mine or rows
        inside = [r for r in rows if (e := self._epoch(r[0])) is not None and t0 - 0.05 <= e <= t1 + 0.05]
        window = "timed region"
        if not inside:
            inside = [r for r in rows if (e := self._epoch(r[0])) is not None and e <= t1 + 0.05][-3:]
            window = "last samples before the end of the timed region"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "window": "none"}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        reasons = sorted({self.REASONS[k] for r in inside for k in range(4) if r[5 + k].lower() == "active"})
        sm = [v for r in inside if (v := num(r[2])) is not None]
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": num(inside[0][3]),
            "power_w_max": max((num(r[4]) or 0.0) for r in inside),
            "reasons": reasons,
            "samples": len(inside),
            "window": window,
        }


class NvmlClock:
    """Fast in-process SM-clock sampler (NVML, ~1 ms period) for the short
    timed repeats that nvidia-smi's 100 ms rows cannot resolve.  samples()
    returns the SM clocks (MHz) read between two perf_counter instants."""

    def __init__(self, uuid: str | None, device_index: int):
        self.rows: list[tuple[float, int]] = []
        self.on = False
        self.stop_flag = False
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            # NVML numbers GPUs physically; the UUID names the one torch uses
            self.h = (pynvml.nvmlDeviceGetHandleByUUID(uuid) if uuid
                      else pynvml.nvmlDeviceGetHandleByIndex(device_index))
        except Exception:
            self.nv = None
            return
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        while not self.stop_flag:
            if self.on:
                try:
                    mhz = self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)
                    self.rows.append((time.perf_counter(), int(mhz)))
                except Exception:
                    pass
                time.sleep(0.001)
            else:
                time.sleep(0.005)

    def samples(self, t0: float, t1: float) -> list[int]:
        return [m for (t, m) in list(self.rows) if t0 <= t <= t1]

    def stop(self):
        self.stop_flag = True


def channel_geometry():
    from lattice_boltzmann_d3q19_b200 import geometry

    flags, _ = geometry.sphere_channel(SHAPE, n_spheres=N_SPHERES, radius=RADIUS, seed=SEED)
    return flags


CELLS_PER_THREAD = 0  # 0: the library's choice
STAGING = "auto"


def step_kernel(storage: str) -> str:
    """Name of the step kernel a lattice of the headline shape runs."""
    if STAGING == "tma" and storage != "f64":
        return f"k_step_tma<{storage}>"
    if STAGING == "pipelined" and storage in ("f16", "bf16") and CELLS_PER_THREAD in (0, 2):
        return f"k_step2_pipe<{storage}>"
    cpt = CELLS_PER_THREAD or (1 if storage == "f64" else (4 if storage in ("f16", "bf16") else 2))
    return f"{ {1: 'k_step', 2: 'k_step2', 4: 'k_step4'}[cpt] }<{storage}>"


def make_lattice(storage: str, flags, device: int):
    from lattice_boltzmann_d3q19_b200 import Lattice

    # the TMA-staged kernel serves the f32-arithmetic storages, the pipelined
    # one the 16-bit storages
    staging = STAGING
    if storage == "f64" or (STAGING == "pipelined" and storage not in ("f16", "bf16")):
        staging = "auto"
    lat = Lattice(SHAPE, TAU, storage=storage, inflow_u=(INFLOW_U, 0.0, 0.0), device=device,
                  cells_per_thread=CELLS_PER_THREAD, staging=staging)
    lat.set_flags(flags)
    lat.set_equilibrium(1.0, (INFLOW_U, 0.0, 0.0))
    return lat


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: the f64 CPU oracle on a bounded sample
# ---------------------------------------------------------------------------
def cpu_reference_rate(flags, budget_s: float, max_steps: int, warmup: int = 1):
    import oracle as O

    threads = O.num_threads()
    lat = O.OracleLattice(SHAPE, TAU, flags=flags, inflow_u=(INFLOW_U, 0.0, 0.0))
    u0 = np.zeros((3, *SHAPE))
    u0[0] = INFLOW_U
    lat.set_populations(O.feq_field(np.ones(SHAPE), u0))
    del u0
    warmup = max(1, int(warmup))
    t = time.perf_counter()
    lat.step(warmup)
    first = (time.perf_counter() - t) / warmup
    steps = int(max(1, min(max_steps, budget_s / max(first, 1e-6))))
    t = time.perf_counter()
    lat.step(steps)
    dt = time.perf_counter() - t
    n = SHAPE[0] * SHAPE[1] * SHAPE[2]
    rate = n * steps / dt / 1e9
    sample = (f"{steps} steps (after {warmup} warm-up step{'s' if warmup > 1 else ''}) of the "
              f"{SHAPE[0]}x{SHAPE[1]}x{SHAPE[2]} sphere "
              f"channel, f64 CPU oracle (reference operation order), OpenMP")
    return rate, threads, steps, dt, sample


def run_reference(args, rank: int):
    if rank != 0:
        return
    flags = channel_geometry()
    budget = float(os.environ.get("LBM_REF_BUDGET_S", "30"))
    rate, cores, steps, dt, sample = cpu_reference_rate(flags, budget, max(1, args.steps), args.warmup)
    line = {
        "metric": METRIC,
        "value": rate,
        "unit": "GLUPS",
        "impl": "reference",
        "n_gpus": args.gpus,
        "steps": steps,
        "warmup": max(1, args.warmup),
        "ms_per_step": dt / steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": int(np.prod(SHAPE)), "storage": "f64",
                   "requested_steps": args.steps},
        "cpu_baseline": {"value": rate, "unit": "GLUPS", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
REPEATS = 5          # timed repeats of the requested step count per arm
PRECISION_STEPS = 5000
PRECISION_TAUS = (0.51, 0.56, 0.8)


def timed_steps(lat, steps: int, stream, torch, dist_on: bool):
    """One timed region: exactly `steps` steps bracketed by a barrier and a
    device synchronisation on both sides; CUDA events on the launching stream."""
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    if dist_on:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.time()
    p0 = time.perf_counter()
    start.record(stream)
    lat.step(steps)
    end.record(stream)
    torch.cuda.synchronize()
    t1 = time.time()
    p1 = time.perf_counter()
    if dist_on:
        torch.distributed.barrier()
    return start.elapsed_time(end), t0, t1, p0, p1


def timed_repeats(lat, steps: int, repeats: int, stream, torch, dist_on: bool, nvml):
    """`repeats` timed regions of `steps` steps each; per repeat its device
    milliseconds, wall interval and the median SM clock NVML saw inside it."""
    if nvml is not None:
        nvml.on = True
    reps = []
    for _ in range(repeats):
        ms, t0, t1, p0, p1 = timed_steps(lat, steps, stream, torch, dist_on)
        mhz = nvml.samples(p0, p1) if nvml is not None else []
        reps.append({"ms": ms, "t0": t0, "t1": t1,
                     "sm_mhz": statistics.median(mhz) if mhz else None, "clock_samples": len(mhz)})
    if nvml is not None:
        nvml.on = False
    return reps


def median_ms(reps) -> float:
    return statistics.median(r["ms"] for r in reps)


def public_reps(reps):
    return [{"ms": r["ms"], "sm_mhz": r["sm_mhz"], "clock_samples": r["clock_samples"]} for r in reps]


def precision_leg(torch, shape_name: str, dev: int):
    """Velocity / density error of each storage against the f64 build of the
    same kernels after PRECISION_STEPS steps from the inflow equilibrium, at
    tau in PRECISION_TAUS, plus the FP64 mass change of each run.  Errors over
    fluid cells, computed on the device: u L2-relative (norm of the error
    field over norm of the f64 field) and max-relative (max error magnitude
    over max f64 speed); rho L2-relative and max-abs."""
    from lattice_boltzmann_d3q19_b200 import Lattice

    shape = {"c3": (512, 256, 256), "c2": SHAPE}[shape_name]
    flags = channel_flags(shape, shape[0] / SHAPE[0])
    n = int(np.prod(shape))
    fluid = torch.from_numpy(flags != 1).to(f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)
    out = {"steps": PRECISION_STEPS, "shape": list(shape),
           "geometry": "sphere channel" + (" scaled x2 (radii U[8,20])" if shape_name == "c3" else ""),
           "reference": "f64 GPU build of the same kernels, same steps", "taus": {}}
    for tau in PRECISION_TAUS:
        row, ref = {}, None
        for storage in ("f64", "f32", "f16", "bf16"):
            lat = Lattice(shape, tau, storage=storage, inflow_u=(INFLOW_U, 0.0, 0.0), device=dev)
            lat.set_stream(stream.cuda_stream)
            lat.set_flags(flags)
            lat.set_equilibrium(1.0, (INFLOW_U, 0.0, 0.0))
            m0 = lat.conservation()[0]
            ms = _device_time(lambda: lat.step(PRECISION_STEPS), torch, stream)
            m1 = lat.conservation()[0]
            healthy = lat.check_health()
            rho = torch.empty(shape, dtype=torch.float64, device=f"cuda:{dev}")
            u = torch.empty((3, *shape), dtype=torch.float64, device=f"cuda:{dev}")
            lat.rho_u_device(rho.data_ptr(), u.data_ptr())
            torch.cuda.synchronize()
            lat.close()
            entry = {"glups": n * PRECISION_STEPS / (ms / 1e3) / 1e9, "healthy": healthy,
                     "mass_change_rel": float((m1 - m0) / m0)}
            if storage == "f64":
                ref = (rho, u)
            else:
                rr, ur = ref
                du = (u - ur)[:, fluid]
                urf = ur[:, fluid]
                dmag = torch.sqrt((du * du).sum(0))
                umax = torch.sqrt((urf * urf).sum(0)).max()
                dr = (rho - rr)[fluid]
                entry.update({
                    "u_err_l2_rel": float(torch.linalg.vector_norm(du) / torch.linalg.vector_norm(urf)),
                    "u_err_max_rel": float(dmag.max() / umax),
                    "rho_err_l2_rel": float(torch.linalg.vector_norm(dr) / torch.linalg.vector_norm(rr[fluid])),
                    "rho_err_max_abs": float(dr.abs().max()),
                })
                del du, urf, dmag, dr
            row[storage] = entry
            del rho, u
        del ref
        out["taus"][str(tau)] = row
    return out


def adjoint_leg(torch, dev: int):
    """Backward / forward time of the 128^3 FP32 porosity-drag channel over
    2000 steps with checkpoints every 50 steps (the adjoint workload's
    timing, without its gradient check)."""
    from lattice_boltzmann_d3q19_b200 import geometry

    shape = adjoint_shape()
    steps = int(os.environ.get("LBM_ADJ_STEPS", ADJ_STEPS))
    alpha = geometry.smooth_porosity(shape, sigma=4.0, seed=SEED)
    stream = torch.cuda.Stream(device=dev)
    box = (3 * shape[0] // 4, shape[0])
    with torch.cuda.stream(stream):
        lat = adjoint_lattice("f32", alpha)
        lat.set_stream(stream.cuda_stream)
        lat.set_equilibrium()
        lat.step(3)
        lat.set_equilibrium()
        t_fwd = _device_time(lambda: lat.step(steps), torch, stream)
        lat.set_equilibrium()
        holder = {}
        t_tape = _device_time(lambda: holder.update(tape=lat.tape(steps, ADJ_EVERY)), torch, stream)
        tape = holder["tape"]
        rho = torch.empty(shape, dtype=torch.float64, device="cuda")
        u = torch.empty((3, *shape), dtype=torch.float64, device="cuda")
        lat.rho_u_device(rho.data_ptr(), u.data_ptr())
        r = rho.clone().requires_grad_(True)
        v = u.clone().requires_grad_(True)
        x0, x1 = box
        L = 0.5 * (r[x0:x1] * (v[:, x0:x1] ** 2).sum(0)).sum()
        L.backward()
        ga = torch.empty(shape, dtype=torch.float64, device="cuda")
        t_bwd = _device_time(lambda: tape.backward(r.grad.data_ptr(), v.grad.data_ptr(), ga.data_ptr()), torch,
                             stream)
        finite = bool(torch.isfinite(ga).all())
        nbytes = tape.nbytes
        tape.close()
        lat.close()
    return {"value": t_bwd / t_fwd, "forward_ms": t_fwd, "taped_forward_ms": t_tape, "backward_ms": t_bwd,
            "tape_gb": nbytes / 1e9, "gradient_finite": finite,
            "config": f"{shape[0]}x{shape[1]}x{shape[2]} drag channel, f32, {steps} steps, checkpoints every "
                      f"{ADJ_EVERY}; backward = segment recompute + adjoint kernels"}


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch

    dist_on = world > 1
    torch.cuda.set_device(local_rank)  # before the process group: each rank's NCCL communicator on its own GPU
    if dist_on:
        torch.distributed.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = local_rank
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        dev_id = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
    except Exception:
        dev_id = None
    n = int(np.prod(SHAPE))
    flags = channel_geometry()
    stream = torch.cuda.Stream(device=dev)
    sampler = ClockSampler(dev_id)
    nvml = NvmlClock(dev_id, dev)
    if nvml.nv is None:
        nvml = None
    hbm, hbm_kind = peak_hbm()
    repeats = max(1, args.repeats)

    def measure(storage: str, steps: int, warmup: int, sync_ranks: bool):
        lat = make_lattice(storage, flags, dev)
        lat.set_stream(stream.cuda_stream)
        lat.step(warmup)
        reps = timed_repeats(lat, steps, repeats, stream, torch, sync_ranks, nvml)
        healthy = lat.check_health()
        lat.close()
        return reps, healthy

    # headline arm (f32), timed across ranks
    reps, healthy = measure(args.storage, args.steps, args.warmup, dist_on)
    ms = median_ms(reps)
    ms_max = ms
    if dist_on:
        t = torch.tensor([ms], device=f"cuda:{dev}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_max = float(t.item())
    clocks = sampler.summary(reps[0]["t0"], reps[-1]["t1"])
    value = world * n * args.steps / (ms_max / 1e3) / 1e9
    ms_per_step = ms_max / args.steps
    bpc = BYTES_PER_CELL[args.storage]
    achieved = n * bpc / (ms / args.steps / 1e3) / 1e9
    tr = traffic_per_cell(args.storage)
    roofline = {
        "bound": "hbm",
        "achieved": achieved,
        "peak": hbm,
        "peak_kind": hbm_kind,
        "unit": "GB/s",
        "frac": achieved / hbm,
        "traffic": None if tr is None else tr * n,
        "algorithmic_bytes_per_launch": n * bpc,
        "kernel": f"{step_kernel(args.storage)} (fused pull-stream + boundary + BGK collide)",
    }

    # storage variants at the same step count (every rank runs them; no collectives inside)
    variants = {}
    if not args.skip_variants:
        results = {args.storage: (reps, healthy)}
        for st in ("f16", "bf16", "f64"):
            if st != args.storage:
                results[st] = measure(st, args.steps, args.warmup, False)
        for st, (reps_v, healthy_v) in results.items():
            ms_v = median_ms(reps_v)
            ach = n * BYTES_PER_CELL[st] / (ms_v / args.steps / 1e3) / 1e9
            variants[st] = {"glups": n * args.steps / (ms_v / 1e3) / 1e9, "ms_per_step": ms_v / args.steps,
                            "hbm_gbs": ach, "frac": ach / hbm, "bytes_per_cell": BYTES_PER_CELL[st],
                            "kernel": step_kernel(st), "healthy": healthy_v, "repeats": public_reps(reps_v)}
        if "f16" in variants and args.storage in variants:
            variants["f16_over_f32_glups"] = variants["f16"]["glups"] / variants[args.storage]["glups"]

    # errors of the reduced-precision storages after a fixed 5000 steps
    precision = None
    if args.precision != "none":
        precision = precision_leg(torch, args.precision, dev)

    # adjoint cost relative to the forward steps
    adjoint = None
    if not args.skip_adjoint:
        adjoint = adjoint_leg(torch, dev)

    # end to end through the public API with host buffers: upload of the
    # initial rho / u fields and the flag grid, the equilibrium built on the
    # device, the steps with per-step FP64 sums to the host, rho / u read back
    e2e = None
    if not args.skip_e2e:
        from lattice_boltzmann_d3q19_b200 import Lattice

        rho0 = torch.empty(SHAPE, dtype=torch.float64, pin_memory=True).numpy()
        u0 = torch.empty((3, *SHAPE), dtype=torch.float64, pin_memory=True).numpy()
        rho0[...] = 1.0
        u0[...] = 0.0
        u0[0] = INFLOW_U
        lat = Lattice(SHAPE, TAU, storage=args.storage, inflow_u=(INFLOW_U, 0.0, 0.0), device=dev,
                      cells_per_thread=CELLS_PER_THREAD, staging=STAGING)
        lat.set_equilibrium(rho0, u0)  # allocates the upload staging outside the timed region
        rho_pinned = torch.empty(SHAPE, dtype=torch.float64, pin_memory=True).numpy()
        u_pinned = torch.empty((3, *SHAPE), dtype=torch.float64, pin_memory=True).numpy()
        torch.cuda.synchronize()
        if dist_on:
            torch.distributed.barrier()
        t = time.perf_counter()
        lat.set_flags(flags)
        lat.set_equilibrium(rho0, u0)
        sums = lat.step_monitor(args.steps)
        lat.rho_u(out=(rho_pinned, u_pinned))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        lat.close()
        if dist_on:
            tt = torch.tensor([dt], device=f"cuda:{dev}", dtype=torch.float64)
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            dt = float(tt.item())
        in_bytes = 4 * n * 8 + n  # rho, u (f64) and the flag grid
        out_bytes = 4 * n * 8     # rho and u as f64
        e2e = {
            "value": world * n * args.steps / dt / 1e9,
            "unit": "GLUPS",
            "h2d_bytes_per_step": in_bytes / args.steps,
            "d2h_bytes_per_step": (4 * 8 * args.steps + out_bytes) / args.steps,
            "what": "set_flags + set_equilibrium(rho, u) from pinned f64 host arrays (equilibrium built on the "
                    "device) + step_monitor (per-step FP64 mass/momentum sums to host) + rho_u readback into "
                    "pinned f64 arrays, wall clock",
            "mass_drift_rel": float((sums[-1, 0] - sums[0, 0]) / sums[0, 0]),
        }
    # strong scaling of the same channel by x-slabs (one slab per rank, the
    # overlapped step; one rank exchanges with itself)
    slab = None
    if not args.skip_slab:
        slab_args = argparse.Namespace(steps=min(args.steps, 1000), warmup=args.warmup)
        ms, slab_healthy, planes = slab_leg(slab_args, rank, world, local_rank, args.storage, True)
        slab = {"value": n * slab_args.steps / (ms / 1e3) / 1e9, "unit": "GLUPS", "scaling": "strong",
                "ms_per_step": ms / slab_args.steps, "steps": slab_args.steps, "slabs": world,
                "planes_per_slab": planes, "healthy": slab_healthy,
                "what": "the channel split in x over the ranks, one halo plane per side, faces exchanged by "
                        "NCCL point-to-point on a second stream while the interior planes step"}
    sampler.stop()
    if nvml is not None:
        nvml.stop()

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        rate, cores, steps, dt, sample = cpu_reference_rate(flags, float(os.environ.get("LBM_CPU_BUDGET_S", "15")),
                                                            args.steps)
        cpu = {"value": rate, "unit": "GLUPS", "cores": cores, "kind": "port", "sample": sample}
        # the same restatement on one thread (the reference's CPU path is serial)
        import oracle as O

        O.set_num_threads(1)
        try:
            r1, _, s1, _, _ = cpu_reference_rate(flags, float(os.environ.get("LBM_CPU1_BUDGET_S", "8")), args.steps)
        finally:
            O.set_num_threads(cores)
        cpu["single_thread"] = {"value": r1, "unit": "GLUPS", "cores": 1, "steps": s1}

    if dist_on:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "GLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": args.storage,
        "data": "synthetic",
        "config": {
            "workload": WORKLOAD,
            "cells": n,
            "storage": args.storage,
            "l2": f"inputs larger than L2: 2 x {19 * n * {'f64': 8, 'f32': 4}.get(args.storage, 2) / 1e6:.0f} MB "
                  f"population buffers",
            "parallelism": "replicas (one independent lattice per GPU)" if world > 1 else "single GPU",
            "timing": f"median of {repeats} timed repeats of {args.steps} steps",
        },
        "repeats": public_reps(reps),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
        "gpu_launches": args.steps,
        "healthy": healthy,
        "variants": variants,
        "precision": precision,
        "adjoint_over_forward": adjoint,
        "slab_strong_scaling": slab,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Other workloads (one JSON line each; single GPU)
# ---------------------------------------------------------------------------
def _device_time(fn, torch, stream):
    """Milliseconds of device time of fn() bracketed by events on stream."""
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    fn()
    end.record(stream)
    torch.cuda.synchronize()
    return start.elapsed_time(end)


def run_cavity(args):
    """64^3 lid-driven cavity, tau 0.6, lid (0.05, 0, 0) on y+, reference wall
    rule on all six faces, rest initial state: f32, f16 and f64 storage."""
    import torch

    import oracle as O
    from lattice_boltzmann_d3q19_b200 import Lattice, geometry

    shape, tau, steps = (64, 64, 64), 0.6, args.steps
    kw = geometry.lid_driven_cavity(0.05)
    # the reference-exact proxy: x, z periodic, walls only in y (the
    # reference's own wall rule), lid on y+
    proxy = {"periodic": (True, False, True), "wall_velocity": {"y+": (0.05, 0.0, 0.0)}}
    stream = torch.cuda.Stream()
    out, out_proxy = {}, {}
    n = int(np.prod(shape))

    def timed(storage, kwargs, staging="auto"):
        lat = Lattice(shape, tau, storage=storage, staging=staging, **kwargs)
        lat.set_stream(stream.cuda_stream)
        lat.set_equilibrium()
        lat.step(args.warmup)
        ms = _device_time(lambda: lat.step(steps), torch, stream)
        healthy = lat.check_health()
        lat.close()
        return {"glups": n * steps / (ms / 1e3) / 1e9, "ms_per_step": ms / steps, "healthy": healthy,
                "hbm_frac": n * BYTES_PER_CELL[storage] / (ms / steps / 1e3) / 1e9 / peak_hbm()[0]}

    for storage in ("f32", "f16", "f64"):
        out[storage] = timed(storage, kw)
        out[storage + "_persistent"] = timed(storage, kw, "persistent")
        out_proxy[storage] = timed(storage, proxy)
        out_proxy[storage + "_persistent"] = timed(storage, proxy, "persistent")
    cpu = O.OracleLattice(shape, tau, periodic=0, wall_velocity=Lattice._wall_array(kw["wall_velocity"]))
    cpu.set_populations(O.feq_field(np.ones(shape), np.zeros((3, *shape))))
    cpu_steps = min(steps, int(os.environ.get("LBM_CAVITY_CPU_STEPS", "200")))
    t = time.perf_counter()
    cpu.step(cpu_steps)
    dt = time.perf_counter() - t
    print(json.dumps({
        "metric": "D3Q19 GLUPS, 64^3 lid-driven cavity", "workload": "cavity", "unit": "GLUPS",
        "value": out["f32"]["glups"], "steps": steps, "warmup": args.warmup, "variants": out,
        "reference_exact_proxy": out_proxy,
        "cpu_baseline": {"value": n * cpu_steps / dt / 1e9, "unit": "GLUPS", "cores": O.num_threads(),
                         "kind": "port", "sample": f"{cpu_steps} steps of the 64^3 cavity, f64 CPU oracle"},
        "config": {"shape": shape, "tau": tau, "lid": 0.05, "walls": "all six faces, reference wall rule"},
    }), flush=True)


def channel_flags(shape, scale):
    """The headline sphere channel's geometry on another grid: radii scaled."""
    from lattice_boltzmann_d3q19_b200 import geometry

    flags, _ = geometry.sphere_channel(shape, n_spheres=N_SPHERES, radius=(RADIUS[0] * scale, RADIUS[1] * scale),
                                       seed=SEED)
    return flags


def run_sweep(args):
    """Precision sweep: the sphere channel on 512 x 256 x 256 (the headline
    geometry scaled by 2, radii U[8, 20]) at tau 0.51, 0.56 and 0.8; f32, f16
    and bf16 storage against the f64 build of the same kernels after the same
    steps (default 5000), from the inflow equilibrium.  Reports each run's
    GLUPS, its velocity error over fluid cells (L2-relative and max-relative)
    and the FP64 mass change.  LBM_SWEEP_SHAPE overrides the size."""
    import torch

    from lattice_boltzmann_d3q19_b200 import Lattice

    shape = tuple(int(v) for v in os.environ.get("LBM_SWEEP_SHAPE", "512,256,256").split(","))
    flags = channel_flags(shape, shape[0] / SHAPE[0])
    fluid = flags != 1
    n = int(np.prod(shape))
    steps = args.steps
    stream = torch.cuda.Stream()
    results = []
    for tau in (0.51, 0.56, 0.8):
        row = {"tau": tau}
        rho64 = u64 = None
        for storage in ("f64", "f32", "f16", "bf16"):
            lat = Lattice(shape, tau, storage=storage, inflow_u=(INFLOW_U, 0.0, 0.0))
            lat.set_stream(stream.cuda_stream)
            lat.set_flags(flags)
            lat.set_equilibrium(1.0, (INFLOW_U, 0.0, 0.0))
            m0 = lat.conservation()[0]
            ms = _device_time(lambda: lat.step(steps), torch, stream)
            m1 = lat.conservation()[0]
            healthy = lat.check_health()
            rho, u = lat.rho_u()
            lat.close()
            entry = {"glups": n * steps / (ms / 1e3) / 1e9, "healthy": healthy,
                     "mass_change_rel": (m1 - m0) / m0}
            if storage == "f64":
                rho64, u64 = rho, u
            else:
                du = (u - u64)[:, fluid]
                ref = u64[:, fluid]
                entry["u_err_l2_rel"] = float(np.linalg.norm(du) / np.linalg.norm(ref))
                entry["u_err_max_rel"] = float(np.abs(du).max() / np.abs(ref).max())
                dr = (rho - rho64)[fluid]
                entry["rho_err_l2_rel"] = float(np.linalg.norm(dr) / np.linalg.norm(rho64[fluid]))
                entry["rho_err_max_abs"] = float(np.abs(dr).max())
            row[storage] = entry
            del rho, u
        results.append(row)
    f16_over_f32 = [r["f16"]["glups"] / r["f32"]["glups"] for r in results]
    print(json.dumps({
        "metric": "precision sweep: GLUPS and velocity error vs the f64 build", "workload": "sweep",
        "unit": "GLUPS", "value": statistics.median(r["f16"]["glups"] for r in results), "steps": steps,
        "shape": shape, "f16_over_f32_glups": f16_over_f32, "results": results,
        "config": {"geometry": "sphere channel scaled x2 (40 spheres, r U[8,20], seed 42)",
                   "inflow_u": INFLOW_U, "initial": "inflow equilibrium"},
    }), flush=True)


def run_ensemble(args):
    """64 independent lid-driven cavities, sizes U[32,128] per axis, tau
    U[0.52,0.9], lid U[0.02,0.08] (seed 42), f16 deviation storage: one
    launch per lattice and step, one batched launch per step (default
    schedule), each lattice's own kernels on 8 parallel graph branches, and
    the autotuned schedule."""
    import torch

    from lattice_boltzmann_d3q19_b200 import Batch, geometry

    ens = geometry.cavity_ensemble(64, seed=SEED)
    specs = []
    for shape, tau, lid in ens:
        kw = geometry.lid_driven_cavity(lid)
        specs.append(dict(shape=shape, tau=tau, storage="f16", **kw))
    cells = sum(int(np.prod(s)) for s, _, _ in ens)
    out = {}
    with Batch(specs) as b:
        for k in range(len(b)):
            b[k].set_equilibrium()
        b.step(args.warmup)
        b.synchronize()

        def timed(fn):
            torch.cuda.synchronize()
            t = time.perf_counter()
            fn()
            b.synchronize()
            return time.perf_counter() - t

        dt = timed(lambda: b.step_unbatched(args.steps))
        out["per_lattice_launches"] = {"glups": cells * args.steps / dt / 1e9, "launches_per_step": len(b)}
        b.set_schedule("single", 256, 0)
        b.step(2)
        dt = timed(lambda: b.step(args.steps))
        out["batched_default"] = {"glups": cells * args.steps / dt / 1e9, "schedule": list(b.schedule()),
                                  "launches_per_step": 1}
        b.set_schedule("branches", 128, 8)
        b.step(2)
        dt = timed(lambda: b.step(args.steps))
        out["batched_branches"] = {"glups": cells * args.steps / dt / 1e9, "schedule": list(b.schedule()),
                                   "launches_per_step": "one graph of per-lattice kernels per two steps"}
        ms = b.autotune(20)
        b.step(2)
        dt = timed(lambda: b.step(args.steps))
        out["batched_autotuned"] = {"glups": cells * args.steps / dt / 1e9, "schedule": list(b.schedule()),
                                    "autotune_ms_per_step": ms, "launches_per_step": 1}
        healthy = all(b[k].check_health() for k in range(len(b)))
    print(json.dumps({"metric": "D3Q19 GLUPS, batched ensemble of 64 cavities", "workload": "ensemble",
                      "unit": "GLUPS", "value": out["batched_autotuned"]["glups"], "steps": args.steps,
                      "cells": cells, "healthy": healthy, "variants": out,
                      "speedup_autotuned_over_per_lattice": out["batched_autotuned"]["glups"]
                      / out["per_lattice_launches"]["glups"]}), flush=True)


def slab_leg(args, rank: int, world: int, local_rank: int, storage: str, overlap: bool):
    """Time args.steps steps of this rank's x-slab of the headline channel
    (after args.warmup steps): whole-slab steps after a blocking exchange, or
    the overlapped step (interior planes while the faces travel on a second
    stream).  Returns (max over ranks of the CUDA-event ms, healthy, planes
    of this slab).  With world > 1 the process group must be up."""
    import torch

    from lattice_boltzmann_d3q19_b200 import Lattice
    from lattice_boltzmann_d3q19_b200.slab import GpuEngine, SlabLattice, exchange_distributed, slab_bounds, \
        step_distributed, with_halos

    nx = SHAPE[0]
    flags = channel_geometry()
    x0, x1 = slab_bounds(nx, world)[rank]
    stream = torch.cuda.Stream()
    comm = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        lat = Lattice((x1 - x0 + 2, *SHAPE[1:]), TAU, storage=storage, inflow_u=(INFLOW_U, 0.0, 0.0),
                      device=local_rank)
        lat.set_stream(stream.cuda_stream)
        lat.set_flags(with_halos(flags, x0, x1, nx))
        lat.set_equilibrium(1.0, (INFLOW_U, 0.0, 0.0))
        slab = SlabLattice(GpuEngine(lat, storage), x0, x1, flags=flags, nx=nx)

        def advance(k):
            for _ in range(k):
                if overlap:
                    step_distributed(slab, rank, world, comm)
                    continue
                if slab.stepped:
                    exchange_distributed(slab, rank, world)
                lat.step(1)
                slab.stepped = True

        advance(max(args.warmup, 2))
        # One rank: two steps captured into a CUDA graph and replayed (the
        # enqueueing of a split step's launches from Python would otherwise
        # set the pace); several ranks step eagerly (NCCL point-to-point).
        graph = None
        if world == 1:
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=stream, capture_error_mode="relaxed"):
                advance(2)
            graph.replay()
        steps = args.steps + args.steps % 2 if graph is not None else args.steps

        def run():
            if graph is None:
                advance(steps)
            else:
                for _ in range(steps // 2):
                    graph.replay()

        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        start.record(stream)
        run()
        end.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ms = start.elapsed_time(end) * args.steps / steps
        healthy = lat.check_health()
        del graph
        lat.close()
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local_rank}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    return ms, healthy, x1 - x0


def run_slab(args, rank: int, world: int, local_rank: int):
    """x-slab strong scaling: the headline sphere channel (256 x 128 x 128)
    split in x over the ranks, one slab per GPU with a halo plane per side;
    every step exchanges 5 populations per face with its neighbours (NCCL
    point-to-point; one rank exchanges with itself).  Both step forms are
    timed; value: the overlapped one, global cells x steps / (max over ranks
    of the CUDA-event time)."""
    import torch

    dist_on = world > 1
    torch.cuda.set_device(local_rank)  # before the process group: each rank's NCCL communicator on its own GPU
    if dist_on:
        torch.distributed.init_process_group("nccl", timeout=timedelta(seconds=300))
    storage = args.storage
    n = int(np.prod(SHAPE))
    legs = {}
    for name, overlap in (("whole_slab", False), ("overlapped", True)):
        ms, healthy, planes = slab_leg(args, rank, world, local_rank, storage, overlap)
        legs[name] = {"glups": n * args.steps / (ms / 1e3) / 1e9, "ms_per_step": ms / args.steps, "healthy": healthy}
    if dist_on:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    elem = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2}[storage]
    print(json.dumps({
        "metric": "D3Q19 GLUPS, x-slab decomposition of one lattice", "workload": "slab", "unit": "GLUPS",
        "value": legs["overlapped"]["glups"], "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": legs["overlapped"]["ms_per_step"], "scaling": "strong",
        "dtype": storage, "variants": legs, "healthy": all(v["healthy"] for v in legs.values()),
        "halo_bytes_per_face_per_step": 5 * SHAPE[1] * SHAPE[2] * elem,
        "config": {"workload": WORKLOAD, "slabs": world, "planes_per_slab": planes},
    }), flush=True)


def run_moments(args):
    """The 16-bit moment-encoded state (the reference's frontier format)
    against FP16-shift storage on the headline sphere channel: per tau an f64
    run that also calibrates the 19 moment ranges over every post-collision
    state (margin 5 %), then the moment-encoded run (f32 step kernels, state
    held as 16-bit moment codes between steps) and the f16 (f - feq(1,
    u_in)) run, each against the f64 result after the same steps.  Reports
    the errors and GLUPS (the moment-encoded GLUPS include its decode and
    encode passes)."""
    import torch

    from lattice_boltzmann_d3q19_b200 import Lattice

    steps = args.steps
    flags = channel_geometry()
    fluid = flags != 1
    n = int(np.prod(SHAPE))
    stream = torch.cuda.Stream()
    rows = []
    for tau in (0.51, 0.56, 0.8):
        def lattice(storage):
            lat = Lattice(SHAPE, tau, storage=storage, inflow_u=(INFLOW_U, 0.0, 0.0))
            lat.set_stream(stream.cuda_stream)
            lat.set_flags(flags)
            lat.set_equilibrium(1.0, (INFLOW_U, 0.0, 0.0))
            return lat

        ref = lattice("f64")
        holder = {}
        t_cal = _device_time(lambda: holder.update(r=ref.moment16_calibrate(steps, 0.05)), torch, stream)
        lo, hi = holder["r"]
        _, u64 = ref.rho_u()
        ref.close()
        ref_f = u64[:, fluid]
        umax = np.sqrt((ref_f * ref_f).sum(0)).max()
        row = {"tau": tau, "calibration_ms": t_cal}
        for mode in ("moment16", "f16"):
            lat = lattice("f32" if mode == "moment16" else "f16")
            if mode == "moment16":
                ms = _device_time(lambda: lat.moment16_step(lo, hi, steps), torch, stream)
            else:
                ms = _device_time(lambda: lat.step(steps), torch, stream)
            healthy = lat.check_health()
            _, u = lat.rho_u()
            lat.close()
            du = (u - u64)[:, fluid]
            row[mode] = {"glups": n * steps / (ms / 1e3) / 1e9, "healthy": healthy,
                         "u_err_l2_rel": float(np.linalg.norm(du) / np.linalg.norm(ref_f)),
                         "u_err_max_rel": float(np.sqrt((du * du).sum(0)).max() / umax)}
        rows.append(row)
    print(json.dumps({"metric": "16-bit moment-encoded state vs FP16-shift storage", "workload": "moments",
                      "unit": "GLUPS", "value": statistics.median(r["moment16"]["glups"] for r in rows),
                      "steps": steps, "results": rows,
                      "config": {"workload": WORKLOAD, "ranges": "f64 envelope over the run, margin 5 %",
                                 "moment16_bytes_per_cell": "decode 38 + 76, step 153, encode 76 + 38"}}),
          flush=True)


ADJ_STEPS, ADJ_EVERY = 2000, 50


def adjoint_shape():
    return tuple(int(v) for v in os.environ.get("LBM_ADJ_SHAPE", "128,128,128").split(","))


def adjoint_lattice(storage: str, alpha):
    """Channel on alpha's grid (128^3): inflow u_x = 0.04 at x = 0,
    zero-gradient outflow at the last x plane, walled y (no-slip), periodic
    z, tau 0.6, porosity drag F = -beta(alpha) m with k = 0.05."""
    from lattice_boltzmann_d3q19_b200 import Lattice

    shape = alpha.shape
    flags = np.zeros(shape, np.uint8)
    flags[0] = 2
    flags[-1] = 3
    lat = Lattice(shape, 0.6, storage=storage, periodic=(True, False, True), force_mode="drag", drag_k=0.05,
                  inflow_u=(0.04, 0.0, 0.0))
    lat.set_flags(flags)
    lat.set_porosity(alpha)
    return lat


def run_adjoint(args):
    """Adjoint workload: d(kinetic energy in the last quarter of x after 2000
    steps) / d(alpha) on the 128^3 FP32 channel, alpha = Gaussian-filtered
    (sigma 4, periodic) noise in [0, 1], checkpoints every 50 steps.  Times
    the plain forward, the taped forward and the backward (segment recompute
    + adjoint kernels); checks the gradient against central differences of
    the f64 forward along 16 seeded random directions.  LBM_ADJ_SHAPE,
    LBM_ADJ_STEPS and LBM_ADJ_DIRECTIONS override the size, the step count
    and the number of directions (small cases for profiling)."""
    import torch

    from lattice_boltzmann_d3q19_b200 import geometry

    shape = adjoint_shape()
    box = (3 * shape[0] // 4, shape[0])
    steps = int(os.environ.get("LBM_ADJ_STEPS", ADJ_STEPS))
    n = int(np.prod(shape))
    alpha = geometry.smooth_porosity(shape, sigma=4.0, seed=SEED)
    stream = torch.cuda.Stream()  # torch work and the lattices share it

    def box_energy(rho, u):
        x0, x1 = box
        return 0.5 * (rho[x0:x1] * (u[:, x0:x1] ** 2).sum(0)).sum()

    def gradient(storage):
        lat = adjoint_lattice(storage, alpha)
        lat.set_stream(stream.cuda_stream)
        lat.set_equilibrium()
        lat.step(3)
        lat.set_equilibrium()
        t_fwd = _device_time(lambda: lat.step(steps), torch, stream)
        lat.set_equilibrium()
        holder = {}
        t_tape = _device_time(lambda: holder.update(tape=lat.tape(steps, ADJ_EVERY)), torch, stream)
        tape = holder["tape"]
        rho = torch.empty(shape, dtype=torch.float64, device="cuda")
        u = torch.empty((3, *shape), dtype=torch.float64, device="cuda")
        lat.rho_u_device(rho.data_ptr(), u.data_ptr())
        r = rho.clone().requires_grad_(True)
        v = u.clone().requires_grad_(True)
        L = box_energy(r, v)
        L.backward()
        ga = torch.empty(shape, dtype=torch.float64, device="cuda")
        t_bwd = _device_time(lambda: tape.backward(r.grad.data_ptr(), v.grad.data_ptr(), ga.data_ptr()), torch,
                             stream)
        out = {"loss": float(L.detach()), "forward_ms": t_fwd, "taped_forward_ms": t_tape, "backward_ms": t_bwd,
               "tape_gb": tape.nbytes / 1e9, "forward_glups": n * steps / (t_fwd / 1e3) / 1e9,
               "adjoint_over_forward": t_bwd / t_fwd, "healthy": lat.check_health()}
        tape.close()
        lat.close()
        return out, ga.cpu().numpy()

    with torch.cuda.stream(stream):
        res32, g32 = gradient("f32")
        res64, g64 = gradient("f64")
    # central differences of the f64 forward; the perturbed alpha is stored
    # as float32, so each difference is taken against the stored step
    lat = adjoint_lattice("f64", alpha)
    rng = np.random.default_rng(SEED)
    n_dir = int(os.environ.get("LBM_ADJ_DIRECTIONS", "16"))
    errs32, errs64 = [], []

    def loss_at(a):
        lat.set_porosity(a)
        lat.set_equilibrium()
        lat.step(steps)
        rho, u = lat.rho_u()
        return float(box_energy(torch.from_numpy(rho), torch.from_numpy(u)))

    for _ in range(n_dir):
        d = 1e-3 * rng.standard_normal(shape)
        ap = np.clip(alpha + d, 0, 1).astype(np.float32)
        am = np.clip(alpha - d, 0, 1).astype(np.float32)
        fd = loss_at(ap) - loss_at(am)
        delta = ap.astype(np.float64) - am.astype(np.float64)
        errs64.append(abs(float((g64 * delta).sum()) - fd) / abs(fd))
        errs32.append(abs(float((g32 * delta).sum()) - fd) / abs(fd))
    lat.close()
    rel_l2 = float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))
    print(json.dumps({
        "metric": "adjoint / forward time, FP32 porosity-drag channel", "workload": "adjoint",
        "unit": "ratio", "value": res32["adjoint_over_forward"], "higher_is_better": False, "steps": steps,
        "checkpoint_every": ADJ_EVERY, "f32": res32, "f64": res64,
        "gradient_check": {"directions": n_dir, "per_cell_step": 1e-3, "fd_kind": "central, f64 forward",
                           "max_rel_err_f32_adjoint": max(errs32, default=None),
                           "max_rel_err_f64_adjoint": max(errs64, default=None),
                           "f32_vs_f64_gradient_rel_l2": rel_l2},
        "config": {"shape": shape, "tau": 0.6, "inflow_u": 0.04, "drag_k": 0.05, "walls": "y (no-slip)",
                   "alpha": "gaussian-filtered noise, sigma 4, seed 42, [0, 1]",
                   "loss": f"KE in x in [{box[0]}, {box[1]})"},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16", "f64"])
    ap.add_argument("--skip-variants", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--skip-slab", action="store_true")
    ap.add_argument("--precision", default="c3", choices=["c3", "c2", "none"],
                    help="5000-step error leg: 512x256x256 (c3), the headline 256x128x128 (c2) or none")
    ap.add_argument("--repeats", type=int, default=REPEATS)
    ap.add_argument("--cells-per-thread", type=int, default=0, choices=[0, 1, 2, 4])
    ap.add_argument("--staging", default="auto", choices=["auto", "registers", "tma", "pipelined", "persistent"])
    ap.add_argument("--workload", default="channel",
                    choices=["channel", "cavity", "sweep", "ensemble", "adjoint", "slab", "moments"])
    args = ap.parse_args()
    global CELLS_PER_THREAD, STAGING
    CELLS_PER_THREAD = args.cells_per_thread
    STAGING = args.staging
    if args.warmup < 3 and args.impl == "ours":
        ap.error("--warmup must be >= 3")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "slab":
        run_slab(args, rank, world, local_rank)
        return
    if args.workload != "channel":
        {"cavity": run_cavity, "sweep": run_sweep, "ensemble": run_ensemble, "adjoint": run_adjoint,
         "moments": run_moments}[args.workload](args)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
