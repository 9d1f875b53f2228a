"""Benchmark of the FD hot path: one step = one full-waveform gradient
(forward + adjoint) of a 32-shot 2-D acoustic survey.

Workload (synthetic, seeded): 256 x 768 grid (nz x nx), dh 12.5 m, dt 1 ms,
nt 3000, order 8, CPML 40 cells; a 12-layer model with sinusoidally perturbed
interfaces (1500 -> 4700 m/s, +-5% noise), Gaussian-smoothed (sigma 8 cells)
start model; 32 shots at z = 2 with uneven x, each with its own line of
200-384 receivers at z = 2 padded to 384 with off-grid coordinates; 8 Hz
Ricker wavelet delayed 0.15 s.  Loss 0.5 ||pred - obs||^2 against data
modelled once in the true model before timing.

Prints ONE JSON line.  ``value`` is Gcell-updates/s (runtime-grid cells x
shots x nt per gradient, forward + adjoint) timed with CUDA events with every
input resident in HBM; ``e2e`` is the same metric through the public API with
the model, wavelet and observed data copied from pinned host memory and the
gradient and loss copied back inside each timed step.  Multi-GPU: shots are
independent (``--gpus N`` runs N ranks, each with the full 32-shot survey; weak
scaling), with the per-step gradient all-reduced over NCCL as an FWI step does.

``--impl reference`` times the CPU implementation of the same path (the
float32 oracle restating the reference's impl='c', all host threads) on a
bounded sample of the workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# ----------------------------------------------------------------- workload
NZ, NX, NT, DT, DH, ABCN, ORDER = 256, 768, 3000, 0.001, 12.5, 40, 8
NSHOT, NREC_MIN, NREC_MAX, F0, DELAY = 32, 200, 384, 8.0, 0.15
SEED = 20261203
M = ORDER // 2
RT = (NZ + 2 * ABCN + 2 * M, NX + 2 * ABCN + 2 * M)          # runtime grid
BYTES_FWD, BYTES_REV = 16, 36                                  # algorithmic bytes per cell-step


def layered_model(nz, nx, dh, rng, nlayers=12, vmin=1500.0, vmax=4700.0):
    """Layered model: sorted-uniform interface depths, each interface perturbed
    by 3 sinusoids (total amplitude <= 20 m), monotone velocities with +-5%
    Gaussian noise."""
    depth = np.sort(rng.uniform(0.05 * nz, 0.95 * nz, nlayers - 1))
    x = np.arange(nx)
    surf = np.empty((nlayers - 1, nx))
    for i in range(nlayers - 1):
        amp = rng.uniform(0, 20.0 / dh / 3, 3)
        k = rng.uniform(1, 6, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        surf[i] = depth[i] + sum(amp[j] * np.sin(2 * np.pi * k[j] * x / nx + ph[j]) for j in range(3))
    vel = np.linspace(vmin, vmax, nlayers) * (1 + 0.05 * rng.standard_normal(nlayers))
    z = np.arange(nz)[:, None]
    idx = (z[None] > surf[:, None, :]).sum(0)
    return vel[idx].astype(np.float32)


def survey(seed=SEED):
    from scipy.ndimage import gaussian_filter
    from sweep_b200 import ricker
    rng = np.random.default_rng(seed)
    vp_true = layered_model(NZ, NX, DH, rng)
    vp_init = gaussian_filter(vp_true.astype(np.float64), 8.0).astype(np.float32)
    sx = np.sort(rng.choice(np.arange(8, NX - 8), NSHOT, replace=False))
    src = np.stack([sx, np.full(NSHOT, 2)], -1)
    rec = np.full((NSHOT, NREC_MAX, 2), -10 ** 6, np.int64)
    for b in range(NSHOT):
        n = int(rng.integers(NREC_MIN, NREC_MAX + 1))
        lo = int(np.clip(sx[b] - n, 0, NX - 2 * n)) if 2 * n <= NX else 0
        xs = lo + 2 * np.arange(n)
        xs = xs[xs < NX]
        rec[b, :len(xs), 0] = xs
        rec[b, :len(xs), 1] = 2
    w = ricker(np.arange(NT) * DT - DELAY, F0).astype(np.float32)
    return vp_true, vp_init, w, src, rec


def cell_steps(nshot=NSHOT, nt=None):
    return RT[0] * RT[1] * nshot * (NT if nt is None else nt)


# ------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.path is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


# -------------------------------------------------------------- CPU baseline
def cpu_oracle_run(nt_sample, shots=1):
    """Gradient of `shots` shots of the workload with the CPU oracle (float32,
    OpenMP over all host threads); returns (cell-steps, seconds)."""
    from oracle import oracle as O
    vp_true, vp_init, w, src, rec = survey()
    w = w[:nt_sample]
    src, rec = src[:shots], rec[:shots]
    obs = O.acoustic_forward(vp_true, w, src, rec, DH, DT, ABCN)
    t0 = time.perf_counter()
    O.acoustic_gradient(vp_init, w, src, rec, obs, DH, DT, ABCN)
    dt = time.perf_counter() - t0
    return cell_steps(shots, nt_sample), dt


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- reference
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    nt_sample = 1000
    for _ in range(args.warmup):
        cpu_oracle_run(nt_sample)
    tot_cells, tot_s = 0, 0.0
    for _ in range(args.steps):
        c, s = cpu_oracle_run(nt_sample)
        tot_cells += c
        tot_s += s
    value = tot_cells / tot_s / 1e9
    sample = f"1 of {NSHOT} shots, first {nt_sample} of {NT} steps, forward + adjoint gradient"
    line = {
        "impl": "reference", "metric": "Gcell-updates/s fwd+adj", "value": value,
        "unit": "Gcell/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_s / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_block(args),
        "cpu_baseline": {"value": value, "unit": "Gcell/s", "cores": cpu_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def config_block(args):
    return {"workload": "acoustic2d 256x768 (runtime 344x856), 32 shots, nt 3000, order 8, CPML 40, "
                        "fwd+adj gradient, boundary saving",
            "grid": [NZ, NX], "runtime_grid": list(RT), "shots_per_gpu": NSHOT, "nt": NT,
            "dh": DH, "dt": DT, "abcn": ABCN, "order": ORDER, "seed": SEED,
            "cells_counted": "runtime grid (physical + PML + halo) x shots x nt",
            "physical_fraction": NZ * NX / (RT[0] * RT[1]),
            "l2": "working set per step > L2 (inputs larger than L2; no flush)",
            "parallelism": f"shots: {NSHOT} per GPU x {args.gpus} GPU(s)"}


# ---------------------------------------------------------------------- GPU
def run_gpu(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)

    from sweep_b200 import Acoustic, PropTorch
    vp_true, vp_init, w, src, rec = survey()
    solver = PropTorch(Acoustic(spatial_order=ORDER, device=dev), shape=(NZ, NX), dh=DH, dt=DT,
                       abcn=ABCN, device=dev)
    w_d = torch.tensor(w, device=dev)
    with torch.no_grad():
        obs = solver(w_d, src, rec, models=[torch.tensor(vp_true, device=dev)])
    vp_d = torch.tensor(vp_init, device=dev)
    torch.cuda.synchronize()

    def step(vp_in, w_in, obs_in, ev=None):
        vp = vp_in.detach().requires_grad_(True)
        if ev: ev[0].record()
        pred = solver(w_in, src, rec, models=[vp])
        loss = 0.5 * ((pred - obs_in) ** 2).sum()
        if ev: ev[1].record()
        loss.backward()
        if ev: ev[2].record()
        g = vp.grad
        if world > 1:
            dist.all_reduce(g)
        return loss, g

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step(vp_d, w_d, obs)
    barrier()

    # ---- device-resident timing
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        t0.record()
        for k in range(args.steps):
            step(vp_d, w_d, obs, evs[k])
        t1.record()
        barrier()
    ms = t0.elapsed_time(t1) / args.steps
    fwd_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    rev_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))
    clocks = clk.summary()
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t)

    # ---- end-to-end through the public API with host buffers
    vp_h = torch.tensor(vp_init).pin_memory()
    w_h = torch.tensor(w).pin_memory()
    obs_h = obs.cpu().pin_memory()
    g_h = torch.empty(vp_init.shape, dtype=torch.float32).pin_memory()
    h2d = vp_h.numel() * 4 + w_h.numel() * 4 + obs_h.numel() * 4
    d2h = g_h.numel() * 4 + 4
    for _ in range(2):
        step(vp_h.to(dev, non_blocking=True), w_h.to(dev, non_blocking=True), obs_h.to(dev, non_blocking=True))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        loss, g = step(vp_h.to(dev, non_blocking=True), w_h.to(dev, non_blocking=True),
                       obs_h.to(dev, non_blocking=True))
        g_h.copy_(g, non_blocking=True)
        float(loss)
    e1.record()
    barrier()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t)

    cells = cell_steps()
    value = cells * world / (ms * 1e-3) / 1e9
    e2e_value = cells * world / (e2e_ms * 1e-3) / 1e9
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    per_launch_cells = RT[0] * RT[1] * NSHOT
    rev_launch_ms = rev_ms / NT
    achieved = per_launch_cells * BYTES_REV / (rev_launch_ms * 1e-3) / 1e9
    line = {
        "metric": "Gcell-updates/s fwd+adj", "value": value, "unit": "Gcell/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded layered model, see config)",
        "config": config_block(args),
        "forward_ms": fwd_ms, "backward_ms": rev_ms,
        "roofline": {"kernel": "sweep::a2d::rev_kernel (fused adjoint + reconstruction + imaging step)",
                     "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if pk.exists() else "fallback 6650",
                     "algorithmic_bytes_per_launch": per_launch_cells * BYTES_REV,
                     "launch_ms": rev_launch_ms,
                     "launch_ms_how": "CUDA events around the backward call on the launch stream / nt",
                     "traffic": None},
        "forward_roofline": {"achieved": per_launch_cells * BYTES_FWD / (fwd_ms / NT * 1e-3) / 1e9,
                             "unit": "GB/s", "bytes_per_cell_step": BYTES_FWD},
        "gpu_launches": args.steps * (2 * NT + 1),
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": "Gcell/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
    }
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        c, s = cpu_oracle_run(1000)
        line["cpu_baseline"] = {"value": c / s / 1e9, "unit": "Gcell/s", "cores": cpu_threads(),
                                "kind": "port",
                                "sample": f"1 of {NSHOT} shots, first 1000 of {NT} steps, fwd+adj gradient"}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nt", type=int, default=None,
                    help="shorter time axis (profiling captures only; the bench line is for the full nt)")
    args = ap.parse_args()
    if args.nt:
        global NT
        NT = int(args.nt)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
