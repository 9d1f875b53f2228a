"""Benchmark of the FD hot path: Gcell-updates/s of the forward + adjoint
gradient, with every figure the measurement needs in one JSON line.

Default workload (``--workload acoustic3d``): the 3-D acoustic survey,
256^3 (runtime grid 312^3), dh 10 m, dt 1 ms, nt 2000, order 8, CPML 24; an
8-layer dipping model (1500-4000 m/s) with a +600 m/s Gaussian anomaly
(seeded; its largest velocity 4247 m/s keeps the Courant number 0.425 below
the 3-D limit 0.4529), Gaussian-smoothed start model; 16 shots on a 4 x 4
surface grid, a 128 x 128 receiver array at 2-cell spacing, 10 Hz Ricker.
The shots run in groups whose boundary-saving tape fits a 60 GB budget (3
shots; a group that did not fit would checkpoint every 100 steps).

One bench step is one FWI gradient step: each GPU computes the forward and
adjoint of one shot group (the survey's shots taken in turn), then one NCCL
all-reduce sums the loss and the gradient over the GPUs.  ``value`` counts
runtime-grid cells x shots x nt of every GPU, timed with CUDA events with
every input resident in HBM (max over ranks); ``e2e`` is the same through the
public API with the model, wavelet and the group's observed data copied from
pinned host memory and the gradient and loss read back inside each step.

Other workloads: ``acoustic2d`` (the 32-shot 256 x 768 survey: one step is
the 32-shot gradient), ``elastic2d`` (the 16-shot 400 x 1200 elastic
survey), ``elastic3d`` (the 4-shot 128^3 elastic survey), ``acoustic2d_c1``
(96 x 128, one shot) and ``fwi`` (learned vs plain FWI).

``--gpus N`` without a launcher starts N ranks itself (torch.distributed.run
on 127.0.0.1); under torchrun the ranks come from the environment.

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


# Elastic workload (--workload elastic2d): 400 x 1200, dh 5 m, dt 0.5 ms,
# nt 4000, order 8, CPML 40; vp layered 1800-4500 m/s, vs = vp / 1.73,
# rho = 310 vp^0.25; 16 explosive shots (10 Hz Ricker), 600 two-component
# receivers per shot at z = 3.
E_NZ, E_NX, E_NT, E_DT, E_DH, E_ABCN = 400, 1200, 4000, 0.0005, 5.0, 40
E_NSHOT, E_NREC, E_F0, E_DELAY = 16, 600, 10.0, 0.12
E_RT = (E_NZ + 2 * E_ABCN + 2 * M, E_NX + 2 * E_ABCN + 2 * M)
# algorithmic bytes per runtime cell-step: forward velocity 7 floats + stress
# 8; reverse stress half 15, stress-adjoint 7, velocity-adjoint + velocity
# reconstruction 17 (one read and one write of every field a kernel touches;
# CPML memories and the shared, L2-resident models not counted)
E_BYTES_FWD, E_BYTES_REV = 60, 156


def elastic_survey(seed=SEED):
    from scipy.ndimage import gaussian_filter
    from sweep_b200 import ricker
    rng = np.random.default_rng(seed + 3)
    vp_true = layered_model(E_NZ, E_NX, E_DH, rng, nlayers=12, vmin=1800.0, vmax=4500.0)
    vp_init = gaussian_filter(vp_true.astype(np.float64), 8.0).astype(np.float32)
    models = []
    for vp in (vp_true, vp_init):
        models.append([vp, (vp / 1.73).astype(np.float32), (310.0 * vp ** 0.25).astype(np.float32)])
    sx = np.sort(rng.choice(np.arange(10, E_NX - 10), E_NSHOT, replace=False))
    src = np.stack([sx, np.full(E_NSHOT, 3)], -1)
    rec = np.zeros((E_NSHOT, E_NREC, 2), np.int64)
    rec[:, :, 0] = np.linspace(0, E_NX - 1, E_NREC).astype(np.int64)[None]
    rec[:, :, 1] = 3
    w = ricker(np.arange(E_NT) * E_DT - E_DELAY, E_F0).astype(np.float32)
    return models[0], models[1], w, src, rec


# Acoustic VTI workload (--workload vti2d): the elastic survey's grid, shots,
# receivers and wavelet (400 x 1200, dh 5 m, dt 0.5 ms, nt 4000, CPML 40, 16
# shots, vz receivers), vp the same layers, Thomsen epsilon 0.05-0.2 growing
# with vp, delta = epsilon / 2, rho = 310 vp^0.25; sources on (sH, sV).
# Algorithmic bytes per runtime cell-step (one read and one write of every
# field a kernel touches; CPML memories and the models not counted): forward
# velocity 6 floats + stress 6; reverse stress reconstruction 6, half-step A 4
# + 6, gradient 8 + 8 slots, half-step B 4 + 6, velocity reconstruction 6.
V_BYTES_FWD, V_BYTES_REV = 48, 192


def vti_survey(seed=SEED):
    (vp, _, rho), (vp0, _, rho0), w, src, rec = elastic_survey(seed)
    out = []
    for v, r in ((vp, rho), (vp0, rho0)):
        eps = (0.05 + 0.15 * (v - 1800.0) / 2700.0).astype(np.float32)
        out.append([v, eps, (0.5 * eps).astype(np.float32), r])
    return out[0], out[1], w, src, rec


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


# Boundary-saving tape of the acoustic workloads: (storage, strip dtype); the
# default line is the reference's default, fp32 strips in GPU memory
STRIPS = ["gpu", "fp32"]


def boundary_memory():
    from sweep_b200 import BoundarySaving
    return BoundarySaving(storage=STRIPS[0], storage_dtype=STRIPS[1])


# --------------------------------------------------------------- workloads
class AcousticWorkload:
    name = "acoustic2d"
    nt, nshot, rt = NT, NSHOT, RT
    bytes_fwd, bytes_rev = BYTES_FWD, BYTES_REV
    kernel = "sweep::a2d::rev_kernel (fused adjoint + reconstruction + imaging step)"
    cpu_nt = 1000
    # ncu dram__bytes_read.sum + dram__bytes_write.sum of one rev_kernel launch of
    # this grid at 32 shots (241.9 + 69.3 MB; the capture's time axis is 20
    # steps, which does not change a launch), per shot
    traffic = {"bytes_per_shot": 311.2e6 / 32, "source": "ncu, one rev_kernel launch, 256x768 x 32 shots (nt 20)"}

    def config(self, args):
        return {"workload": f"acoustic2d {NZ}x{NX} (runtime {RT[0]}x{RT[1]}), {NSHOT} shots, nt {NT}, "
                            f"order {ORDER}, CPML {ABCN}, fwd+adj gradient, boundary saving",
                "grid": [NZ, NX], "runtime_grid": list(RT), "shots_per_gpu": NSHOT, "nt": NT,
                "dh": DH, "dt": DT, "abcn": ABCN, "order": ORDER, "seed": SEED,
                "cells_counted": "runtime grid (physical + PML + halo) x shots x nt",
                "physical_fraction": NZ * NX / (RT[0] * RT[1]),
                "l2": "working set per step > L2 (inputs larger than L2; no flush)",
                "boundary_tape": f"{STRIPS[1]} strips in {STRIPS[0]} memory",
                "parallelism": f"shots: {NSHOT} per GPU x {args.gpus} GPU(s)"}

    dh, dt, abcn, ref_gpu_nt = DH, DT, ABCN, 3000

    def survey_inputs(self):
        vp_true, vp_init, w, src, rec = survey()
        return [vp_true], [vp_init], w, src, rec

    def build(self, dev):
        from sweep_b200 import Acoustic, PropTorch
        vp_true, vp_init, w, src, rec = survey()
        solver = PropTorch(Acoustic(spatial_order=ORDER, device=dev), shape=(NZ, NX), dh=DH, dt=DT,
                           abcn=ABCN, device=dev, memory=boundary_memory())
        return solver, [vp_true], [vp_init], w, src, rec

    def launches(self, group):
        # per gradient: the forward's prep_kernel and one fwd_kernel per step,
        # the backward's prep_kernel, one rev_kernel per step and finalize_kernel
        return 2 * self.nt + 3

    def cpu_run(self, nt_sample, shots=1):
        """Gradient of `shots` shots with the CPU oracle (float32, OpenMP over
        all host threads); returns (cell-steps, seconds)."""
        from oracle import oracle as O
        vp_true, vp_init, w, src, rec = survey()
        w, src, rec = w[:nt_sample], src[:shots], rec[:shots]
        obs = O.acoustic_forward(vp_true, w, src, rec, DH, DT, ABCN)
        t0 = time.perf_counter()
        O.acoustic_gradient(vp_init, w, src, rec, obs, DH, DT, ABCN)
        return RT[0] * RT[1] * shots * nt_sample, time.perf_counter() - t0


# Small 2-D workload (--workload acoustic2d_c1): the reference's own
# CPU-runnable case.  96 x 128, dh 10 m, dt 2 ms, nt 800, order 8, CPML 20;
# two layers (1500 m/s upper half, 2500 m/s lower half), start model 1500
# m/s; one 10 Hz Ricker delayed 0.14 s at (x 32, z 48), one receiver at
# (x 96, z 48).  The runtime grid (144 x 176) fits in L2: the step loop is
# launch- and latency-bound, which is where the captured CUDA graphs count.
C1_NZ, C1_NX, C1_NT, C1_DT, C1_DH, C1_ABCN = 96, 128, 800, 0.002, 10.0, 20
C1_RT = (C1_NZ + 2 * C1_ABCN + 2 * M, C1_NX + 2 * C1_ABCN + 2 * M)


def c1_survey():
    from sweep_b200 import ricker
    vp_true = np.full((C1_NZ, C1_NX), 1500.0, np.float32)
    vp_true[C1_NZ // 2:] = 2500.0
    vp_init = np.full((C1_NZ, C1_NX), 1500.0, np.float32)
    w = ricker(np.arange(C1_NT) * C1_DT - 0.14, 10.0).astype(np.float32)
    return vp_true, vp_init, w, np.array([[32, 48]]), np.array([[[96, 48]]])


class AcousticC1Workload:
    name = "acoustic2d_c1"
    nt, nshot, rt = C1_NT, 1, C1_RT
    bytes_fwd, bytes_rev = BYTES_FWD, BYTES_REV
    kernel = "sweep::a2d::rev_kernel (fused adjoint + reconstruction + imaging step)"
    cpu_nt = C1_NT
    traffic = None

    def config(self, args):
        return {"workload": f"acoustic2d {C1_NZ}x{C1_NX} (runtime {C1_RT[0]}x{C1_RT[1]}), 1 shot, nt {C1_NT}, "
                            f"order {ORDER}, CPML {C1_ABCN}, fwd+adj gradient, boundary saving",
                "grid": [C1_NZ, C1_NX], "runtime_grid": list(C1_RT), "shots_per_gpu": 1, "nt": C1_NT,
                "dh": C1_DH, "dt": C1_DT, "abcn": C1_ABCN, "order": ORDER,
                "cells_counted": "runtime grid (physical + PML + halo) x shots x nt",
                "l2": "working set fits in L2 (0.5 MB per field): latency- and launch-bound, no flush",
                "boundary_tape": f"{STRIPS[1]} strips in {STRIPS[0]} memory",
                "parallelism": f"replicas: 1 shot per GPU x {args.gpus} GPU(s)"}

    dh, dt, abcn, ref_gpu_nt = C1_DH, C1_DT, C1_ABCN, C1_NT

    def survey_inputs(self):
        vp_true, vp_init, w, src, rec = c1_survey()
        return [vp_true], [vp_init], w, src, rec

    def build(self, dev):
        from sweep_b200 import Acoustic, PropTorch
        vp_true, vp_init, w, src, rec = c1_survey()
        solver = PropTorch(Acoustic(spatial_order=ORDER, device=dev), shape=(C1_NZ, C1_NX), dh=C1_DH,
                           dt=C1_DT, abcn=C1_ABCN, device=dev, memory=boundary_memory())
        return solver, [vp_true], [vp_init], w, src, rec

    def launches(self, group):
        # per gradient: the forward's prep_kernel and one fwd_kernel per step,
        # the backward's prep_kernel, one rev_kernel per step and finalize_kernel
        return 2 * self.nt + 3

    def cpu_run(self, nt_sample, shots=1):
        from oracle import oracle as O
        vp_true, vp_init, w, src, rec = c1_survey()
        w = w[:nt_sample]
        obs = O.acoustic_forward(vp_true, w, src, rec, C1_DH, C1_DT, C1_ABCN)
        t0 = time.perf_counter()
        O.acoustic_gradient(vp_init, w, src, rec, obs, C1_DH, C1_DT, C1_ABCN)
        return C1_RT[0] * C1_RT[1] * nt_sample, time.perf_counter() - t0


class ElasticWorkload:
    name = "elastic2d"
    nt, nshot, rt = E_NT, E_NSHOT, E_RT
    bytes_fwd, bytes_rev = E_BYTES_FWD, E_BYTES_REV
    kernel = ("sweep::el2d reverse step (rev_str + rev_sadj + rev_vadj: reconstruction, imaging, "
              "stress- and velocity-adjoint)")
    cpu_nt = 300
    traffic = None

    def config(self, args):
        return {"workload": f"elastic2d {E_NZ}x{E_NX} (runtime {E_RT[0]}x{E_RT[1]}), {E_NSHOT} shots, "
                            f"nt {E_NT}, order 8, CPML {E_ABCN}, vp/vs/rho fwd+adj gradient, boundary saving",
                "grid": [E_NZ, E_NX], "runtime_grid": list(E_RT), "shots_per_gpu": E_NSHOT, "nt": E_NT,
                "dh": E_DH, "dt": E_DT, "abcn": E_ABCN, "order": ORDER, "receivers": E_NREC,
                "seed": SEED, "cells_counted": "runtime grid (physical + PML + halo) x shots x nt",
                "physical_fraction": E_NZ * E_NX / (E_RT[0] * E_RT[1]),
                "l2": "working set per step > L2 (inputs larger than L2; no flush)",
                "parallelism": f"shots: {E_NSHOT} per GPU x {args.gpus} GPU(s)"}

    dh, dt, abcn, ref_gpu_nt = E_DH, E_DT, E_ABCN, 1000

    def survey_inputs(self):
        return elastic_survey()

    def build(self, dev):
        from sweep_b200 import Elastic, PropTorch
        m_true, m_init, w, src, rec = elastic_survey()
        solver = PropTorch(Elastic(spatial_order=ORDER, device=dev), shape=(E_NZ, E_NX), dh=E_DH,
                           dt=E_DT, abcn=E_ABCN, device=dev)
        return solver, m_true, m_init, w, src, rec

    def launches(self, group):
        return 5 * self.nt + 2

    def cpu_run(self, nt_sample, shots=1):
        from oracle import oracle as O
        m_true, m_init, w, src, rec = elastic_survey()
        w, src, rec = w[:nt_sample], src[:shots], rec[:shots]
        obs = O.elastic_forward(*m_true, w, src, rec, E_DH, E_DT, E_ABCN)
        t0 = time.perf_counter()
        O.elastic_gradient(*m_init, w, src, rec, obs, E_DH, E_DT, E_ABCN)
        return E_RT[0] * E_RT[1] * shots * nt_sample, time.perf_counter() - t0


class VTIWorkload(ElasticWorkload):
    name = "vti2d"
    bytes_fwd, bytes_rev = V_BYTES_FWD, V_BYTES_REV
    kernel = "sweep::vti reverse step (srev + premA + appA + grad + premB + appB + vrev + band restores)"
    tunable = False

    def config(self, args):
        c = super().config(args)
        c["workload"] = (f"vti2d (AcousticVTI1st) {E_NZ}x{E_NX} (runtime {E_RT[0]}x{E_RT[1]}), {E_NSHOT} shots, "
                         f"nt {E_NT}, order {ORDER}, CPML {E_ABCN}, vp/epsilon/delta/rho fwd+adj gradient, "
                         f"boundary saving")
        return c

    def survey_inputs(self):
        return vti_survey()

    def build(self, dev):
        from sweep_b200 import AcousticVTI1st, PropTorch
        m_true, m_init, w, src, rec = vti_survey()
        solver = PropTorch(AcousticVTI1st(spatial_order=ORDER, device=dev), shape=(E_NZ, E_NX), dh=E_DH,
                           dt=E_DT, abcn=E_ABCN, device=dev)
        return solver, m_true, m_init, w, src, rec

    def launches(self, group):
        return 5 * self.nt + 11 * (self.nt - 1) + 6

    def cpu_run(self, nt_sample, shots=1):
        from oracle import oracle as O
        m_true, m_init, w, src, rec = vti_survey()
        w, src, rec = w[:nt_sample], src[:shots], rec[:shots]
        obs = O.vti2d_forward(*m_true, w, src, rec, E_DH, E_DT, E_ABCN)
        t0 = time.perf_counter()
        O.vti2d_gradient(*m_init, w, src, rec, obs, E_DH, E_DT, E_ABCN)
        return E_RT[0] * E_RT[1] * shots * nt_sample, time.perf_counter() - t0


# 3-D workload (--workload acoustic3d, the default): 256^3, dh 10 m, dt 1 ms,
# nt 2000, order 8, CPML 24; 8-layer dipping model (1500-4000 m/s) with a
# +600 m/s Gaussian anomaly; 16 shots on a 4 x 4 surface grid, a 128 x 128
# receiver array at 2-cell spacing, 10 Hz Ricker.  Shots run in groups whose
# boundary-saving tape fits the 60 GB budget: 3 shots (47 GB; 4 would be
# 63 GB).
A3_N, A3_NT, A3_DT, A3_DH, A3_ABCN = 256, 2000, 0.001, 10.0, 24
A3_NSHOT, A3_BATCH, A3_F0, A3_DELAY = 16, 4, 10.0, 0.12
# boundary storage budget of one call: a shot group whose boundary-saving tape
# exceeds it checkpoints every 100 steps instead
A3_BUDGET_GB, A3_CKPT = 60.0, 100
A3_RT = (A3_N + 2 * A3_ABCN + 2 * M,) * 3


def acoustic3d_survey(seed=SEED):
    from scipy.ndimage import gaussian_filter
    from sweep_b200 import ricker
    rng = np.random.default_rng(seed + 7)
    n = A3_N
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    depth = np.sort(rng.uniform(0.08 * n, 0.92 * n, 7))
    vel = np.linspace(1500.0, 4000.0, 8)
    idx = np.zeros((n, n, n), np.int32)
    for d0 in depth:
        strike = rng.uniform(0, 2 * np.pi)
        dip = np.deg2rad(rng.uniform(0, 15))
        surf = d0 + np.tan(dip) * ((x - n / 2) * np.cos(strike) + (y - n / 2) * np.sin(strike))
        idx += (z > surf).astype(np.int32)
    vp = vel[idx]
    cz, cy, cx = rng.uniform(0.3 * n, 0.7 * n), rng.uniform(0.3 * n, 0.7 * n), rng.uniform(0.3 * n, 0.7 * n)
    vp += 600.0 * np.exp(-((z - cz) ** 2 + (y - cy) ** 2 + (x - cx) ** 2) / (2 * 30.0 ** 2))
    vp_true = vp.astype(np.float32)
    courant = float(vp_true.max()) * A3_DT / A3_DH
    if courant >= 0.4529:
        raise ValueError(f"3-D survey: Courant number {courant:.3f} above the order-8 leapfrog limit 0.4529")
    vp_init = gaussian_filter(vp_true.astype(np.float64), 8.0).astype(np.float32)
    g = np.linspace(n / 8, n - n / 8, 4).astype(np.int64)
    src = np.array([[xs, ys, 2] for ys in g for xs in g], np.int64)
    r = np.arange(0, 2 * 128, 2)
    rx, ry = np.meshgrid(r, r, indexing="xy")
    one = np.stack([rx.ravel(), ry.ravel(), np.full(rx.size, 2)], -1)
    rec = np.broadcast_to(one, (A3_NSHOT,) + one.shape).copy()
    w = ricker(np.arange(A3_NT) * A3_DT - A3_DELAY, A3_F0).astype(np.float32)
    return [vp_true], [vp_init], w, src, rec


class Acoustic3DWorkload:
    name = "acoustic3d"
    nt, nshot, rt = A3_NT, A3_NSHOT, A3_RT
    bytes_fwd, bytes_rev = BYTES_FWD, BYTES_REV
    kernel = "sweep::a3d reverse step (a3_step + r3_recon + strip kernels)"
    cpu_nt = 16
    # ncu DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of a3_step +
    # r3_recon for one 256^3 shot (860 + 856 MB), scaled by the shots of a
    # reverse step: both kernels stream every shot's fields once, so traffic
    # grows with the shots
    traffic = {"bytes_per_shot": 860e6 + 856e6,
               "source": "ncu, a3_step + r3_recon of one 256^3 shot, x shots per step"}
    batch = A3_BATCH
    budget_gb = A3_BUDGET_GB

    def config(self, args):
        return {"workload": f"acoustic3d {A3_N}^3 (runtime {A3_RT[0]}^3), {A3_NSHOT}-shot survey in calls of "
                            f"{self.batch} shots, nt {self.nt}, order {ORDER}, CPML {A3_ABCN}, fwd+adj gradient, "
                            f"boundary saving",
                "grid": [A3_N] * 3, "runtime_grid": list(A3_RT), "shots_per_gpu": A3_NSHOT,
                "shots_per_call": self.batch, "nt": self.nt, "dh": A3_DH, "dt": A3_DT, "abcn": A3_ABCN,
                "order": ORDER, "receivers": 128 * 128, "seed": SEED,
                "cells_counted": "runtime grid (physical + PML + halo) x shots x nt",
                "physical_fraction": (A3_N / A3_RT[0]) ** 3,
                "l2": "working set per step > L2 (inputs larger than L2; no flush)",
                "boundary_tape": f"{STRIPS[1]} strips in {STRIPS[0]} memory",
                "memory_rule": f"boundary saving when a call's tape fits {A3_BUDGET_GB:g} GB, else checkpoints "
                               f"every {A3_CKPT} steps; shots per call: the most whose boundary tape fits "
                               f"(at most {A3_BATCH}) unless --shots-per-call is given",
                "courant_max": 4247.13 * A3_DT / A3_DH}

    dh, dt, abcn, ref_gpu_nt = A3_DH, A3_DT, A3_ABCN, 200

    def survey_inputs(self):
        return acoustic3d_survey()

    def build(self, dev):
        from sweep_b200 import Acoustic3D, PropTorch
        m_true, m_init, w, src, rec = acoustic3d_survey()
        from sweep_b200 import BoundarySaving
        solver = PropTorch(Acoustic3D(spatial_order=ORDER, device=dev), shape=(A3_N,) * 3, dh=A3_DH,
                           dt=A3_DT, abcn=A3_ABCN, device=dev,
                           memory=BoundarySaving(storage=STRIPS[0], storage_dtype=STRIPS[1],
                                                 budget_gb=A3_BUDGET_GB, ckpt_chunks=A3_CKPT))
        return solver, m_true, m_init, w, src, rec

    def launches(self, group):
        # per call (one shot group): forward 4 per step (stencil, strips,
        # injection, gather) and reverse 7 (adjoint, cotangent injection,
        # reconstruction, strip restore, strip un-injection, strip image, source
        # re-injection); per pass prep3 and three pack_prof3, and finalize3
        return 11 * self.nt + 9

    def cpu_run(self, nt_sample, shots=1):
        from oracle import oracle as O
        m_true, m_init, w, src, rec = acoustic3d_survey()
        w, src, rec = w[:nt_sample], src[:shots], rec[:shots]
        obs = O.acoustic_forward(m_true[0], w, src, rec, A3_DH, A3_DT, A3_ABCN)
        t0 = time.perf_counter()
        O.acoustic_gradient(m_init[0], w, src, rec, obs, A3_DH, A3_DT, A3_ABCN)
        return A3_RT[0] ** 3 * shots * nt_sample, time.perf_counter() - t0


# 3-D elastic workload (--workload elastic3d): 128^3, dh 10 m, dt 0.8 ms,
# nt 600, order 8, CPML 16; 6-layer dipping model (1800-4200 m/s), vs =
# vp / 1.73, rho = 310 vp^0.25; 4 explosive shots on a 2 x 2 surface grid, a
# 64 x 64 three-component receiver array at 2-cell spacing, 15 Hz Ricker.
E3_N, E3_NT, E3_DT, E3_DH, E3_ABCN = 128, 600, 0.0008, 10.0, 16
E3_NSHOT, E3_F0, E3_DELAY = 4, 15.0, 0.08
E3_RT = (E3_N + 2 * E3_ABCN + 2 * M,) * 3
# algorithmic floats per runtime cell-step (one read and one write of every
# field a kernel touches; models and CPML memories not counted): forward
# velocity step 6 stresses read + 3 velocities read and written (12), stress
# step 3 + 6 + 6 (15); reverse: stress reconstruction 15, stress-adjoint
# prepare 6 + 3 + 3 + 3 read, 3 gradient slots read and written, 9 q written
# (30), its apply 9 + 6 (15), velocity-adjoint prepare 3 + 9 (12), its apply
# 9 + 12 (21), carriers 6, velocity reconstruction 12 (111)
E3_BYTES_FWD, E3_BYTES_REV = 4 * 27, 4 * 111


def elastic3d_survey(seed=SEED):
    from scipy.ndimage import gaussian_filter
    from sweep_b200 import ricker
    rng = np.random.default_rng(seed + 13)
    n = E3_N
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    depth = np.sort(rng.uniform(0.1 * n, 0.9 * n, 5))
    vel = np.linspace(1800.0, 4200.0, 6)
    idx = np.zeros((n, n, n), np.int32)
    for d0 in depth:
        strike = rng.uniform(0, 2 * np.pi)
        dip = np.deg2rad(rng.uniform(0, 12))
        surf = d0 + np.tan(dip) * ((x - n / 2) * np.cos(strike) + (y - n / 2) * np.sin(strike))
        idx += (z > surf).astype(np.int32)
    vp_true = vel[idx].astype(np.float32)
    courant = float(vp_true.max()) * E3_DT / E3_DH
    if courant >= 0.4547:
        raise ValueError(f"3-D elastic survey: Courant number {courant:.3f} above the staggered order-8 limit")
    vp_init = gaussian_filter(vp_true.astype(np.float64), 6.0).astype(np.float32)
    models = []
    for vp in (vp_true, vp_init):
        models.append([vp, (vp / 1.73).astype(np.float32), (310.0 * vp ** 0.25).astype(np.float32)])
    g = np.linspace(n / 4, n - n / 4, 2).astype(np.int64)
    src = np.array([[xs, ys, 3] for ys in g for xs in g], np.int64)
    r = np.arange(0, 2 * 64, 2)
    rx, ry = np.meshgrid(r, r, indexing="xy")
    one = np.stack([rx.ravel(), ry.ravel(), np.full(rx.size, 3)], -1)
    rec = np.broadcast_to(one, (E3_NSHOT,) + one.shape).copy()
    w = ricker(np.arange(E3_NT) * E3_DT - E3_DELAY, E3_F0).astype(np.float32)
    return models[0], models[1], w, src, rec


class Elastic3DWorkload:
    name = "elastic3d"
    nt, nshot, rt = E3_NT, E3_NSHOT, E3_RT
    bytes_fwd, bytes_rev = E3_BYTES_FWD, E3_BYTES_REV
    kernel = ("sweep::el3d reverse step (srev3 + sprep3 + sapp3 + vprep3 + vapp3 + cap3 + vrev3 + strip "
              "kernels)")
    cpu_nt = 24
    traffic = None
    tunable = False             # one built-in launch schedule

    def config(self, args):
        return {"workload": f"elastic3d {E3_N}^3 (runtime {E3_RT[0]}^3), {E3_NSHOT} shots, nt {E3_NT}, "
                            f"order 8, CPML {E3_ABCN}, vp/vs/rho fwd+adj gradient, boundary saving",
                "grid": [E3_N] * 3, "runtime_grid": list(E3_RT), "shots_per_gpu": E3_NSHOT, "nt": E3_NT,
                "dh": E3_DH, "dt": E3_DT, "abcn": E3_ABCN, "order": ORDER, "receivers": 64 * 64,
                "seed": SEED, "cells_counted": "runtime grid (physical + PML + halo) x shots x nt",
                "physical_fraction": (E3_N / E3_RT[0]) ** 3,
                "l2": "working set per step > L2 (inputs larger than L2; no flush)",
                "parallelism": f"shots: {E3_NSHOT} per GPU x {args.gpus} GPU(s)"}

    dh, dt, abcn, ref_gpu_nt = E3_DH, E3_DT, E3_ABCN, 200

    def survey_inputs(self):
        return elastic3d_survey()

    def build(self, dev):
        from sweep_b200 import Elastic3D, PropTorch
        m_true, m_init, w, src, rec = elastic3d_survey()
        solver = PropTorch(Elastic3D(spatial_order=ORDER, device=dev), shape=(E3_N,) * 3, dh=E3_DH,
                           dt=E3_DT, abcn=E3_ABCN, device=dev)
        return solver, m_true, m_init, w, src, rec

    def launches(self, group):
        # forward 5 per step (velocity, stress, source, strips, record);
        # reverse 12 (body-force correction only with velocity sources: not
        # here; residuals, source removal, two reconstructions, two restores,
        # two prepares, two applies, carriers, receiver rho); prep3 and three
        # finalize3 per pass
        return 5 * self.nt + 12 * (self.nt - 1) + 4

    def cpu_run(self, nt_sample, shots=1):
        from oracle import oracle as O
        m_true, m_init, w, src, rec = elastic3d_survey()
        w, src, rec = w[:nt_sample], src[:shots], rec[:shots]
        obs = O.elastic3d_forward(*m_true, w, src, rec, E3_DH, E3_DT, E3_ABCN)
        t0 = time.perf_counter()
        O.elastic3d_gradient(*m_init, w, src, rec, obs, E3_DH, E3_DT, E3_ABCN)
        return E3_RT[0] ** 3 * shots * nt_sample, time.perf_counter() - t0


# 3-D acoustic VTI workload (--workload vti3d): the 3-D elastic survey's grid,
# shots, receivers and wavelet (128^3, dh 10 m, dt 0.8 ms, nt 600, CPML 16,
# 4 shots, vz receivers), vp the same dipping layers, Thomsen epsilon
# 0.05-0.2 growing with vp, delta = epsilon / 2, rho = 310 vp^0.25; sources
# on (sH, sV).  Algorithmic floats per runtime cell-step (one read and one
# write of every field a kernel touches; CPML memories and the models not
# counted): forward velocity step 2 stresses read + 3 velocities read and
# written (8), stress step 3 + 4 (7); reverse: stress reconstruction 7,
# half-step A pre-multiply 2 + 3 and apply 3 + 6, gradient 10 + 8 slots,
# half-step B 3 + 3 and 3 + 4, velocity reconstruction 8 (60).
V3_BYTES_FWD, V3_BYTES_REV = 4 * 15, 4 * 60


def vti3d_survey(seed=SEED):
    (vp, _, rho), (vp0, _, rho0), w, src, rec = elastic3d_survey(seed)
    out = []
    for v, r in ((vp, rho), (vp0, rho0)):
        eps = (0.05 + 0.15 * (v - 1800.0) / 2400.0).astype(np.float32)
        out.append([v, eps, (0.5 * eps).astype(np.float32), r])
    return out[0], out[1], w, src, rec


class VTI3DWorkload(Elastic3DWorkload):
    name = "vti3d"
    bytes_fwd, bytes_rev = V3_BYTES_FWD, V3_BYTES_REV
    kernel = "sweep::vti3 reverse step (srev + premA + appA + grad + premB + appB + vrev + band restores)"
    cpu_nt = 24

    def config(self, args):
        c = super().config(args)
        c["workload"] = (f"vti3d (AcousticVTI1st3D) {E3_N}^3 (runtime {E3_RT[0]}^3), {E3_NSHOT} shots, "
                         f"nt {E3_NT}, order {ORDER}, CPML {E3_ABCN}, vp/epsilon/delta/rho fwd+adj gradient, "
                         f"boundary saving")
        return c

    def survey_inputs(self):
        return vti3d_survey()

    def build(self, dev):
        from sweep_b200 import AcousticVTI1st3D, PropTorch
        m_true, m_init, w, src, rec = vti3d_survey()
        solver = PropTorch(AcousticVTI1st3D(spatial_order=ORDER, device=dev), shape=(E3_N,) * 3, dh=E3_DH,
                           dt=E3_DT, abcn=E3_ABCN, device=dev, receiver_type=["vz"])
        return solver, m_true, m_init, w, src, rec

    def launches(self, group):
        # forward 5 per step (velocity, stress, source, bands, record); reverse
        # 11 (residuals, source removal, two reconstructions, two band
        # restores, two pre-multiplies, two applies, gradient); prep per pass
        # and four finalize
        return 5 * self.nt + 11 * (self.nt - 1) + 6

    def cpu_run(self, nt_sample, shots=1):
        from oracle import oracle as O
        m_true, m_init, w, src, rec = vti3d_survey()
        w, src, rec = w[:nt_sample], src[:shots], rec[:shots]
        obs = O.vti3d_forward(*m_true, w, src, rec, E3_DH, E3_DT, E3_ABCN, order=ORDER)
        t0 = time.perf_counter()
        O.vti3d_gradient(*m_init, w, src, rec, obs, E3_DH, E3_DT, E3_ABCN, order=ORDER)
        return E3_RT[0] ** 3 * shots * nt_sample, time.perf_counter() - t0


WORKLOADS = {"acoustic2d": AcousticWorkload, "acoustic2d_c1": AcousticC1Workload, "elastic2d": ElasticWorkload,
             "vti2d": VTIWorkload, "vti3d": VTI3DWorkload,
             "acoustic3d": Acoustic3DWorkload, "elastic3d": Elastic3DWorkload}


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- reference
def run_reference(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    nt_sample = wl.cpu_nt
    for _ in range(args.warmup):
        wl.cpu_run(nt_sample)
    tot_cells, tot_s = 0, 0.0
    for _ in range(args.steps):
        c, s = wl.cpu_run(nt_sample)
        tot_cells += c
        tot_s += s
    value = tot_cells / tot_s / 1e9
    sample = f"1 of {wl.nshot} shots, first {nt_sample} of {wl.nt} steps, forward + adjoint gradient"
    line = {
        "impl": "reference", "metric": "Gcell-updates/s fwd+adj", "value": value,
        "unit": "Gcell/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_s / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": wl.config(args),
        "cpu_baseline": {"value": value, "unit": "Gcell/s", "cores": cpu_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ------------------------------------------------- the reference's CUDA core
REF_DIR = ROOT / "baseline" / "_ref"


def reference_cuda(wl, group, nt_sample, dev, reps=2):
    """The reference's own impl='c' CUDA core (installed under baseline/_ref
    with its core built for this GPU) on the same workload: `group` shots of
    the survey over the first `nt_sample` steps, forward + adjoint gradient
    through its public PropTorch API, timed with CUDA events (best of `reps`
    after one warm-up).  Runs after every timed region of this bench."""
    import torch
    core = list(REF_DIR.glob("sweep/lib/cu*/libsweep_core.so"))
    if not core:
        return {"unavailable": "the reference's CUDA core is not built under baseline/_ref"}
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    try:
        from sweep.equations import Acoustic, Acoustic3D, Elastic, Elastic3D
        from sweep.equations.acoustic_vti_1st import AcousticVTI1st, AcousticVTI1st3D
        from sweep.propagator.options import BoundarySaving
        from sweep.propagator.torch import PropTorch
    except Exception as e:                       # noqa: BLE001
        return {"unavailable": f"the reference does not import: {e}"}
    m_true, m_init, w, src, rec = wl.survey_inputs()
    eq = {"acoustic2d": Acoustic, "acoustic2d_c1": Acoustic, "elastic2d": Elastic, "vti2d": AcousticVTI1st,
          "acoustic3d": Acoustic3D, "elastic3d": Elastic3D, "vti3d": AcousticVTI1st3D}[wl.name]
    solver = PropTorch(eq(spatial_order=ORDER, device=dev), shape=tuple(m_true[0].shape), dh=wl.dh,
                       dt=wl.dt, abcn=wl.abcn, impl="c", device=dev, memory=BoundarySaving())
    wt = torch.tensor(w[:nt_sample], device=dev)
    sh = list(range(min(group, len(src))))
    with torch.no_grad():
        obs = solver(wt, src[sh], rec[sh], models=[torch.tensor(m, device=dev) for m in m_true])
    best = None
    for r in range(reps + 1):
        ms = [torch.tensor(m, device=dev, requires_grad=True) for m in m_init]
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record()
        pred = solver(wt, src[sh], rec[sh], models=ms)
        loss = 0.5 * ((pred - obs) ** 2).sum()
        e1.record()
        loss.backward()
        e2.record()
        torch.cuda.synchronize()
        t = (e0.elapsed_time(e2), e0.elapsed_time(e1), e1.elapsed_time(e2))
        if r > 0 and (best is None or t[0] < best[0]):
            best = t
    cells = int(np.prod(wl.rt)) * len(sh) * nt_sample
    return {"value": cells / (best[0] * 1e-3) / 1e9, "unit": "Gcell/s", "forward_ms": best[1],
            "backward_ms": best[2], "sample": f"{len(sh)} shot(s), first {nt_sample} of {wl.nt} steps, "
                                              "forward + adjoint gradient, boundary saving",
            "how": "reference PropTorch(impl='c') on this GPU, CUDA events, best of "
                   f"{reps} after a warm-up",
            "core": str(core[0].relative_to(ROOT))}


# ---------------------------------------------------------------------- GPU
def step_shots(k, group, nshot, world, rank):
    """Shots rank `rank` computes in step `k`: the step's window is the next
    world x group shots of the survey (cyclically), split into contiguous
    blocks by sweep_b200.distributed.shot_slice -- the same split
    sharded_gradient makes, so each rank runs `group` shots of its own."""
    from sweep_b200.distributed import shot_slice
    window = [(k * world * group + i) % nshot for i in range(world * group)]
    return window[shot_slice(len(window), world, rank)]


def run_gpu(args, wl):
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

    from sweep_b200.distributed import sharded_gradient
    solver, m_true, m_init, w, src, rec = wl.build(dev)
    solver.autotune = bool(args.autotune) and getattr(wl, "tunable", True) and ORDER == 8
    src, rec = src[:wl.nshot], rec[:wl.nshot]
    if getattr(wl, "budget_gb", None) and not args.shots_per_call:
        # shot groups: the most shots whose boundary-saving tape fits the budget
        per_shot = solver.tape_bytes(len(w), src[:1], rec[:1], [torch.tensor(m, device=dev) for m in m_init])
        wl.batch = max(1, min(wl.batch, wl.nshot, int(wl.budget_gb * 1e9 // per_shot)))
    group = getattr(wl, "batch", wl.nshot)
    w_d = torch.tensor(w, device=dev)
    with torch.no_grad():
        mt = [torch.tensor(m, device=dev) for m in m_true]
        # observed data of every shot, modelled once in the true model; the
        # first call of the step's shape (group shots) tunes its schedule
        # (untimed; --no-autotune skips it).  A last, smaller group is another
        # shape: it is modelled without tuning.
        parts = [solver(w_d, src[:group], rec[:group], models=mt)]
        tune_report = solver.tune_report
        solver.autotune = False
        parts += [solver(w_d, src[b:b + group], rec[b:b + group], models=mt) for b in range(group, wl.nshot, group)]
        obs = torch.cat(parts)
        del mt, parts
    ms_d = [torch.tensor(m, device=dev) for m in m_init]
    schedule = solver.launch_schedule(len(w), src[:group], rec[:group], ms_d)
    torch.cuda.synchronize()

    def step(k, ms_in, w_in, obs_of, ev=None):
        """One FWI gradient step: this rank's shot group (forward + adjoint),
        then one SUM all-reduce of the loss and the model gradients over the
        ranks (sharded_gradient).  obs_of(shots): their observed data."""
        def compute(_):
            sh = step_shots(k, group, wl.nshot, world, rank)
            ms = [m.detach().requires_grad_(True) for m in ms_in]
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)] if ev is not None else None
            if e: e[0].record()
            pred = solver(w_in, src[sh], rec[sh], models=ms)
            lb = 0.5 * ((pred - obs_of(sh)) ** 2).sum()
            if e: e[1].record()
            lb.backward()
            if e:
                e[2].record()
                ev.append(e)
            return lb.detach(), [m.grad for m in ms]
        return sharded_gradient(compute, world * group)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def obs_dev(sh):
        return obs[sh]

    for k in range(args.warmup):
        step(k, ms_d, w_d, obs_dev)
    barrier()

    # ---- device-resident timing
    evs = [[] for _ in range(args.steps)]     # per step: (start, forward done, backward done)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        t0.record()
        for k in range(args.steps):
            step(args.warmup + k, ms_d, w_d, obs_dev, evs[k])
        t1.record()
        barrier()
    ms = t0.elapsed_time(t1) / args.steps
    fwd_ms = float(np.mean([sum(e[0].elapsed_time(e[1]) for e in st) for st in evs]))
    rev_ms = float(np.mean([sum(e[1].elapsed_time(e[2]) for e in st) for st in evs]))
    clocks = clk.summary()
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t)

    # ---- end-to-end through the public API with host buffers: each step
    # copies the models, the wavelet and its shots' observed data from pinned
    # host memory and reads the gradients and the loss back
    ms_h = [torch.tensor(m).pin_memory() for m in m_init]
    w_h = torch.tensor(w).pin_memory()
    obs_h = obs.cpu().pin_memory()
    g_h = [torch.empty(m.shape, dtype=torch.float32).pin_memory() for m in m_init]
    h2d = sum(m.numel() * 4 for m in ms_h) + w_h.numel() * 4 + obs_h[:group].numel() * 4
    d2h = sum(g.numel() * 4 for g in g_h) + 8

    o_d = torch.empty((group,) + tuple(obs.shape[1:]), dtype=obs.dtype, device=dev)

    def obs_host(sh):
        # the shots' observed data from pinned host memory, one copy per run
        # of consecutive shots
        i = 0
        while i < len(sh):
            j = i + 1
            while j < len(sh) and sh[j] == sh[j - 1] + 1:
                j += 1
            o_d[i:j].copy_(obs_h[sh[i]:sh[j - 1] + 1], non_blocking=True)
            i = j
        return o_d[:len(sh)]

    def e2e_step(k):
        loss, gs = step(k, [m.to(dev, non_blocking=True) for m in ms_h], w_h.to(dev, non_blocking=True), obs_host)
        for gh, g in zip(g_h, gs):
            gh.copy_(g, non_blocking=True)
        float(loss)

    e2e_ms = float("nan")
    if not args.no_e2e:
        for k in range(2):
            e2e_step(k)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(args.steps):
            e2e_step(k)
        e1.record()
        barrier()
        e2e_ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t)

    per_launch_cells = int(np.prod(wl.rt)) * group
    cells = per_launch_cells * wl.nt                  # per rank and step
    value = cells * world / (ms * 1e-3) / 1e9
    e2e_value = cells * world / (e2e_ms * 1e-3) / 1e9
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    rev_launch_ms = rev_ms / wl.nt
    achieved = per_launch_cells * wl.bytes_rev / (rev_launch_ms * 1e-3) / 1e9
    line = {
        "metric": "Gcell-updates/s fwd+adj", "value": value, "unit": "Gcell/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded layered model, see config)",
        "config": dict(wl.config(args), shots_per_step_per_gpu=group,
                       step=f"one FWI gradient step: {group} shot(s) per GPU (forward + adjoint), the "
                            f"survey's shots taken in turn, then one all-reduce of the gradient over the GPUs",
                       parallelism=f"shots: {group} per GPU per step x {world} GPU(s), NCCL all-reduce "
                                   f"of the gradient (weak scaling)",
                       schedule=schedule, memory=solver.last_memory,
                       autotune=None if tune_report is None else
                       {"seconds": tune_report["seconds"], "nt": tune_report["nt"],
                        "trials_ms": {kk: {str(v): 1e3 * t for v, t in r.items()}
                                      for kk, r in tune_report["trials"].items()}}),
        "forward_ms": fwd_ms, "backward_ms": rev_ms,
        "roofline": {"kernel": wl.kernel,
                     "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if pk.exists() else "fallback 6650",
                     "algorithmic_bytes_per_launch": per_launch_cells * wl.bytes_rev,
                     "launch_ms": rev_launch_ms,
                     "launch_ms_how": "CUDA events around the backward call on the launch stream / nt",
                     "traffic": wl.traffic["bytes_per_shot"] * group if wl.traffic else None,
                     "traffic_source": wl.traffic["source"] if wl.traffic else None},
        "forward_roofline": {"achieved": per_launch_cells * wl.bytes_fwd / (fwd_ms / wl.nt * 1e-3) / 1e9,
                             "unit": "GB/s", "bytes_per_cell_step": wl.bytes_fwd},
        "gpu_launches": args.steps * wl.launches(group),
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": "Gcell/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
    }
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        c, s = wl.cpu_run(wl.cpu_nt)
        line["cpu_baseline"] = {"value": c / s / 1e9, "unit": "Gcell/s", "cores": cpu_threads(),
                                "kind": "port",
                                "sample": f"1 of {wl.nshot} shots, first {wl.cpu_nt} of {wl.nt} steps, "
                                          "fwd+adj gradient"}
    if rank == 0 and not args.no_reference_gpu:
        try:
            line["reference_gpu"] = reference_cuda(wl, group, min(wl.nt, wl.ref_gpu_nt), dev)
        except Exception as e:                   # noqa: BLE001
            line["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


# ----------------------------------------------------------------- FWI (C5)
def run_fwi(args):
    """Learned-preconditioned FWI against the plain illumination-preconditioned
    gradient: the U-Net (4 levels, 32 base channels, BF16 tensor-core
    convolutions) is trained on pairs this solver makes from seeded random
    layered models; both FWIs then run from the same smoothed start on a
    held-out model.  value = plain 20-iteration wall time / the learned run's
    wall time to reach the plain run's final data misfit."""
    import torch
    from sweep_b200.precondition import Survey, fwi, layered_model, make_pairs, smooth, train
    from sweep_b200.unet import UNet
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    sv = Survey(device="cuda:0")
    t0 = time.perf_counter()
    xs, ys = make_pairs(sv, args.pairs, seed=SEED)
    torch.cuda.synchronize()
    t_pairs = time.perf_counter() - t0
    net = UNet(base=32, levels=4, seed=0).to(dev)
    t0 = time.perf_counter()
    hist = train(net, xs, ys, steps=args.train_steps, batch=16, lr=1e-3, seed=SEED)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    rng = np.random.default_rng(SEED + 99)
    vt = torch.tensor(layered_model(sv.nz, sv.nx, rng), device=dev)
    v0 = torch.tensor(smooth(vt.cpu().numpy()), device=dev)
    with torch.no_grad():
        obs = sv.model(vt)
    sv.misfit(v0, obs)                                   # warm-up of the solver path
    vp_p, hp, tp, _ = fwi(sv, v0, obs, 20)
    vp_l, hl, tl, nl = fwi(sv, v0, obs, 20, net=net)
    target = hp[-1]
    reach = next((t for f, t in zip(hl[1:], tl) if f <= target), None)
    rms = lambda v: float(((v - vt) ** 2).mean().sqrt())
    line = {
        "metric": "FWI time-to-misfit learned vs plain", "unit": "x (plain time / learned time)",
        "value": (tp[-1] / reach) if reach else None, "higher_is_better": True, "n_gpus": 1,
        "data": "synthetic (seeded random layered models)",
        "config": {"workload": "learned-preconditioned 2-D acoustic FWI, 128x384, dh 10, dt 1 ms, nt 1200, "
                               "8 shots, 20 iterations, 3-point line search",
                   "pairs": args.pairs, "train_steps": args.train_steps, "batch": 16, "lr": 1e-3,
                   "unet": "4 levels, 32 base channels, 3x3 conv, GELU, BF16 / FP32 accumulation"},
        "plain": {"misfit": hp, "seconds": tp, "model_rms": rms(vp_p)},
        "learned": {"misfit": hl, "seconds": tl, "model_rms": rms(vp_l), "learned_steps": nl,
                    "seconds_to_plain_misfit": reach},
        "start_model_rms": rms(v0),
        "train": {"pair_seconds": t_pairs, "train_seconds": t_train, "loss_first": float(np.mean(hist[:50])),
                  "loss_last": float(np.mean(hist[-50:]))},
    }
    print(json.dumps(line))


def relaunch(n):
    """Start n ranks of this same command line under torch.distributed.run
    (one process per GPU, rendezvous on 127.0.0.1) and exit with its status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()),
           *sys.argv[1:]]
    sys.exit(subprocess.call(cmd))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shots-per-call", type=int, default=None,
                    help="acoustic3d: shots per solver call (default 4, what a device tape fits)")
    ap.add_argument("--storage", default="gpu", choices=["gpu", "cpu"],
                    help="acoustic workloads: boundary tape in GPU memory or pinned host memory")
    ap.add_argument("--strip-dtype", default="fp32", choices=["fp32", "fp16", "bf16", "int8"],
                    help="acoustic workloads: boundary strip storage format (fp32 is exact)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the leg that times the reference's own CUDA core (baseline/_ref) on a sample")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end leg (long workloads; the bench line then has no e2e value)")
    ap.add_argument("--pairs", type=int, default=2000, help="fwi workload: training pairs")
    ap.add_argument("--train-steps", type=int, default=20000, help="fwi workload: U-Net training steps")
    ap.add_argument("--workload", default="acoustic3d", choices=sorted(WORKLOADS) + ["fwi"],
                    help="acoustic3d: the 16-shot 256^3 survey (default); acoustic2d: the 32-shot 256x768 "
                         "survey; elastic2d: the 16-shot 400x1200 elastic survey; elastic3d: the 4-shot "
                         "128^3 elastic survey")
    ap.add_argument("--graph-steps", type=int, default=None,
                    help="time steps per captured CUDA graph in the step loops (0: plain stream launches; "
                         "default: the library's built-in choice)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip the launch-schedule autotuner (by default the first call of the workload's "
                         "shape tunes its schedule, before and outside the timed region)")
    ap.add_argument("--order", type=int, default=8,
                    help="spatial order of the acoustic workloads: 8 runs the tiled kernels, the other even "
                         "orders 2-14 the any-order ones (the elastic workloads run order 8 only)")
    ap.add_argument("--nt", type=int, default=None,
                    help="shorter time axis (profiling captures only; the bench line is for the full nt)")
    ap.add_argument("--shots", type=int, default=None,
                    help="fewer shots (profiling captures of a few GB only; the bench line is for the full survey)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        relaunch(args.gpus)
    STRIPS[:] = [args.storage, args.strip_dtype]
    if args.graph_steps is not None:
        os.environ["SWEEP_B200_GRAPH_STEPS"] = str(int(args.graph_steps))
    if args.workload == "fwi":
        run_fwi(args)
        return
    global ORDER
    ORDER = int(args.order)
    wl = WORKLOADS[args.workload]()
    if ORDER != 8:
        # the any-order kernels: one reverse step is adj + recon + strip kernels
        wl.kernel = (f"sweep::aord reverse step at order {ORDER} (adj{2 if wl.name != 'acoustic3d' else 3} + "
                     "recon + strip kernels)")
        wl.traffic = None
    if args.nt:
        wl.nt = int(args.nt)
        global NT, E_NT, A3_NT, E3_NT
        NT, E_NT, A3_NT, E3_NT = wl.nt, wl.nt, wl.nt, wl.nt
    if args.shots:
        wl.nshot = min(int(args.shots), wl.nshot)
    if args.shots_per_call and hasattr(wl, "batch"):
        wl.batch = int(args.shots_per_call)
    if hasattr(wl, "batch"):
        wl.batch = min(wl.batch, wl.nshot)
    if args.impl == "reference":
        run_reference(args, wl)
    else:
        run_gpu(args, wl)


if __name__ == "__main__":
    main()
