"""Generate the golden fixtures under ``tests/golden/`` from the reference itself.

This script imports the reference package (DeepWave-KAUST/sweep) from its
source tree and runs its own compiled path, ``PropTorch(..., impl='c')`` on
the CPU device.  On a CPU device the reference builds its "host core": the
same C++/CUDA kernel sources as its CUDA core compiled by g++ with
``-ffp-contract=off`` (reference ``src/sweep/backend/c/hostcore.py:1-80``),
which the reference's own tests hold to rel < 1e-5 of its CUDA core
(reference ``test/test_host_core.py:250-255``).  The outputs (records and
gradients, float32) are saved as small ``.npz`` files together with every input,
so the parity tests never need the reference at run time.

Usage (with the reference's source tree checked out somewhere)::

    SWEEP_REFERENCE_SRC=<reference checkout>/src \
    TORCH_EXTENSIONS_DIR=<scratch build dir> \
    python tests/golden/make_golden.py [case ...]

``SWEEP_REFERENCE_SRC`` is required.  The reference's own build step (a
one-time g++ build of its host core into ``TORCH_EXTENSIONS_DIR``) runs on
first use.  Nothing here is imported by the library or the tests.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import torch

REF_SRC = os.environ.get("SWEEP_REFERENCE_SRC")
if not REF_SRC:
    sys.exit("make_golden.py: set SWEEP_REFERENCE_SRC to the reference's src directory")
if REF_SRC not in sys.path:
    sys.path.insert(0, REF_SRC)

from sweep.equations import Acoustic, Acoustic3D, Elastic  # noqa: E402
from sweep.propagator.options import BoundarySaving, Ckpt, Full  # noqa: E402
from sweep.propagator.torch import PropTorch  # noqa: E402
from sweep.signal import ricker  # noqa: E402

OUT = Path(__file__).resolve().parent
torch.set_num_threads(max(1, os.cpu_count() or 1))


def _wavelet(nt, dt, f, delay):
    t = np.arange(nt, dtype=np.float64) * dt
    return ricker(t - delay, f).astype(np.float32)


def _layered(nz, nx, rng, vmin, vmax, nlayers):
    """Small layered model: sorted random interface depths, monotone velocities."""
    depths = np.sort(rng.uniform(0, nz, size=nlayers - 1))
    vels = np.linspace(vmin, vmax, nlayers) * (1 + 0.03 * rng.standard_normal(nlayers))
    z = np.arange(nz)[:, None] + 2.0 * np.sin(np.arange(nx)[None, :] * 2 * np.pi / nx * rng.uniform(1, 3))
    idx = np.searchsorted(depths, z)
    return vels[idx].astype(np.float32)


def _run(solver, wavelet, src, rec, models, obs, need_wavelet_grad):
    """Forward plus backward of 0.5 * ||pred - obs||^2, all in float32."""
    models = [torch.tensor(m, requires_grad=True) for m in models]
    w = torch.tensor(wavelet, requires_grad=need_wavelet_grad)
    pred = solver(w, src, rec, models=models)
    loss = 0.5 * ((pred - torch.tensor(obs)) ** 2).sum()
    loss.backward()
    out = {"pred": pred.detach().numpy(), "loss": np.float64(loss.detach())}
    for i, m in enumerate(models):
        out[f"grad{i}"] = m.grad.numpy().copy()
    if need_wavelet_grad:
        out["grad_wavelet"] = w.grad.numpy().copy()
    return out


def _forward(solver, wavelet, src, rec, models):
    with torch.no_grad():
        return solver(torch.tensor(wavelet), src, rec,
                      models=[torch.tensor(m) for m in models]).numpy()


def acoustic2d_c1():
    """The 2-D two-layer case: 96x128, dh 10, dt 2 ms, nt 800, order 8, CPML 20."""
    nz, nx, nt, dt, dh, abcn = 96, 128, 800, 0.002, 10.0, 20
    vp_true = np.full((nz, nx), 1500.0, np.float32)
    vp_true[nz // 2:] = 2500.0
    vp_init = np.full((nz, nx), 1500.0, np.float32)
    w = _wavelet(nt, dt, 10.0, 0.14)
    src = np.array([[32, 48]], np.int64)
    rec = np.array([[[96, 48]]], np.int64)
    res = {}
    for mode, mem in (("bs", BoundarySaving()), ("full", Full())):
        eq = Acoustic(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c",
                           device="cpu", memory=mem)
        obs = _forward(solver, w, src, rec, [vp_true])
        r = _run(solver, w, src, rec, [vp_init], obs, True)
        res[mode] = (obs, r)
    obs, r = res["bs"]
    np.savez_compressed(
        OUT / "acoustic2d_c1.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec,
        obs=obs, pred=r["pred"], loss=r["loss"], grad_vp=r["grad0"],
        grad_wavelet=r["grad_wavelet"],
        grad_vp_full=res["full"][1]["grad0"],
        grad_wavelet_full=res["full"][1]["grad_wavelet"],
    )


def acoustic2d_multi():
    """3 shots of uneven geometry on a layered model, per-shot wavelets,
    receiver lists padded with off-grid coordinates, one source inside the
    boundary-saving restore strip and one receiver in the CPML pad."""
    rng = np.random.default_rng(7)
    nz, nx, nt, dt, dh, abcn = 40, 60, 300, 0.001, 10.0, 10
    vp_true = _layered(nz, nx, rng, 1500.0, 3000.0, 5)
    vp_init = np.full((nz, nx), 1800.0, np.float32) + 20.0 * rng.standard_normal((nz, nx)).astype(np.float32)
    w = np.stack([_wavelet(nt, dt, 15.0, 0.06), _wavelet(nt, dt, 12.0, 0.08),
                  _wavelet(nt, dt, 18.0, 0.05)]).astype(np.float32)
    # (x, z) per shot; shot 1 sits inside the restore strip (z = 2)
    src = np.array([[10, 8], [33, 2], [50, 20]], np.int64)
    nrec = [12, 7, 9]
    nrec_max = max(nrec)
    rec = np.full((3, nrec_max, 2), -1000, np.int64)       # off-grid padding
    for b, n in enumerate(nrec):
        xs = np.sort(rng.choice(np.arange(1, nx - 1), size=n, replace=False))
        rec[b, :n, 0] = xs
        rec[b, :n, 1] = rng.integers(1, nz - 1, size=n)
    rec[2, 0] = (nx + 3, 5)                                 # inside the CPML pad, still on the grid
    res = {}
    for mode, mem in (("bs", BoundarySaving()), ("full", Full()), ("ckpt", Ckpt(chunks=37))):
        eq = Acoustic(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c",
                           device="cpu", memory=mem)
        obs = _forward(solver, w, src, rec, [vp_true])
        r = _run(solver, w, src, rec, [vp_init], obs, True)
        res[mode] = (obs, r)
    obs, r = res["bs"]
    np.savez_compressed(
        OUT / "acoustic2d_multi.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec,
        obs=obs, pred=r["pred"], loss=r["loss"], grad_vp=r["grad0"],
        grad_wavelet=r["grad_wavelet"],
        grad_vp_full=res["full"][1]["grad0"], grad_vp_ckpt=res["ckpt"][1]["grad0"],
    )


def acoustic2d_pershot():
    """Per-shot models (B, nz, nx): each shot propagates in its own model and
    keeps its own gradient."""
    rng = np.random.default_rng(11)
    nz, nx, nt, dt, dh, abcn = 32, 44, 220, 0.001, 10.0, 8
    B = 2
    vp_true = np.stack([_layered(nz, nx, rng, 1500.0, 2800.0, 4) for _ in range(B)])
    vp_init = np.stack([np.full((nz, nx), 1700.0 + 100 * b, np.float32) for b in range(B)])
    w = _wavelet(nt, dt, 15.0, 0.06)
    src = np.array([[12, 6], [30, 10]], np.int64)
    rec = np.array([[[5, 3], [20, 3], [35, 3]], [[8, 25], [22, 25], [40, 25]]], np.int64)
    eq = Acoustic(spatial_order=8, device="cpu")
    solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                       memory=BoundarySaving())
    obs = _forward(solver, w, src, rec, [vp_true])
    r = _run(solver, w, src, rec, [vp_init], obs, False)
    np.savez_compressed(
        OUT / "acoustic2d_pershot.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec,
        obs=obs, pred=r["pred"], loss=r["loss"], grad_vp=r["grad0"],
    )


def acoustic2d_storage():
    """Boundary saving with the strips held as fp16 / bf16 / int8 (reference
    BoundarySaving(storage_dtype=...)): 3 shots on a 48 x 300 layered model, so
    each strip face spans several 256-cell quantisation blocks."""
    rng = np.random.default_rng(23)
    nz, nx, nt, dt, dh, abcn = 48, 300, 300, 0.001, 10.0, 10
    vp_true = _layered(nz, nx, rng, 1500.0, 3200.0, 5)
    vp_init = np.full((nz, nx), 1900.0, np.float32) + 25.0 * rng.standard_normal((nz, nx)).astype(np.float32)
    w = _wavelet(nt, dt, 15.0, 0.06)
    src = np.array([[40, 6], [150, 3], [260, 20]], np.int64)
    rx = np.arange(4, nx - 4, 6)
    rec = np.broadcast_to(np.stack([rx, np.full(rx.size, 2)], -1), (3, rx.size, 2)).copy()
    out = {}
    for sd in ("fp32", "fp16", "bf16", "int8"):
        eq = Acoustic(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                           memory=BoundarySaving(storage_dtype=sd))
        if sd == "fp32":
            obs = _forward(solver, w, src, rec, [vp_true])
        r = _run(solver, w, src, rec, [vp_init], obs, False)
        out[f"grad_vp_{sd}"] = r["grad0"]
        out[f"loss_{sd}"] = r["loss"]
    np.savez_compressed(
        OUT / "acoustic2d_storage.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec, obs=obs, **out,
    )


def acoustic3d_storage():
    """3-D boundary saving with fp16 / bf16 / int8 strips (reference
    BoundarySaving(storage_dtype=...)): 2 shots on a 22 x 20 x 26 model, so the
    six faces span several 256-cell quantisation blocks."""
    rng = np.random.default_rng(29)
    nz, ny, nx, nt, dt, dh, abcn = 22, 20, 26, 160, 0.001, 10.0, 8
    vp_true = np.full((nz, ny, nx), 1800.0, np.float32)
    vp_true[nz // 2:] = 2500.0
    vp_true += (30.0 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    vp_init = np.full((nz, ny, nx), 2000.0, np.float32)
    w = _wavelet(nt, dt, 15.0, 0.06)
    src = np.array([[7, 6, 5], [18, 13, 4]], np.int64)           # (x, y, z)
    rec = np.zeros((2, 8, 3), np.int64)
    for b in range(2):
        rec[b, :, 0] = rng.integers(1, nx - 1, 8)
        rec[b, :, 1] = rng.integers(1, ny - 1, 8)
        rec[b, :, 2] = rng.integers(1, nz - 1, 8)
    out = {}
    for sd in ("fp32", "fp16", "bf16", "int8"):
        eq = Acoustic3D(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, ny, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                           memory=BoundarySaving(storage_dtype=sd))
        if sd == "fp32":
            obs = _forward(solver, w, src, rec, [vp_true])
        r = _run(solver, w, src, rec, [vp_init], obs, False)
        out[f"grad_vp_{sd}"] = r["grad0"]
    np.savez_compressed(
        OUT / "acoustic3d_storage.npz",
        nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec, obs=obs, **out,
    )


def acoustic3d():
    """A small 3-D case: 2 shots, 6 receivers each, order 8, CPML 8."""
    rng = np.random.default_rng(3)
    nz, ny, nx, nt, dt, dh, abcn = 20, 18, 24, 160, 0.001, 10.0, 8
    vp_true = np.full((nz, ny, nx), 1800.0, np.float32)
    vp_true[nz // 2:] = 2600.0
    vp_true += (30.0 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    vp_init = np.full((nz, ny, nx), 2000.0, np.float32)
    w = _wavelet(nt, dt, 15.0, 0.06)
    src = np.array([[6, 5, 4], [17, 12, 3]], np.int64)          # (x, y, z)
    rec = np.zeros((2, 6, 3), np.int64)
    for b in range(2):
        rec[b, :, 0] = rng.integers(1, nx - 1, 6)
        rec[b, :, 1] = rng.integers(1, ny - 1, 6)
        rec[b, :, 2] = rng.integers(1, nz - 1, 6)
    res = {}
    for mode, mem in (("bs", BoundarySaving()), ("full", Full())):
        eq = Acoustic3D(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, ny, nx), dh=dh, dt=dt, abcn=abcn, impl="c",
                           device="cpu", memory=mem)
        obs = _forward(solver, w, src, rec, [vp_true])
        r = _run(solver, w, src, rec, [vp_init], obs, True)
        res[mode] = (obs, r)
    obs, r = res["bs"]
    np.savez_compressed(
        OUT / "acoustic3d.npz",
        nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec,
        obs=obs, pred=r["pred"], loss=r["loss"], grad_vp=r["grad0"],
        grad_wavelet=r["grad_wavelet"], grad_vp_full=res["full"][1]["grad0"],
    )


def elastic2d():
    """Isotropic elastic: 2 explosive shots, (vx, vz) receivers, vp/vs/rho gradients."""
    rng = np.random.default_rng(5)
    nz, nx, nt, dt, dh, abcn = 40, 56, 300, 0.0005, 5.0, 10
    vp_true = _layered(nz, nx, rng, 1800.0, 3200.0, 4)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, nx), 2200.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 25.0, 0.04)
    src = np.array([[14, 6], [40, 9]], np.int64)
    rec = np.zeros((2, 8, 2), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(3, nx - 4, 8).astype(np.int64)
        rec[b, :, 1] = 3 + b
    res = {}
    for mode, mem in (("bs", BoundarySaving()), ("full", Full())):
        eq = Elastic(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c",
                           device="cpu", memory=mem)
        obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
        r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
        res[mode] = (obs, r)
    obs, r = res["bs"]
    np.savez_compressed(
        OUT / "elastic2d.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
        vp_init=vp_init, vs_init=vs_init, rho_init=rho_init,
        wavelet=w, src=src, rec=rec, obs=obs, pred=r["pred"], loss=r["loss"],
        grad_vp=r["grad0"], grad_vs=r["grad1"], grad_rho=r["grad2"],
        grad_vp_full=res["full"][1]["grad0"], grad_vs_full=res["full"][1]["grad1"],
        grad_rho_full=res["full"][1]["grad2"],
    )


def elastic2d_vsrc():
    """Isotropic elastic with body-force (velocity) sources on vx and vz: shot
    0 has its source inside the boundary-strip band and a receiver on the
    source cell; (vx, vz, sxx) receivers; vp/vs/rho gradients."""
    rng = np.random.default_rng(11)
    nz, nx, nt, dt, dh, abcn = 40, 56, 300, 0.0005, 5.0, 10
    vp_true = _layered(nz, nx, rng, 1800.0, 3200.0, 4)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, nx), 2200.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 25.0, 0.04)
    src = np.array([[14, 2], [40, 9]], np.int64)
    rec = np.zeros((2, 8, 2), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(3, nx - 4, 8).astype(np.int64)
        rec[b, :, 1] = 3 + b
    rec[0, 0] = (14, 2)                       # a receiver on shot 0's source cell
    eq = Elastic(spatial_order=8, device="cpu")
    solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                       memory=BoundarySaving(), source_type=["vx", "vz"], receiver_type=["vx", "vz", "sxx"])
    obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
    r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
    np.savez_compressed(
        OUT / "elastic2d_vsrc.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
        vp_init=vp_init, vs_init=vs_init, rho_init=rho_init,
        wavelet=w, src=src, rec=rec, obs=obs, pred=r["pred"], loss=r["loss"],
        grad_vp=r["grad0"], grad_vs=r["grad1"], grad_rho=r["grad2"],
    )


def elastic2d_storage():
    """Elastic boundary saving with fp16 / bf16 / int8 strips (reference
    BoundarySaving(storage_dtype=...): each of the five fields quantised per
    band on its own): 2 explosive shots on a 40 x 120 layered model."""
    rng = np.random.default_rng(31)
    nz, nx, nt, dt, dh, abcn = 40, 120, 300, 0.0005, 5.0, 10
    vp_true = _layered(nz, nx, rng, 1800.0, 3200.0, 4)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, nx), 2200.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 25.0, 0.04)
    src = np.array([[30, 6], [90, 9]], np.int64)
    rec = np.zeros((2, 12, 2), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(3, nx - 4, 12).astype(np.int64)
        rec[b, :, 1] = 3 + b
    out = {}
    for sd in ("fp32", "fp16", "bf16", "int8"):
        eq = Elastic(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                           memory=BoundarySaving(storage_dtype=sd))
        if sd == "fp32":
            obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
        r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
        for i, name in enumerate(("vp", "vs", "rho")):
            out[f"grad_{name}_{sd}"] = r[f"grad{i}"]
    np.savez_compressed(
        OUT / "elastic2d_storage.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
        vp_init=vp_init, vs_init=vs_init, rho_init=rho_init,
        wavelet=w, src=src, rec=rec, obs=obs, **out,
    )


def acoustic2d_free_surface():
    """2-D free surface (reference PropTorch(free_surface=True): no PML on the
    top face): 2 shots near the surface, receivers on the surface rows, a
    layered model; boundary saving and full modes, wavelet gradient."""
    rng = np.random.default_rng(37)
    nz, nx, nt, dt, dh, abcn = 48, 90, 500, 0.001, 10.0, 12
    vp_true = _layered(nz, nx, rng, 1500.0, 3000.0, 5)
    vp_init = np.full((nz, nx), 1800.0, np.float32) + 20.0 * rng.standard_normal((nz, nx)).astype(np.float32)
    w = np.stack([_wavelet(nt, dt, 15.0, 0.06), _wavelet(nt, dt, 12.0, 0.08)]).astype(np.float32)
    src = np.array([[20, 2], [70, 0]], np.int64)
    rx = np.arange(2, nx - 2, 5)
    rec = np.broadcast_to(np.stack([rx, np.full(rx.size, 1)], -1), (2, rx.size, 2)).copy()
    res = {}
    for mode, mem in (("bs", BoundarySaving()), ("full", Full())):
        eq = Acoustic(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                           memory=mem, free_surface=True)
        obs = _forward(solver, w, src, rec, [vp_true])
        r = _run(solver, w, src, rec, [vp_init], obs, True)
        res[mode] = (obs, r)
    obs, r = res["bs"]
    np.savez_compressed(
        OUT / "acoustic2d_free_surface.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec,
        obs=obs, pred=r["pred"], loss=r["loss"], grad_vp=r["grad0"], grad_wavelet=r["grad_wavelet"],
        grad_vp_full=res["full"][1]["grad0"],
    )


def acoustic2d_free_faces():
    """2-D per-face free surfaces (reference PropTorch(free_surface=[...])):
    ['bottom', 'right'] and ['top', 'left'], one shot each near the free
    faces, receivers along them."""
    rng = np.random.default_rng(43)
    nz, nx, nt, dt, dh, abcn = 40, 64, 400, 0.001, 10.0, 10
    vp_true = _layered(nz, nx, rng, 1500.0, 2800.0, 4)
    vp_init = np.full((nz, nx), 1800.0, np.float32) + 20.0 * rng.standard_normal((nz, nx)).astype(np.float32)
    w = _wavelet(nt, dt, 15.0, 0.06)
    out = {}
    for tag, faces, src, rec in (
            ("br", ["bottom", "right"], [[50, 30]], [[[60, z] for z in range(4, 38, 3)]]),
            ("tl", ["top", "left"], [[8, 3]], [[[x, 1] for x in range(2, 60, 4)]])):
        src = np.array(src, np.int64)
        rec = np.array(rec, np.int64)
        eq = Acoustic(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                           memory=BoundarySaving(), free_surface=faces)
        obs = _forward(solver, w, src, rec, [vp_true])
        r = _run(solver, w, src, rec, [vp_init], obs, True)
        out.update({f"src_{tag}": src, f"rec_{tag}": rec, f"obs_{tag}": obs, f"pred_{tag}": r["pred"],
                    f"grad_vp_{tag}": r["grad0"], f"grad_wavelet_{tag}": r["grad_wavelet"]})
    np.savez_compressed(
        OUT / "acoustic2d_free_faces.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, **out,
    )


def acoustic3d_free_surface():
    """3-D free surface: 2 shots just under the surface, receivers on it."""
    rng = np.random.default_rng(41)
    nz, ny, nx, nt, dt, dh, abcn = 20, 18, 24, 180, 0.001, 10.0, 8
    vp_true = np.full((nz, ny, nx), 1800.0, np.float32)
    vp_true[nz // 2:] = 2600.0
    vp_true += (30.0 * rng.standard_normal((nz, ny, nx))).astype(np.float32)
    vp_init = np.full((nz, ny, nx), 2000.0, np.float32)
    w = _wavelet(nt, dt, 15.0, 0.06)
    src = np.array([[6, 5, 1], [17, 12, 2]], np.int64)          # (x, y, z)
    rec = np.zeros((2, 8, 3), np.int64)
    for b in range(2):
        rec[b, :, 0] = rng.integers(1, nx - 1, 8)
        rec[b, :, 1] = rng.integers(1, ny - 1, 8)
        rec[b, :, 2] = 0
    eq = Acoustic3D(spatial_order=8, device="cpu")
    solver = PropTorch(eq, shape=(nz, ny, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                       memory=BoundarySaving(), free_surface=True)
    obs = _forward(solver, w, src, rec, [vp_true])
    r = _run(solver, w, src, rec, [vp_init], obs, True)
    np.savez_compressed(
        OUT / "acoustic3d_free_surface.npz",
        nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec,
        obs=obs, pred=r["pred"], loss=r["loss"], grad_vp=r["grad0"], grad_wavelet=r["grad_wavelet"],
    )


def _illum_model(shape):
    """Ramp plus bump (the heterogeneous model of the reference's illumination
    pins, test/test_illumination_pin.py:30-35)."""
    idx = np.indices(shape).astype(np.float32)
    bump = sum((i - n / 2) ** 2 / n for i, n in zip(idx, shape))
    return (2500.0 + 4.0 * idx[0] + 60.0 * np.sin(bump)).astype(np.float32)


def _illum_case(cls, shape, src, rec, nt, dt, dh, abcn):
    """Gradient with solver.compute_illumination = True in boundary-saving and
    full modes, plus the boundary-saving gradient with illumination off."""
    vp_true = _illum_model(shape)
    vp_init = (0.97 * vp_true).astype(np.float32)
    w = _wavelet(nt, dt, 15.0, 0.05)
    out = {}
    obs = None
    for tag, mem, illum in (("bs", BoundarySaving(), True), ("full", Full(), True),
                            ("off", BoundarySaving(), False)):
        solver = PropTorch(cls(spatial_order=8, device="cpu"), shape=shape, dh=dh, dt=dt, abcn=abcn,
                           impl="c", device="cpu", memory=mem)
        if obs is None:
            obs = _forward(solver, w, src, rec, [vp_true])
        solver.compute_illumination = illum
        r = _run(solver, w, src, rec, [vp_init], obs, False)
        out[f"pred_{tag}"] = r["pred"]
        out[f"grad_vp_{tag}"] = r["grad0"]
        if illum:
            out[f"src_illum_{tag}"] = solver.source_illumination.detach().numpy().copy()
            out[f"rec_illum_{tag}"] = solver.receiver_illumination.detach().numpy().copy()
    return dict(vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec, obs=obs, **out)


def acoustic2d_illum():
    """Source / receiver illumination (solver.compute_illumination = True) in
    2-D: 2 shots on an 80 x 100 ramp-plus-bump model, boundary saving and full."""
    nz, nx, nt, dt, dh, abcn = 80, 100, 260, 0.0012, 10.0, 8
    src = np.array([[nx // 2, nz // 3], [20, 10]], np.int64)
    rx = np.arange(4, nx - 4, 4, dtype=np.int64)
    rec = np.broadcast_to(np.stack([rx, np.full(rx.size, 4)], -1), (2, rx.size, 2)).copy()
    d = _illum_case(Acoustic, (nz, nx), src, rec, nt, dt, dh, abcn)
    np.savez_compressed(OUT / "acoustic2d_illum.npz", nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn,
                        order=8, **d)


def acoustic3d_illum():
    """Source / receiver illumination in 3-D: one shot on a 30 x 28 x 34
    ramp-plus-bump model, boundary saving and full."""
    nz, ny, nx, nt, dt, dh, abcn = 30, 28, 34, 160, 0.0012, 10.0, 8
    src = np.array([[nx // 2, ny // 2, nz // 3]], np.int64)
    rx = np.arange(4, nx - 4, 4, dtype=np.int64)
    rec = np.stack([rx, np.full(rx.size, ny // 2), np.full(rx.size, 4)], -1)[None]
    d = _illum_case(Acoustic3D, (nz, ny, nx), src, rec, nt, dt, dh, abcn)
    np.savez_compressed(OUT / "acoustic3d_illum.npz", nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh,
                        abcn=abcn, order=8, **d)


def acoustic3d_clean():
    """A 3-D grid whose clear box is wider than one 32 x 8 column block in x
    and y (64 x 72 x 96, CPML 8): split into z chunks, the stencil kernels'
    CTAs clear of the CPML shell take their clean path.  2 shots inside the
    volume, 24 receivers spread through it; boundary saving."""
    rng = np.random.default_rng(53)
    nz, ny, nx, nt, dt, dh, abcn = 64, 72, 96, 220, 0.001, 10.0, 8
    zz = (np.arange(nz)[:, None, None] + 3.0 * np.sin(np.arange(nx)[None, None, :] * 2 * np.pi / nx)
          + 2.0 * np.cos(np.arange(ny)[None, :, None] * 2 * np.pi / ny))
    vp_true = np.where(zz < nz / 2, 1800.0, 2600.0) + np.zeros((nz, ny, nx))
    vp_true = np.where((zz > 0.7 * nz) & (np.arange(nx)[None, None, :] > nx / 3), 2300.0, vp_true)
    vp_true = vp_true.astype(np.float32)
    vp_init = np.full((nz, ny, nx), 2100.0, np.float32)
    w = np.stack([_wavelet(nt, dt, 15.0, 0.06), _wavelet(nt, dt, 12.0, 0.07)]).astype(np.float32)
    src = np.array([[48, 36, 20], [30, 44, 40]], np.int64)          # (x, y, z)
    rec = np.zeros((2, 24, 3), np.int64)
    for b in range(2):
        rec[b, :, 0] = rng.integers(2, nx - 2, 24)
        rec[b, :, 1] = rng.integers(2, ny - 2, 24)
        rec[b, :, 2] = rng.integers(2, nz - 2, 24)
    eq = Acoustic3D(spatial_order=8, device="cpu")
    solver = PropTorch(eq, shape=(nz, ny, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                       memory=BoundarySaving())
    obs = _forward(solver, w, src, rec, [vp_true])
    r = _run(solver, w, src, rec, [vp_init], obs, True)
    np.savez_compressed(
        OUT / "acoustic3d_clean.npz",
        nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec,
        obs=obs, pred=r["pred"], loss=r["loss"], grad_vp=r["grad0"], grad_wavelet=r["grad_wavelet"],
    )


def acoustic2d_many():
    """20 shots of uneven geometry (per-shot wavelets, 5-30 receivers each
    padded with off-grid coordinates, sources at several depths) on a
    64 x 160 layered model: enough shots to fill 8- and 16-shot CTA groups."""
    rng = np.random.default_rng(59)
    nz, nx, nt, dt, dh, abcn = 64, 160, 300, 0.001, 10.0, 12
    B = 20
    vp_true = _layered(nz, nx, rng, 1500.0, 3200.0, 6)
    vp_init = np.full((nz, nx), 1900.0, np.float32) + 20.0 * rng.standard_normal((nz, nx)).astype(np.float32)
    w = np.stack([_wavelet(nt, dt, rng.uniform(10, 20), rng.uniform(0.05, 0.09)) for _ in range(B)])
    w = w.astype(np.float32)
    src = np.stack([rng.integers(2, nx - 2, B), rng.integers(1, nz // 3, B)], -1).astype(np.int64)
    nrec = rng.integers(5, 31, B)
    rec = np.full((B, int(nrec.max()), 2), -1000, np.int64)
    for b, n in enumerate(nrec):
        rec[b, :n, 0] = np.sort(rng.choice(np.arange(1, nx - 1), size=n, replace=False))
        rec[b, :n, 1] = rng.integers(1, nz - 1, size=n)
    eq = Acoustic(spatial_order=8, device="cpu")
    solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                       memory=BoundarySaving())
    obs = _forward(solver, w, src, rec, [vp_true])
    r = _run(solver, w, src, rec, [vp_init], obs, True)
    np.savez_compressed(
        OUT / "acoustic2d_many.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vp_init=vp_init, wavelet=w, src=src, rec=rec,
        obs=obs, pred=r["pred"], loss=r["loss"], grad_vp=r["grad0"], grad_wavelet=r["grad_wavelet"],
    )


def elastic2d_interior():
    """Isotropic elastic on a 120 x 170 model (CPML 10): the runtime grid has
    32 x 32 tiles clear of the CPML band.  4 explosive shots, (vx, vz)
    receivers; vp/vs/rho gradients, boundary saving."""
    rng = np.random.default_rng(61)
    nz, nx, nt, dt, dh, abcn = 120, 170, 320, 0.0005, 5.0, 10
    vp_true = _layered(nz, nx, rng, 1800.0, 3200.0, 5)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, nx), 2300.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 25.0, 0.04)
    src = np.array([[30, 40], [85, 60], [140, 30], [60, 90]], np.int64)
    rec = np.zeros((4, 20, 2), np.int64)
    for b in range(4):
        rec[b, :, 0] = np.linspace(3, nx - 4, 20).astype(np.int64)
        rec[b, :, 1] = 3 + 20 * b
    eq = Elastic(spatial_order=8, device="cpu")
    solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                       memory=BoundarySaving())
    obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
    r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
    np.savez_compressed(
        OUT / "elastic2d_interior.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
        vp_init=vp_init, vs_init=vs_init, rho_init=rho_init,
        wavelet=w, src=src, rec=rec, obs=obs, pred=r["pred"], loss=r["loss"],
        grad_vp=r["grad0"], grad_vs=r["grad1"], grad_rho=r["grad2"],
    )


def elastic2d_free_surface():
    """Isotropic elastic with a traction-free top face (reference
    PropTorch(free_surface=True): no PML on top, the image method of
    elastic_free_surface.cuh, the Robertsson sxx correction and szz = 0 on the
    surface row).  2 explosive shots (one on the surface row, one 3 cells
    below it); shot 0 records (vx, vz) on the surface row, shot 1 at depth
    1 and 5; vp/vs/rho gradients, boundary saving and checkpoints."""
    rng = np.random.default_rng(71)
    nz, nx, nt, dt, dh, abcn = 40, 56, 300, 0.0005, 5.0, 10
    vp_true = _layered(nz, nx, rng, 1800.0, 3200.0, 4)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, nx), 2200.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 25.0, 0.04)
    src = np.array([[14, 0], [40, 3]], np.int64)
    rec = np.zeros((2, 8, 2), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(3, nx - 4, 8).astype(np.int64)
    rec[0, :, 1] = 0
    rec[1, :4, 1] = 1
    rec[1, 4:, 1] = 5
    res = {}
    for mode, mem in (("bs", BoundarySaving()), ("ckpt", Ckpt(chunks=7))):
        eq = Elastic(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c",
                           device="cpu", memory=mem, free_surface=True)
        obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
        r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
        res[mode] = (obs, r)
    obs, r = res["bs"]
    np.savez_compressed(
        OUT / "elastic2d_free_surface.npz",
        nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
        vp_init=vp_init, vs_init=vs_init, rho_init=rho_init,
        wavelet=w, src=src, rec=rec, obs=obs, pred=r["pred"], loss=r["loss"],
        grad_vp=r["grad0"], grad_vs=r["grad1"], grad_rho=r["grad2"],
        grad_vp_ckpt=res["ckpt"][1]["grad0"], grad_vs_ckpt=res["ckpt"][1]["grad1"],
        grad_rho_ckpt=res["ckpt"][1]["grad2"],
    )


def elastic2d_free_faces():
    """Isotropic elastic with traction-free faces other than the top
    (reference PropTorch(free_surface=[...]) per edge): ['bottom', 'right']
    (the high-side images, zeroed shear on the surface row / column),
    ['top', 'left'] and all four faces (corners where two surfaces meet).
    One explosive shot near a corner, one in the middle; (vx, vz, sxx)
    receivers on the surface rows and columns; vp/vs/rho gradients, boundary
    saving."""
    rng = np.random.default_rng(83)
    nz, nx, nt, dt, dh, abcn = 36, 48, 260, 0.0005, 5.0, 8
    vp_true = _layered(nz, nx, rng, 1800.0, 3000.0, 4)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, nx), 2200.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 25.0, 0.04)
    src = np.array([[nx - 3, nz - 2], [20, 15]], np.int64)
    rec = np.zeros((2, 12, 2), np.int64)
    for b in range(2):
        rec[b, :6, 0] = np.linspace(0, nx - 1, 6).astype(np.int64)
        rec[b, :6, 1] = nz - 1 if b == 0 else 0
        rec[b, 6:, 0] = nx - 1 if b == 0 else 0
        rec[b, 6:, 1] = np.linspace(1, nz - 2, 6).astype(np.int64)
    out = dict(nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
               vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
               vp_init=vp_init, vs_init=vs_init, rho_init=rho_init, wavelet=w, src=src, rec=rec)
    for tag, faces in (("br", ["bottom", "right"]), ("tl", ["top", "left"]),
                       ("all", ["top", "bottom", "left", "right"])):
        eq = Elastic(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                           memory=BoundarySaving(), free_surface=faces,
                           receiver_type=["vx", "vz", "sxx"])
        obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
        r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
        out.update({f"obs_{tag}": obs, f"pred_{tag}": r["pred"], f"loss_{tag}": r["loss"],
                    f"grad_vp_{tag}": r["grad0"], f"grad_vs_{tag}": r["grad1"], f"grad_rho_{tag}": r["grad2"]})
    np.savez_compressed(OUT / "elastic2d_free_faces.npz", **out)


def elastic3d():
    """3-D isotropic elastic (reference sweep.equations.Elastic3D, order 8):
    2 explosive shots on a 20 x 22 x 24 layered model (CPML 6), (vx, vy, vz)
    receivers, vp/vs/rho gradients, boundary saving; a third run with
    body-force sources on (vx, vz) and (vx, vz, syy) receivers."""
    from sweep.equations import Elastic3D
    rng = np.random.default_rng(91)
    nz, ny, nx, nt, dt, dh, abcn = 20, 22, 24, 160, 0.0005, 5.0, 6
    base = _layered(nz, nx, rng, 1900.0, 3000.0, 3)
    vp_true = np.ascontiguousarray(np.repeat(base[:, None, :], ny, axis=1)
                                   * (1 + 0.02 * np.sin(np.arange(ny) / 3.0))[None, :, None]).astype(np.float32)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, ny, nx), 2300.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 30.0, 0.03)
    src = np.array([[8, 10, 6], [16, 12, 13]], np.int64)            # (x, y, z)
    rec = np.zeros((2, 10, 3), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(1, nx - 2, 10).astype(np.int64)
        rec[b, :, 1] = np.linspace(2, ny - 3, 10).astype(np.int64)
        rec[b, :, 2] = 2 + 3 * b
    out = dict(nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
               vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
               vp_init=vp_init, vs_init=vs_init, rho_init=rho_init, wavelet=w, src=src, rec=rec)
    for tag, kw in (("", {}), ("_vsrc", dict(source_type=["vx", "vz"], receiver_type=["vx", "vz", "syy"]))):
        eq = Elastic3D(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, ny, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                           memory=BoundarySaving(), **kw)
        obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
        r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
        out.update({f"obs{tag}": obs, f"pred{tag}": r["pred"], f"loss{tag}": r["loss"],
                    f"grad_vp{tag}": r["grad0"], f"grad_vs{tag}": r["grad1"], f"grad_rho{tag}": r["grad2"]})
    np.savez_compressed(OUT / "elastic3d.npz", **out)


def elastic3d_free_surface():
    """3-D isotropic elastic with a traction-free top face (reference
    Elastic3D, PropTorch(free_surface=True): no PML on top, the full stencil
    over image values, Robertsson sxx / syy and szz = 0 on the surface row).
    2 explosive shots, one on the surface row; (vx, vy, vz, sxx) receivers on
    the surface row and two rows below; vp/vs/rho gradients."""
    from sweep.equations import Elastic3D
    rng = np.random.default_rng(97)
    nz, ny, nx, nt, dt, dh, abcn = 18, 20, 22, 150, 0.0005, 5.0, 6
    base = _layered(nz, nx, rng, 1900.0, 3000.0, 3)
    vp_true = np.ascontiguousarray(np.repeat(base[:, None, :], ny, axis=1)
                                   * (1 + 0.02 * np.cos(np.arange(ny) / 4.0))[None, :, None]).astype(np.float32)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, ny, nx), 2300.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 30.0, 0.03)
    src = np.array([[8, 9, 0], [14, 11, 3]], np.int64)               # (x, y, z)
    rec = np.zeros((2, 10, 3), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(1, nx - 2, 10).astype(np.int64)
        rec[b, :, 1] = np.linspace(2, ny - 3, 10).astype(np.int64)
        rec[b, :, 2] = 2 * b
    eq = Elastic3D(spatial_order=8, device="cpu")
    solver = PropTorch(eq, shape=(nz, ny, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                       memory=BoundarySaving(), free_surface=True, receiver_type=["vx", "vy", "vz", "sxx"])
    obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
    r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
    np.savez_compressed(
        OUT / "elastic3d_free_surface.npz",
        nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
        vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
        vp_init=vp_init, vs_init=vs_init, rho_init=rho_init, wavelet=w, src=src, rec=rec,
        obs=obs, pred=r["pred"], loss=r["loss"], grad_vp=r["grad0"], grad_vs=r["grad1"], grad_rho=r["grad2"],
    )


def acoustic_orders():
    """Spatial orders other than 8 (the reference's Acoustic / Acoustic3D
    default to order 4): 2-D at orders 2, 4, 6 and 12 (2 shots on a 40 x 60
    layered model, CPML 10, a source inside the restore strip), 3-D at orders
    4 and 6 (2 shots on a 16 x 18 x 20 model, CPML 6); records, vp and wavelet
    gradients, boundary saving."""
    rng = np.random.default_rng(211)
    nz, nx, nt, dt, dh, abcn = 40, 60, 300, 0.001, 10.0, 10
    vp_true = _layered(nz, nx, rng, 1500.0, 3000.0, 4)
    vp_init = np.full((nz, nx), 1900.0, np.float32)
    w = np.stack([_wavelet(nt, dt, 15.0, 0.06), _wavelet(nt, dt, 12.0, 0.07)]).astype(np.float32)
    src = np.array([[12, 9], [40, 2]], np.int64)                 # (x, z); shot 1 in the restore strip
    rec = np.zeros((2, 10, 2), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(2, nx - 3, 10).astype(np.int64)
        rec[b, :, 1] = 3 + 5 * b
    out = dict(nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, vp_true=vp_true, vp_init=vp_init,
               wavelet=w, src=src, rec=rec)
    for order in (2, 4, 6, 12):
        solver = PropTorch(Acoustic(spatial_order=order, device="cpu"), shape=(nz, nx), dh=dh, dt=dt,
                           abcn=abcn, impl="c", device="cpu", memory=BoundarySaving())
        obs = _forward(solver, w, src, rec, [vp_true])
        r = _run(solver, w, src, rec, [vp_init], obs, True)
        out.update({f"obs_o{order}": obs, f"pred_o{order}": r["pred"], f"grad_vp_o{order}": r["grad0"],
                    f"grad_wavelet_o{order}": r["grad_wavelet"]})
    rng = np.random.default_rng(212)
    nz3, ny3, nx3, nt3, dt3, abcn3 = 16, 18, 20, 150, 0.001, 6
    vp3_true = np.full((nz3, ny3, nx3), 1800.0, np.float32)
    vp3_true[nz3 // 2:] = 2500.0
    vp3_true += (25.0 * rng.standard_normal((nz3, ny3, nx3))).astype(np.float32)
    vp3_init = np.full((nz3, ny3, nx3), 2000.0, np.float32)
    w3 = _wavelet(nt3, dt3, 15.0, 0.06)
    src3 = np.array([[5, 6, 4], [14, 11, 1]], np.int64)          # (x, y, z)
    rec3 = np.zeros((2, 6, 3), np.int64)
    for b in range(2):
        rec3[b, :, 0] = rng.integers(1, nx3 - 1, 6)
        rec3[b, :, 1] = rng.integers(1, ny3 - 1, 6)
        rec3[b, :, 2] = rng.integers(1, nz3 - 1, 6)
    out.update(nz3=nz3, ny3=ny3, nx3=nx3, nt3=nt3, dt3=dt3, abcn3=abcn3, vp3_true=vp3_true, vp3_init=vp3_init,
               wavelet3=w3, src3=src3, rec3=rec3)
    for order in (4, 6):
        solver = PropTorch(Acoustic3D(spatial_order=order, device="cpu"), shape=(nz3, ny3, nx3), dh=dh, dt=dt3,
                           abcn=abcn3, impl="c", device="cpu", memory=BoundarySaving())
        obs = _forward(solver, w3, src3, rec3, [vp3_true])
        r = _run(solver, w3, src3, rec3, [vp3_init], obs, True)
        out.update({f"obs3_o{order}": obs, f"pred3_o{order}": r["pred"], f"grad3_vp_o{order}": r["grad0"],
                    f"grad3_wavelet_o{order}": r["grad_wavelet"]})
    np.savez_compressed(OUT / "acoustic_orders.npz", **out)


def elastic_orders():
    """2-D isotropic elastic at spatial orders 2, 4 and 6 (the reference's
    Elastic defaults to order 4): 2 explosive shots on a 40 x 56 layered model
    (CPML 10), (vx, vz) receivers, vp/vs/rho gradients; order 4 once more with
    a traction-free top face, a shot on the surface row and (vx, vz, sxx)
    receivers on it and below it."""
    rng = np.random.default_rng(223)
    nz, nx, nt, dt, dh, abcn = 40, 56, 300, 0.0005, 5.0, 10
    vp_true = _layered(nz, nx, rng, 1800.0, 3200.0, 4)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, nx), 2200.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 25.0, 0.04)
    src = np.array([[14, 6], [40, 0]], np.int64)                 # shot 1 on the surface row
    rec = np.zeros((2, 8, 2), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(3, nx - 4, 8).astype(np.int64)
        rec[b, :, 1] = 2 * b
    out = dict(nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
               vp_init=vp_init, vs_init=vs_init, rho_init=rho_init, wavelet=w, src=src, rec=rec)
    runs = [(f"o{o}", o, {}) for o in (2, 4, 6)]
    runs.append(("o4_fs", 4, dict(free_surface=True, receiver_type=["vx", "vz", "sxx"])))
    for tag, order, kw in runs:
        solver = PropTorch(Elastic(spatial_order=order, device="cpu"), shape=(nz, nx), dh=dh, dt=dt, abcn=abcn,
                           impl="c", device="cpu", memory=BoundarySaving(), **kw)
        obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
        r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
        out.update({f"obs_{tag}": obs, f"pred_{tag}": r["pred"], f"grad_vp_{tag}": r["grad0"],
                    f"grad_vs_{tag}": r["grad1"], f"grad_rho_{tag}": r["grad2"]})
    np.savez_compressed(OUT / "elastic_orders.npz", **out)


def elastic3d_orders():
    """3-D isotropic elastic at spatial orders 2, 4 and 6 (the reference's
    Elastic3D defaults to order 4): 2 explosive shots on an 18 x 20 x 22
    layered model (CPML 6), (vx, vy, vz) receivers, vp/vs/rho gradients;
    order 4 once more with a traction-free top face and a shot on it."""
    from sweep.equations import Elastic3D
    rng = np.random.default_rng(227)
    nz, ny, nx, nt, dt, dh, abcn = 18, 20, 22, 140, 0.0005, 5.0, 6
    base = _layered(nz, nx, rng, 1900.0, 3000.0, 3)
    vp_true = np.ascontiguousarray(np.repeat(base[:, None, :], ny, axis=1)
                                   * (1 + 0.02 * np.sin(np.arange(ny) / 3.0))[None, :, None]).astype(np.float32)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, ny, nx), 2300.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 30.0, 0.03)
    src = np.array([[8, 9, 5], [14, 11, 0]], np.int64)              # (x, y, z); shot 1 on the top row
    rec = np.zeros((2, 10, 3), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(1, nx - 2, 10).astype(np.int64)
        rec[b, :, 1] = np.linspace(2, ny - 3, 10).astype(np.int64)
        rec[b, :, 2] = 2 * b
    out = dict(nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, vp_true=vp_true, vs_true=vs_true,
               rho_true=rho_true, vp_init=vp_init, vs_init=vs_init, rho_init=rho_init, wavelet=w, src=src, rec=rec)
    runs = [(f"o{o}", o, {}) for o in (2, 4, 6)] + [("o4_fs", 4, dict(free_surface=True))]
    for tag, order, kw in runs:
        solver = PropTorch(Elastic3D(spatial_order=order, device="cpu"), shape=(nz, ny, nx), dh=dh, dt=dt,
                           abcn=abcn, impl="c", device="cpu", memory=BoundarySaving(), **kw)
        obs = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
        r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], obs, False)
        out.update({f"obs_{tag}": obs, f"pred_{tag}": r["pred"], f"grad_vp_{tag}": r["grad0"],
                    f"grad_vs_{tag}": r["grad1"], f"grad_rho_{tag}": r["grad2"]})
    np.savez_compressed(OUT / "elastic3d_orders.npz", **out)


def vti2d():
    """First-order acoustic VTI (reference sweep.equations.AcousticVTI1st,
    Duveneck et al. 2008; vx, vz, sH, sV on a staggered grid): 2 shots on a
    40 x 56 layered model (CPML 10) with Thomsen epsilon / delta layers, the
    default sources (sH, sV) and receivers (vz), vp / epsilon / delta / rho
    gradients, boundary saving, at orders 8 and 4; at order 8 once more with
    (vx, vz, sH) receivers and a second model set per shot."""
    from sweep.equations.acoustic_vti_1st import AcousticVTI1st
    rng = np.random.default_rng(229)
    nz, nx, nt, dt, dh, abcn = 40, 56, 300, 0.0005, 5.0, 10
    vp_true = _layered(nz, nx, rng, 1800.0, 3200.0, 4)
    eps_true = (0.05 + 0.1 * (vp_true - 1800.0) / 1400.0).astype(np.float32)
    dlt_true = (0.5 * eps_true).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, nx), 2300.0, np.float32)
    eps_init = np.full((nz, nx), 0.1, np.float32)
    dlt_init = np.full((nz, nx), 0.05, np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 25.0, 0.04)
    src = np.array([[14, 6], [40, 9]], np.int64)
    rec = np.zeros((2, 8, 2), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(3, nx - 4, 8).astype(np.int64)
        rec[b, :, 1] = 3 + b
    names = ("vp", "eps", "dlt", "rho")
    true = [vp_true, eps_true, dlt_true, rho_true]
    init = [vp_init, eps_init, dlt_init, rho_init]
    out = dict(nz=nz, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, wavelet=w, src=src, rec=rec,
               **{f"{n}_true": m for n, m in zip(names, true)}, **{f"{n}_init": m for n, m in zip(names, init)})
    for tag, order, kw in (("o8", 8, {}), ("o4", 4, {}), ("o8_rec", 8, dict(receiver_type=["vx", "vz", "sH"]))):
        solver = PropTorch(AcousticVTI1st(spatial_order=order, device="cpu"), shape=(nz, nx), dh=dh, dt=dt,
                           abcn=abcn, impl="c", device="cpu", memory=BoundarySaving(), **kw)
        obs = _forward(solver, w, src, rec, true)
        r = _run(solver, w, src, rec, init, obs, False)
        out.update({f"obs_{tag}": obs, f"pred_{tag}": r["pred"]})
        out.update({f"grad_{n}_{tag}": r[f"grad{i}"] for i, n in enumerate(names)})
    np.savez_compressed(OUT / "vti2d.npz", **out)


def vti3d():
    """3-D first-order acoustic VTI (reference AcousticVTI1st3D; vx, vy, vz,
    sH, sV): 2 shots on an 18 x 20 x 22 layered model (CPML 6) with Thomsen
    epsilon / delta layers, the default sources (sH, sV) and receivers (vz),
    vp / epsilon / delta / rho gradients, boundary saving, at orders 4 (the
    reference's default) and 8; at order 4 once more with (vx, vy, sH)
    receivers."""
    from sweep.equations.acoustic_vti_1st import AcousticVTI1st3D
    rng = np.random.default_rng(233)
    nz, ny, nx, nt, dt, dh, abcn = 18, 20, 22, 140, 0.0005, 5.0, 6
    base = _layered(nz, nx, rng, 1800.0, 3000.0, 3)
    vp_true = np.ascontiguousarray(np.repeat(base[:, None, :], ny, axis=1)
                                   * (1 + 0.02 * np.sin(np.arange(ny) / 3.0))[None, :, None]).astype(np.float32)
    eps_true = (0.05 + 0.1 * (vp_true - 1800.0) / 1200.0).astype(np.float32)
    dlt_true = (0.5 * eps_true).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, ny, nx), 2300.0, np.float32)
    eps_init = np.full((nz, ny, nx), 0.1, np.float32)
    dlt_init = np.full((nz, ny, nx), 0.05, np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 30.0, 0.03)
    src = np.array([[8, 9, 5], [14, 11, 7]], np.int64)              # (x, y, z)
    rec = np.zeros((2, 10, 3), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(1, nx - 2, 10).astype(np.int64)
        rec[b, :, 1] = np.linspace(2, ny - 3, 10).astype(np.int64)
        rec[b, :, 2] = 2 + b
    names = ("vp", "eps", "dlt", "rho")
    true = [vp_true, eps_true, dlt_true, rho_true]
    init = [vp_init, eps_init, dlt_init, rho_init]
    out = dict(nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, wavelet=w, src=src, rec=rec,
               **{f"{n}_true": m for n, m in zip(names, true)}, **{f"{n}_init": m for n, m in zip(names, init)})
    for tag, order, kw in (("o4", 4, {}), ("o8", 8, {}), ("o4_rec", 4, dict(receiver_type=["vx", "vy", "sH"]))):
        solver = PropTorch(AcousticVTI1st3D(spatial_order=order, device="cpu"), shape=(nz, ny, nx), dh=dh, dt=dt,
                           abcn=abcn, impl="c", device="cpu", memory=BoundarySaving(), **kw)
        obs = _forward(solver, w, src, rec, true)
        r = _run(solver, w, src, rec, init, obs, False)
        out.update({f"obs_{tag}": obs, f"pred_{tag}": r["pred"]})
        out.update({f"grad_{n}_{tag}": r[f"grad{i}"] for i, n in enumerate(names)})
    np.savez_compressed(OUT / "vti3d.npz", **out)


def elastic3d_storage():
    """3-D elastic boundary saving with fp16 / bf16 / int8 strips (reference
    Elastic3D, BoundarySaving(storage_dtype=...): each of the nine fields
    quantised per face and shot on its own): 2 explosive shots on a
    20 x 18 x 22 layered model (CPML 6), vp/vs/rho gradients per format."""
    from sweep.equations import Elastic3D
    rng = np.random.default_rng(103)
    nz, ny, nx, nt, dt, dh, abcn = 20, 18, 22, 140, 0.0005, 5.0, 6
    base = _layered(nz, nx, rng, 1900.0, 3000.0, 3)
    vp_true = np.ascontiguousarray(np.repeat(base[:, None, :], ny, axis=1)
                                   * (1 + 0.02 * np.sin(np.arange(ny) / 2.5))[None, :, None]).astype(np.float32)
    vs_true = (vp_true / 1.73).astype(np.float32)
    rho_true = (310.0 * vp_true ** 0.25).astype(np.float32)
    vp_init = np.full((nz, ny, nx), 2300.0, np.float32)
    vs_init = (vp_init / 1.73).astype(np.float32)
    rho_init = (310.0 * vp_init ** 0.25).astype(np.float32)
    w = _wavelet(nt, dt, 30.0, 0.03)
    src = np.array([[7, 8, 5], [15, 10, 12]], np.int64)             # (x, y, z)
    rec = np.zeros((2, 10, 3), np.int64)
    for b in range(2):
        rec[b, :, 0] = np.linspace(1, nx - 2, 10).astype(np.int64)
        rec[b, :, 1] = np.linspace(2, ny - 3, 10).astype(np.int64)
        rec[b, :, 2] = 2 + 2 * b
    out = dict(nz=nz, ny=ny, nx=nx, nt=nt, dt=dt, dh=dh, abcn=abcn, order=8,
               vp_true=vp_true, vs_true=vs_true, rho_true=rho_true,
               vp_init=vp_init, vs_init=vs_init, rho_init=rho_init, wavelet=w, src=src, rec=rec)
    for sd in ("fp32", "fp16", "bf16", "int8"):
        eq = Elastic3D(spatial_order=8, device="cpu")
        solver = PropTorch(eq, shape=(nz, ny, nx), dh=dh, dt=dt, abcn=abcn, impl="c", device="cpu",
                           memory=BoundarySaving(storage_dtype=sd))
        if sd == "fp32":
            out["obs"] = _forward(solver, w, src, rec, [vp_true, vs_true, rho_true])
        r = _run(solver, w, src, rec, [vp_init, vs_init, rho_init], out["obs"], False)
        for i, name in enumerate(("vp", "vs", "rho")):
            out[f"grad_{name}_{sd}"] = r[f"grad{i}"]
        out[f"pred_{sd}"] = r["pred"]
    np.savez_compressed(OUT / "elastic3d_storage.npz", **out)


CASES = {
    "acoustic2d_c1": acoustic2d_c1,
    "acoustic2d_multi": acoustic2d_multi,
    "acoustic2d_pershot": acoustic2d_pershot,
    "acoustic2d_storage": acoustic2d_storage,
    "acoustic3d": acoustic3d,
    "acoustic2d_free_surface": acoustic2d_free_surface,
    "acoustic3d_free_surface": acoustic3d_free_surface,
    "acoustic2d_free_faces": acoustic2d_free_faces,
    "acoustic3d_storage": acoustic3d_storage,
    "elastic2d": elastic2d,
    "elastic2d_storage": elastic2d_storage,
    "elastic2d_vsrc": elastic2d_vsrc,
    "acoustic2d_illum": acoustic2d_illum,
    "acoustic3d_illum": acoustic3d_illum,
    "acoustic3d_clean": acoustic3d_clean,
    "acoustic2d_many": acoustic2d_many,
    "elastic2d_interior": elastic2d_interior,
    "elastic2d_free_surface": elastic2d_free_surface,
    "elastic2d_free_faces": elastic2d_free_faces,
    "elastic3d": elastic3d,
    "elastic3d_free_surface": elastic3d_free_surface,
    "elastic3d_storage": elastic3d_storage,
    "acoustic_orders": acoustic_orders,
    "elastic_orders": elastic_orders,
    "elastic3d_orders": elastic3d_orders,
    "vti2d": vti2d,
    "vti3d": vti3d,
}

if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for name in names:
        CASES[name]()
        print("wrote", name)
