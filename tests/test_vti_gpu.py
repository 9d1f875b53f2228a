"""First-order acoustic VTI (reference sweep.equations.AcousticVTI1st and
AcousticVTI1st3D, Duveneck et al. 2008) on the GPU.

Bars: records within 1e-4 and vp / epsilon / delta / rho gradients within
1e-3 relative L2 of the reference's own runs (fixtures ``vti2d`` and
``vti3d``, made by the reference's impl='c') at two orders each and with
other receiver fields; per-shot models against the float32 oracle, the
float64 oracle printed beside."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3
NAMES = ("vp", "eps", "dlt", "rho")


def _solver(order, shape, dh, dt, abcn, **kw):
    from sweep_b200 import AcousticVTI1st, PropTorch
    return PropTorch(AcousticVTI1st(spatial_order=order, device=DEV), shape=shape, dh=dh, dt=dt, abcn=abcn,
                     device=DEV, **kw)


def _grad_run(s, w, src, rec, models, obs):
    ms = [torch.tensor(m, device=DEV, requires_grad=True) for m in models]
    pred = s(torch.tensor(w, device=DEV), src, rec, models=ms)
    (0.5 * ((pred - torch.tensor(obs, device=DEV)) ** 2).sum()).backward()
    torch.cuda.synchronize()
    return pred.detach().cpu().numpy(), [m.grad.cpu().numpy() for m in ms]


@pytest.mark.parametrize("tag,order,kw", [("o8", 8, {}), ("o4", 4, {}),
                                          ("o8_rec", 8, dict(receiver_type=["vx", "vz", "sH"]))])
def test_matches_reference_golden(tag, order, kw):
    d = load("vti2d")
    s = _solver(order, tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]), **kw)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d[f"{n}_true"], device=DEV) for n in NAMES]).cpu().numpy()
    assert obs.shape == d[f"obs_{tag}"].shape
    assert rel(obs, d[f"obs_{tag}"]) < REC_TOL
    pred, grads = _grad_run(s, d["wavelet"], d["src"], d["rec"], [d[f"{n}_init"] for n in NAMES], d[f"obs_{tag}"])
    errs = [rel(g, d[f"grad_{n}_{tag}"]) for g, n in zip(grads, NAMES)]
    print(f"vti {tag}: record {rel(pred, d[f'pred_{tag}']):.2e}, vp / eps / delta / rho "
          + " / ".join(f"{e:.2e}" for e in errs))
    assert rel(pred, d[f"pred_{tag}"]) < REC_TOL
    assert max(errs) < GRAD_TOL


def test_per_shot_models_match_oracle():
    """Two shots, each in its own model set, order 6, body sources on vx /
    vz recorded on (vz, sV), against the oracle (per-shot gradients)."""
    rng = np.random.default_rng(53)
    nz, nx, nt, dt, dh, abcn, B = 34, 46, 220, 0.0005, 5.0, 8, 2
    z = np.arange(nz)[:, None] + 0 * np.arange(nx)[None, :]
    vp = np.stack([(1900.0 + 700.0 * (z > nz // 2) + 20 * rng.standard_normal((nz, nx))) for _ in range(B)])
    vp = vp.astype(np.float32)
    eps = np.full_like(vp, 0.12) + (0.05 * (z > nz // 3)).astype(np.float32)
    dlt = (0.4 * eps).astype(np.float32)
    rho = (310.0 * vp ** 0.25).astype(np.float32)
    init = [np.full_like(vp, 2100.0), np.full_like(vp, 0.1), np.full_like(vp, 0.04), np.full_like(vp, 2100.0)]
    w = np.stack([np.sin(np.arange(nt) * dt * 2 * np.pi * f) * np.exp(-((np.arange(nt) * dt - 0.03) / 0.012) ** 2)
                  for f in (20.0, 26.0)]).astype(np.float32)
    src = np.array([[12, 8], [30, 14]], np.int64)
    rec = np.zeros((B, 6, 2), np.int64)
    for b in range(B):
        rec[b, :, 0] = np.linspace(2, nx - 3, 6).astype(np.int64)
        rec[b, :, 1] = 3 + 2 * b
    kw = dict(source_fields=("vx", "vz"), receiver_fields=("vz", "sV"))
    obs = O.vti2d_forward(vp, eps, dlt, rho, w, src, rec, dh, dt, abcn, order=6, **kw)
    s = _solver(6, (nz, nx), dh, dt, abcn, source_type=["vx", "vz"], receiver_type=["vz", "sV"])
    pred, grads = _grad_run(s, w, src, rec, init, obs)
    for prec in ("f32", "f64"):
        po, _, go = O.vti2d_gradient(*init, w, src, rec, obs, dh, dt, abcn, order=6, prec=prec, **kw)
        errs = [rel(a, b) for a, b in zip(grads, go)]
        print(f"vti per-shot vs {prec} oracle: record {rel(pred, po):.2e}, vp / eps / delta / rho "
              + " / ".join(f"{e:.2e}" for e in errs))
        if prec == "f32":
            assert rel(pred, po) < REC_TOL
            assert max(errs) < GRAD_TOL


def test_wavelet_gradient_and_other_memory_modes_are_refused():
    from sweep_b200 import Ckpt
    d = load("vti2d")
    s = _solver(8, tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    ms = [torch.tensor(d[f"{n}_init"], device=DEV) for n in NAMES]
    with pytest.raises(NotImplementedError, match="wavelet gradient"):
        s(torch.tensor(d["wavelet"], device=DEV, requires_grad=True), d["src"], d["rec"], models=ms)
    s = _solver(8, tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]), memory=Ckpt(chunks=50))
    ms = [torch.tensor(d[f"{n}_init"], device=DEV, requires_grad=True) for n in NAMES]
    with pytest.raises(RuntimeError, match="boundary saving with fp32 strips"):
        s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms).sum().backward()


def _solver3(order, shape, dh, dt, abcn, **kw):
    from sweep_b200 import AcousticVTI1st3D, PropTorch
    return PropTorch(AcousticVTI1st3D(spatial_order=order, device=DEV), shape=shape, dh=dh, dt=dt, abcn=abcn,
                     device=DEV, **kw)


@pytest.mark.parametrize("tag,order,kw", [("o4", 4, {}), ("o8", 8, {}),
                                          ("o4_rec", 4, dict(receiver_type=["vx", "vy", "sH"]))])
def test_3d_matches_reference_golden(tag, order, kw):
    """3-D (AcousticVTI1st3D), fixture ``vti3d`` made by the reference's
    impl='c': records within 1e-4 and the four gradients within 1e-3."""
    d = load("vti3d")
    s = _solver3(order, tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]), **kw)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d[f"{n}_true"], device=DEV) for n in NAMES]).cpu().numpy()
    assert obs.shape == d[f"obs_{tag}"].shape
    assert rel(obs, d[f"obs_{tag}"]) < REC_TOL
    pred, grads = _grad_run(s, d["wavelet"], d["src"], d["rec"], [d[f"{n}_init"] for n in NAMES], d[f"obs_{tag}"])
    errs = [rel(g, d[f"grad_{n}_{tag}"]) for g, n in zip(grads, NAMES)]
    print(f"vti3d {tag}: record {rel(pred, d[f'pred_{tag}']):.2e}, vp / eps / delta / rho "
          + " / ".join(f"{e:.2e}" for e in errs))
    assert rel(pred, d[f"pred_{tag}"]) < REC_TOL
    assert max(errs) < GRAD_TOL


def test_3d_per_shot_models_match_oracle():
    """3-D, two shots each in its own model set, order 6, sources on
    (vy, sV) recorded on (vx, vz, sH), against the oracle (per-shot
    gradients)."""
    rng = np.random.default_rng(59)
    nz, ny, nx, nt, dt, dh, abcn, B = 12, 14, 16, 120, 0.0005, 5.0, 4, 2
    z = (np.arange(nz)[:, None, None] + 0 * np.arange(ny)[None, :, None] + 0 * np.arange(nx)[None, None, :])
    vp = np.stack([(1900.0 + 600.0 * (z > nz // 2) + 20 * rng.standard_normal((nz, ny, nx))) for _ in range(B)])
    vp = vp.astype(np.float32)
    eps = (np.full_like(vp, 0.1) + 0.06 * (z > nz // 3)).astype(np.float32)
    dlt = (0.5 * eps).astype(np.float32)
    rho = (310.0 * vp ** 0.25).astype(np.float32)
    init = [np.full_like(vp, 2100.0), np.full_like(vp, 0.1), np.full_like(vp, 0.05), np.full_like(vp, 2100.0)]
    w = np.stack([np.sin(np.arange(nt) * dt * 2 * np.pi * f) * np.exp(-((np.arange(nt) * dt - 0.025) / 0.01) ** 2)
                  for f in (25.0, 32.0)]).astype(np.float32)
    src = np.array([[5, 6, 3], [10, 8, 5]], np.int64)
    rec = np.zeros((B, 5, 3), np.int64)
    for b in range(B):
        rec[b, :, 0] = np.linspace(1, nx - 2, 5).astype(np.int64)
        rec[b, :, 1] = np.linspace(2, ny - 3, 5).astype(np.int64)
        rec[b, :, 2] = 2 + b
    kw = dict(source_fields=("vy", "sV"), receiver_fields=("vx", "vz", "sH"))
    obs = O.vti3d_forward(vp, eps, dlt, rho, w, src, rec, dh, dt, abcn, order=6, **kw)
    s = _solver3(6, (nz, ny, nx), dh, dt, abcn, source_type=["vy", "sV"], receiver_type=["vx", "vz", "sH"])
    pred, grads = _grad_run(s, w, src, rec, init, obs)
    for prec in ("f32", "f64"):
        po, _, go = O.vti3d_gradient(*init, w, src, rec, obs, dh, dt, abcn, order=6, prec=prec, **kw)
        errs = [rel(a, b) for a, b in zip(grads, go)]
        print(f"vti3d per-shot vs {prec} oracle: record {rel(pred, po):.2e}, vp / eps / delta / rho "
              + " / ".join(f"{e:.2e}" for e in errs))
        if prec == "f32":
            assert rel(pred, po) < REC_TOL
            assert max(errs) < GRAD_TOL


def test_3d_wavelet_gradient_is_refused():
    d = load("vti3d")
    s = _solver3(4, tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    ms = [torch.tensor(d[f"{n}_init"], device=DEV) for n in NAMES]
    with pytest.raises(NotImplementedError, match="AcousticVTI1st3D does not return the wavelet gradient"):
        s(torch.tensor(d["wavelet"], device=DEV, requires_grad=True), d["src"], d["rec"], models=ms)
