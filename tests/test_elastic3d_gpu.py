"""3-D isotropic elastic parity on the GPU (reference sweep.equations.Elastic3D,
order 8, boundary saving).

Bars: records within 1e-4 and vp / vs / rho gradients within 1e-3 relative L2
of the reference's own run (golden fixture, made by the reference) and of the
float32 CPU oracle; the float64 oracle's distance is printed beside."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3


def _solver(shape, dh, dt, abcn, **kw):
    from sweep_b200 import Elastic3D, PropTorch
    return PropTorch(Elastic3D(spatial_order=8, device=DEV), shape=shape, dh=dh, dt=dt, abcn=abcn,
                     device=DEV, **kw)


def _grad_run(s, w, src, rec, models, obs):
    ms = [torch.tensor(m, device=DEV, requires_grad=True) for m in models]
    pred = s(torch.tensor(w, device=DEV), src, rec, models=ms)
    loss = 0.5 * ((pred - torch.tensor(obs, device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return pred.detach().cpu().numpy(), [m.grad.cpu().numpy() for m in ms]


@pytest.mark.parametrize("tag,kw", [("", {}),
                                    ("_vsrc", dict(source_type=["vx", "vz"], receiver_type=["vx", "vz", "syy"]))])
def test_matches_reference_golden(tag, kw):
    """Explosive shots with (vx, vy, vz) receivers; body-force sources on
    (vx, vz) with (vx, vz, syy) receivers."""
    d = load("elastic3d")
    s = _solver(tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]), **kw)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d[k], device=DEV) for k in ("vp_true", "vs_true", "rho_true")])
    obs = obs.cpu().numpy()
    assert obs.shape == d[f"obs{tag}"].shape
    assert rel(obs, d[f"obs{tag}"]) < REC_TOL
    pred, (gvp, gvs, grho) = _grad_run(s, d["wavelet"], d["src"], d["rec"],
                                       [d["vp_init"], d["vs_init"], d["rho_init"]], d[f"obs{tag}"])
    print(f"elastic3d{tag} vs reference: record {rel(pred, d[f'pred{tag}']):.2e} "
          f"vp {rel(gvp, d[f'grad_vp{tag}']):.2e} vs {rel(gvs, d[f'grad_vs{tag}']):.2e} "
          f"rho {rel(grho, d[f'grad_rho{tag}']):.2e}")
    assert rel(pred, d[f"pred{tag}"]) < REC_TOL
    assert rel(gvp, d[f"grad_vp{tag}"]) < GRAD_TOL
    assert rel(gvs, d[f"grad_vs{tag}"]) < GRAD_TOL
    assert rel(grho, d[f"grad_rho{tag}"]) < GRAD_TOL


def _case(shape, B, nt, seed=3, per_shot=False):
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    z = np.arange(nz)[:, None, None] + 2.0 * np.sin(np.arange(nx)[None, None, :] / 7.0) + \
        1.5 * np.cos(np.arange(ny)[None, :, None] / 5.0)
    vp = (2000.0 + 14.0 * z + 30 * rng.standard_normal(shape)).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    rho = (310.0 * vp ** 0.25).astype(np.float32)
    if per_shot:
        f = (1.0 + 0.02 * np.arange(B, dtype=np.float32))[:, None, None, None]
        vp, vs, rho = vp[None] * f, vs[None] * f, rho[None] * f
    t = np.arange(nt) * 0.0006
    a = (np.pi * 22 * (t - 0.05)) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    src = np.stack([np.linspace(6, nx - 7, B), np.linspace(5, ny - 6, B), np.linspace(4, nz - 5, B)], 1)
    src = src.astype(np.int64)
    rec = np.zeros((B, 16, 3), np.int64)
    for b in range(B):
        rec[b, :, 0] = np.linspace(1, nx - 2, 16).astype(np.int64)
        rec[b, :, 1] = np.linspace(1, ny - 2, 16).astype(np.int64)[::-1]
        rec[b, :, 2] = 2 + b
    rec[-1, -1] = (-500, 3, 3)                      # padding receiver off the grid: records zero
    obs = (0.3 * rng.standard_normal((B, nt, 16, 3)) * 1e-9).astype(np.float32)
    return dict(vp=vp, vs=vs, rho=rho, w=w, src=src, rec=rec, obs=obs, dh=6.0, dt=0.0006, abcn=8)


@pytest.mark.parametrize("shape,B,per_shot", [((36, 40, 44), 3, False), ((30, 28, 34), 2, True)])
def test_matches_oracle(shape, B, per_shot):
    """Several shots, shared and per-shot models, against the float32
    oracle; the float64 oracle's distance printed beside."""
    c = _case(shape, B, 300, per_shot=per_shot)
    s = _solver(shape, c["dh"], c["dt"], c["abcn"])
    pred, grads = _grad_run(s, c["w"], c["src"], c["rec"], [c["vp"], c["vs"], c["rho"]], c["obs"])
    assert np.all(pred[-1, :, -1] == 0)
    for prec in ("f32", "f64"):
        run = O.Elastic3D(c["vp"], c["vs"], c["rho"], c["w"], c["src"], c["rec"], c["dh"], c["dt"], c["abcn"],
                          prec=prec)
        p_o = run.forward(keep_tape=True)
        g_o = run.backward(p_o - c["obs"])
        print(f"elastic3d {shape} per_shot={per_shot} vs {prec} oracle: record {rel(pred, p_o):.2e} "
              + " ".join(f"{n} {rel(g, go):.2e}" for n, g, go in zip(("vp", "vs", "rho"), grads, g_o)))
        if prec == "f32":
            assert rel(pred, p_o) < REC_TOL
            for g, go in zip(grads, g_o):
                assert rel(g, go) < GRAD_TOL


def test_free_surface_matches_reference_golden():
    """Traction-free top face: a shot on the surface row, (vx, vy, vz, sxx)
    receivers on it and two rows below."""
    d = load("elastic3d_free_surface")
    s = _solver(tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]), free_surface=True,
                receiver_type=["vx", "vy", "vz", "sxx"])
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d[k], device=DEV) for k in ("vp_true", "vs_true", "rho_true")])
    assert rel(obs.cpu().numpy(), d["obs"]) < REC_TOL
    pred, (gvp, gvs, grho) = _grad_run(s, d["wavelet"], d["src"], d["rec"],
                                       [d["vp_init"], d["vs_init"], d["rho_init"]], d["obs"])
    print(f"elastic3d free surface vs reference: record {rel(pred, d['pred']):.2e} "
          f"vp {rel(gvp, d['grad_vp']):.2e} vs {rel(gvs, d['grad_vs']):.2e} rho {rel(grho, d['grad_rho']):.2e}")
    assert rel(pred, d["pred"]) < REC_TOL
    assert rel(gvp, d["grad_vp"]) < GRAD_TOL
    assert rel(gvs, d["grad_vs"]) < GRAD_TOL
    assert rel(grho, d["grad_rho"]) < GRAD_TOL


def test_free_surface_matches_oracle():
    """A larger box with the free top face, several shots near it, szz
    receivers on the surface row (zero off the source cell), against the
    float32 oracle."""
    shape, B = (30, 36, 40), 3
    c = _case(shape, B, 300)
    c["src"][:, 2] = [0, 1, 3]
    c["rec"][:, :, 2] = 0
    c["rec"][-1, -1] = (shape[2] // 2, shape[1] // 2, -2)          # above the surface: off the grid
    fields = ["vx", "vy", "vz", "szz"]
    c["obs"] = np.concatenate([c["obs"], c["obs"][..., :1]], -1)
    s = _solver(shape, c["dh"], c["dt"], c["abcn"], free_surface=True, receiver_type=fields)
    pred, grads = _grad_run(s, c["w"], c["src"], c["rec"], [c["vp"], c["vs"], c["rho"]], c["obs"])
    run = O.Elastic3D(c["vp"], c["vs"], c["rho"], c["w"], c["src"], c["rec"], c["dh"], c["dt"], c["abcn"],
                      receiver_fields=tuple(fields), free_surface=True)
    run.rec[-1, -1] = -(1 << 20)
    p_o = run.forward(keep_tape=True)
    g_o = run.backward(p_o - c["obs"])
    assert np.all(pred[-1, :, -1] == 0)
    for b in range(B):
        off = [r for r in range(16) if tuple(c["rec"][b, r]) != tuple(c["src"][b])]
        assert np.all(pred[b][:, off, 3] == 0)
    print(f"elastic3d free surface vs f32 oracle: record {rel(pred, p_o):.2e} "
          + " ".join(f"{n} {rel(g, go):.2e}" for n, g, go in zip(("vp", "vs", "rho"), grads, g_o)))
    assert rel(pred, p_o) < REC_TOL
    for g, go in zip(grads, g_o):
        assert rel(g, go) < GRAD_TOL
