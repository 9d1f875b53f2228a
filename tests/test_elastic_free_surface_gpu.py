"""Elastic traction-free faces on the GPU (reference PropTorch(Elastic,
free_surface=...)): the image method, the 2nd-order cells next to a surface,
the Robertsson corrections and the zeroed normal (and, on high-side faces,
shear) stresses on the surface rows and columns, and their exact transposes
in the adjoint.

Bars: records within 1e-4 and vp / vs / rho gradients within 1e-3 relative L2
of the reference's own run (golden fixture) and of the float32 CPU oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3


def _solver(shape, dh, dt, abcn, **kw):
    from sweep_b200 import Elastic, PropTorch
    return PropTorch(Elastic(spatial_order=8, device=DEV), shape=shape, dh=dh, dt=dt, abcn=abcn,
                     device=DEV, free_surface=True, **kw)


def _grad_run(s, w, src, rec, models, obs):
    ms = [torch.tensor(m, device=DEV, requires_grad=True) for m in models]
    pred = s(torch.tensor(w, device=DEV), src, rec, models=ms)
    loss = 0.5 * ((pred - torch.tensor(obs, device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return pred.detach().cpu().numpy(), [m.grad.cpu().numpy() for m in ms]


@pytest.mark.parametrize("memory", ["bs", "ckpt"])
def test_matches_reference_golden(memory):
    """A shot on the surface row recorded on it, a shot three rows below it."""
    from sweep_b200 import Ckpt
    d = load("elastic2d_free_surface")
    kw = {"memory": Ckpt(chunks=7)} if memory == "ckpt" else {}
    s = _solver(tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]), **kw)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d[k], device=DEV) for k in ("vp_true", "vs_true", "rho_true")])
    obs = obs.cpu().numpy()
    assert obs.shape == d["obs"].shape
    assert rel(obs, d["obs"]) < REC_TOL
    pred, (gvp, gvs, grho) = _grad_run(s, d["wavelet"], d["src"], d["rec"],
                                       [d["vp_init"], d["vs_init"], d["rho_init"]], d["obs"])
    sfx = "_ckpt" if memory == "ckpt" else ""
    print(f"elastic free surface ({memory}) vs reference: record {rel(pred, d['pred']):.2e} "
          f"vp {rel(gvp, d['grad_vp' + sfx]):.2e} vs {rel(gvs, d['grad_vs' + sfx]):.2e} "
          f"rho {rel(grho, d['grad_rho' + sfx]):.2e}")
    assert rel(pred, d["pred"]) < REC_TOL
    assert rel(gvp, d["grad_vp" + sfx]) < GRAD_TOL
    assert rel(gvs, d["grad_vs" + sfx]) < GRAD_TOL
    assert rel(grho, d["grad_rho" + sfx]) < GRAD_TOL


def _case(nz, nx, B, nt, seed=5):
    rng = np.random.default_rng(seed)
    z = np.arange(nz)[:, None] + 3.0 * np.sin(np.arange(nx)[None, :] / 11.0)
    vp = (1900.0 + 10.0 * z + 30 * rng.standard_normal((nz, nx))).astype(np.float32)
    vs = (vp / 1.75).astype(np.float32)
    rho = (310.0 * vp ** 0.25).astype(np.float32)
    t = np.arange(nt) * 0.0006
    a = (np.pi * 20 * (t - 0.05)) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    src = np.stack([np.linspace(12, nx - 13, B), np.arange(B) % 3], 1).astype(np.int64)
    rec = np.zeros((B, 24, 2), np.int64)
    for b in range(B):
        rec[b, :, 0] = np.linspace(1, nx - 2, 24).astype(np.int64)
        rec[b, :, 1] = (b % 2) * 2                 # on the surface row, or two rows below
    rec[0, -1] = (nx // 2, -2)                     # above the surface: off the grid, records zero
    obs = (0.3 * rng.standard_normal((B, nt, 24, 3)) * 1e-9).astype(np.float32)
    return dict(vp=vp, vs=vs, rho=rho, w=w, src=src, rec=rec, obs=obs, dh=5.0, dt=0.0006, abcn=12)


@pytest.mark.parametrize("shape,B", [((90, 140), 5), ((40, 300), 9)])
def test_matches_oracle_many_shots(shape, B):
    """Several shots per forward and reverse CTA, tiles clear of the CPML
    band under the surface, (vx, vz, szz) receivers (szz on the surface row
    is zero), against the float32 oracle."""
    c = _case(*shape, B, 360)
    kw = dict(receiver_type=["vx", "vz", "szz"])
    s = _solver(shape, c["dh"], c["dt"], c["abcn"], **kw)
    pred, (gvp, gvs, grho) = _grad_run(s, c["w"], c["src"], c["rec"], [c["vp"], c["vs"], c["rho"]], c["obs"])
    run = O.Elastic2D(c["vp"], c["vs"], c["rho"], c["w"], c["src"], c["rec"], c["dh"], c["dt"], c["abcn"],
                      receiver_fields=("vx", "vz", "szz"), free_surface=True)
    run.rec[0, -1] = -(1 << 20)                    # the oracle keeps air rows: skip that receiver there too
    p_o = run.forward(keep_tape=True)
    g_o = run.backward(p_o - c["obs"])
    assert np.all(pred[0, :, -1] == 0)
    for b in range(0, B, 2):                        # szz on the surface row, off the source cell
        off_src = [r for r in range(24) if tuple(c["rec"][b, r]) != tuple(c["src"][b])]
        assert np.all(pred[b, :, off_src, 2] == 0)
    assert rel(pred, p_o) < REC_TOL
    for g, go in zip((gvp, gvs, grho), g_o):
        assert rel(g, go) < GRAD_TOL


def test_velocity_sources_and_strip_formats():
    """Body-force sources on the surface row; fp32 strips against the oracle,
    bf16 strips against fp32 strips."""
    from sweep_b200 import BoundarySaving
    c = _case(60, 90, 3, 300, seed=9)
    c["obs"] = c["obs"][..., :2]
    kw = dict(source_type=["vx", "vz"])
    s = _solver((60, 90), c["dh"], c["dt"], c["abcn"], **kw)
    pred, grads = _grad_run(s, c["w"], c["src"], c["rec"], [c["vp"], c["vs"], c["rho"]], c["obs"])
    run = O.Elastic2D(c["vp"], c["vs"], c["rho"], c["w"], c["src"], c["rec"], c["dh"], c["dt"], c["abcn"],
                      source_fields=("vx", "vz"), free_surface=True)
    run.rec[0, -1] = -(1 << 20)
    p_o = run.forward(keep_tape=True)
    g_o = run.backward(p_o - c["obs"])
    assert rel(pred, p_o) < REC_TOL
    for g, go in zip(grads, g_o):
        assert rel(g, go) < GRAD_TOL
    s16 = _solver((60, 90), c["dh"], c["dt"], c["abcn"], memory=BoundarySaving(storage_dtype="bf16"), **kw)
    _, g16 = _grad_run(s16, c["w"], c["src"], c["rec"], [c["vp"], c["vs"], c["rho"]], c["obs"])
    for g, gb in zip(grads, g16):
        assert rel(gb, g) < 2e-2


@pytest.mark.parametrize("tag,faces", [("br", ["bottom", "right"]), ("tl", ["top", "left"]),
                                       ("all", ["top", "bottom", "left", "right"])])
def test_free_faces_match_reference_golden(tag, faces):
    """Traction-free faces per edge: high-side images with zeroed shear, the
    x-normal correction of szz, corners; (vx, vz, sxx) receivers on the
    surface rows and columns."""
    from sweep_b200 import Elastic, PropTorch
    d = load("elastic2d_free_faces")
    s = PropTorch(Elastic(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                  dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, free_surface=faces,
                  receiver_type=["vx", "vz", "sxx"])
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d[k], device=DEV) for k in ("vp_true", "vs_true", "rho_true")])
    assert rel(obs.cpu().numpy(), d[f"obs_{tag}"]) < REC_TOL
    pred, (gvp, gvs, grho) = _grad_run(s, d["wavelet"], d["src"], d["rec"],
                                       [d["vp_init"], d["vs_init"], d["rho_init"]], d[f"obs_{tag}"])
    print(f"elastic free faces {faces} vs reference: record {rel(pred, d[f'pred_{tag}']):.2e} "
          f"vp {rel(gvp, d[f'grad_vp_{tag}']):.2e} vs {rel(gvs, d[f'grad_vs_{tag}']):.2e} "
          f"rho {rel(grho, d[f'grad_rho_{tag}']):.2e}")
    assert rel(pred, d[f"pred_{tag}"]) < REC_TOL
    assert rel(gvp, d[f"grad_vp_{tag}"]) < GRAD_TOL
    assert rel(gvs, d[f"grad_vs_{tag}"]) < GRAD_TOL
    assert rel(grho, d[f"grad_rho_{tag}"]) < GRAD_TOL


@pytest.mark.parametrize("shape,faces,B", [((48, 48), ["bottom", "right"], 3),
                                           ((70, 100), ["top", "bottom", "left", "right"], 4)])
def test_free_faces_match_oracle(shape, faces, B):
    """Surface rows and columns on tile edges (48 x 48 with CPML 12 puts the
    bottom row and the right column on the last row / column of a tile),
    several shots per CTA, (vx, vz, szz, sxz) receivers on the surfaces,
    against the float32 oracle."""
    from sweep_b200 import Elastic, PropTorch
    nz, nx = shape
    rng = np.random.default_rng(17)
    vp = (2000.0 + 300.0 * rng.random(shape)).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    rho = (300.0 * vp ** 0.25).astype(np.float32)
    nt, dt, dh, abcn = 420, 0.0005, 5.0, 12
    t = np.arange(nt) * dt
    a = (np.pi * 30 * (t - 0.035)) ** 2
    w = ((1 - 2 * a) * np.exp(-a)).astype(np.float32)
    src = np.stack([np.linspace(3, nx - 4, B), np.linspace(nz - 3, 2, B)], 1).astype(np.int64)
    rec = np.zeros((B, 16, 2), np.int64)
    rec[:, :8, 0] = np.linspace(0, nx - 1, 8).astype(np.int64)
    rec[:, :8, 1] = nz - 1
    rec[:, 8:, 0] = nx - 1
    rec[:, 8:, 1] = np.linspace(0, nz - 1, 8).astype(np.int64)
    fields = ["vx", "vz", "szz", "sxz"]
    obs = (0.3 * rng.standard_normal((B, nt, 16, 4)) * 1e-9).astype(np.float32)
    s = PropTorch(Elastic(spatial_order=8, device=DEV), shape=shape, dh=dh, dt=dt, abcn=abcn, device=DEV,
                  free_surface=faces, receiver_type=fields)
    pred, grads = _grad_run(s, w, src, rec, [vp, vs, rho], obs)
    run = O.Elastic2D(vp, vs, rho, w, src, rec, dh, dt, abcn, receiver_fields=tuple(fields), free_surface=faces)
    p_o = run.forward(keep_tape=True)
    g_o = run.backward(p_o - obs)
    assert rel(pred, p_o) < REC_TOL
    for g, go in zip(grads, g_o):
        assert rel(g, go) < GRAD_TOL
