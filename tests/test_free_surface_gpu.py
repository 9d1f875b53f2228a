"""Free surface (``PropTorch(free_surface=True)``: the top face without PML
cells, the M halo rows above the surface at zero pressure) on the GPU against
the reference's own runs (golden fixtures ``acoustic2d_free_surface`` and
``acoustic3d_free_surface``, reference impl='c' with free_surface=True).

Bars as for the absorbing runs: records within 1e-4 and gradients (vp and the
wavelet) within 1e-3 relative L2."""
import numpy as np
import pytest
import torch

from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3


def _run(d, free_surface=True, **kw):
    from sweep_b200 import Acoustic, Acoustic3D, PropTorch
    eq = (Acoustic3D if d["vp_true"].ndim == 3 else Acoustic)(spatial_order=8, device=DEV)
    s = PropTorch(eq, shape=tuple(d["vp_true"].shape), dh=float(d["dh"]), dt=float(d["dt"]),
                  abcn=int(d["abcn"]), device=DEV, free_surface=free_surface, **kw)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d["vp_true"], device=DEV)]).cpu().numpy()
    vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
    w = torch.tensor(d["wavelet"], device=DEV)
    if w.dim() == 1:                    # one wavelet per shot, so each shot's gradient is its own
        w = w[None].expand(len(d["src"]), -1)
    w = w.clone().requires_grad_(True)
    pred = s(w, d["src"], d["rec"], models=[vp])
    loss = 0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return obs, pred.detach().cpu().numpy(), vp.grad.cpu().numpy(), w.grad.cpu().numpy()


@pytest.mark.parametrize("case", ["acoustic2d_free_surface", "acoustic3d_free_surface"])
def test_free_surface_matches_reference(case):
    d = load(case)
    obs, pred, g, gw = _run(d)
    print(f"{case}: records {rel(obs, d['obs']):.2e} pred {rel(pred, d['pred']):.2e} "
          f"grad {rel(g, d['grad_vp']):.2e}")
    assert rel(obs, d["obs"]) < REC_TOL
    assert rel(pred, d["pred"]) < REC_TOL
    assert rel(g, d["grad_vp"]) < GRAD_TOL
    # the reference's 3-D wavelet gradient holds shot 0 only (its kernel takes
    # the shot from the launch's y axis, acoustic3d/kernels.cu:256-257): its
    # shared-wavelet gradient is shot 0's, against our per-shot gradient 0
    if d["vp_true"].ndim == 3:
        assert rel(gw[0], d["grad_wavelet"]) < GRAD_TOL
    else:
        assert rel(gw, d["grad_wavelet"]) < GRAD_TOL


def test_free_surface_full_mode_and_storage_agree():
    """The reference's full mode gives the boundary-saving gradient; int8
    strips change it by about their quantisation: 1.1e-3 here, where the
    surface keeps the strips' amplitudes high (3e-4 without a surface)."""
    from sweep_b200 import BoundarySaving
    d = load("acoustic2d_free_surface")
    _, _, g_bs, _ = _run(d)
    assert rel(g_bs, d["grad_vp_full"]) < GRAD_TOL
    _, _, g_i8, _ = _run(d, memory=BoundarySaving(storage_dtype="int8"))
    assert rel(g_i8, g_bs) < 5e-3


def test_free_surface_changes_the_data():
    """Sanity: the surface reflects, so the records differ from the
    absorbing-top run by far more than the bars."""
    d = load("acoustic2d_free_surface")
    obs_abs, _, _, _ = _run(d, free_surface=False)
    assert rel(obs_abs, d["obs"]) > 0.1


@pytest.mark.parametrize("tag,faces", [("br", ["bottom", "right"]), ("tl", ["top", "left"])])
def test_per_face_free_surfaces_match_reference(tag, faces):
    """2-D free surfaces on any faces (reference free_surface=[...])."""
    from sweep_b200 import Acoustic, PropTorch
    d = load("acoustic2d_free_faces")
    s = PropTorch(Acoustic(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                  dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, free_surface=faces)
    src, rec = d[f"src_{tag}"], d[f"rec_{tag}"]
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), src, rec,
                models=[torch.tensor(d["vp_true"], device=DEV)]).cpu().numpy()
    vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
    w = torch.tensor(d["wavelet"], device=DEV, requires_grad=True)
    pred = s(w, src, rec, models=[vp])
    loss = 0.5 * ((pred - torch.tensor(d[f"obs_{tag}"], device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    print(f"{faces}: records {rel(obs, d[f'obs_{tag}']):.2e} grad {rel(vp.grad.cpu().numpy(), d[f'grad_vp_{tag}']):.2e}")
    assert rel(obs, d[f"obs_{tag}"]) < REC_TOL
    assert rel(pred.detach().cpu().numpy(), d[f"pred_{tag}"]) < REC_TOL
    assert rel(vp.grad.cpu().numpy(), d[f"grad_vp_{tag}"]) < GRAD_TOL
    assert rel(w.grad.cpu().numpy(), d[f"grad_wavelet_{tag}"]) < GRAD_TOL
