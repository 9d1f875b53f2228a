"""3-D acoustic parity on the GPU, through the public API and the C ABI.

Bars: records within 1e-4 and gradients within 1e-3 relative L2 of the
reference's impl='c' (golden fixtures made by the reference itself) and of the
float32 and float64 CPU oracles."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3


def _solver(d):
    from sweep_b200 import Acoustic3D, PropTorch
    return PropTorch(Acoustic3D(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape),
                     dh=float(d["dh"]), dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV)


def _grad_run(s, d, m_key="vp_init"):
    vp = torch.tensor(d[m_key], device=DEV, requires_grad=True)
    w = torch.tensor(d["wavelet"], device=DEV)
    w_b = w[None].expand(len(d["src"]), -1).clone().requires_grad_(True)      # per-shot wavelets
    pred = s(w_b, d["src"], d["rec"], models=[vp])
    loss = 0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return pred.detach().cpu().numpy(), vp.grad.cpu().numpy(), w_b.grad.cpu().numpy()


def test_matches_reference_golden():
    d = load("acoustic3d")
    s = _solver(d)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d["vp_true"], device=DEV)]).cpu().numpy()
    assert rel(obs, d["obs"]) < REC_TOL
    pred, g, gw = _grad_run(s, d)
    assert rel(pred, d["pred"]) < REC_TOL
    assert rel(g, d["grad_vp"]) < GRAD_TOL
    # the reference's 3-D wavelet gradient holds shot 0 only (see tests/test_oracle_golden.py)
    assert rel(gw[0], d["grad_wavelet"]) < GRAD_TOL


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_matches_oracle(prec):
    d = load("acoustic3d")
    run = O.Acoustic3D(d["vp_init"], d["wavelet"], d["src"], d["rec"], float(d["dh"]), float(d["dt"]),
                       int(d["abcn"]), prec=prec)
    pred_o = run.forward()
    g_o, gw_o = run.backward(pred_o - d["obs"])
    pred, g, gw = _grad_run(_solver(d), d)
    print(f"3-D vs oracle {prec}: record {rel(pred, pred_o):.2e} grad {rel(g, g_o):.2e} wavelet {rel(gw, gw_o):.2e}")
    assert rel(pred, pred_o) < REC_TOL
    assert rel(g, g_o) < GRAD_TOL
    assert rel(gw, gw_o) < GRAD_TOL


def test_run_to_run_bit_exact():
    d = load("acoustic3d")
    a = _grad_run(_solver(d), d)
    b = _grad_run(_solver(d), d)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_gradient_matches_central_differences():
    d = load("acoustic3d")
    s = _solver(d)
    _, g, _ = _grad_run(s, d)
    rng = np.random.default_rng(2)
    dm = rng.standard_normal(g.shape).astype(np.float32)
    dm[:2], dm[-2:], dm[:, :2], dm[:, -2:], dm[:, :, :2], dm[:, :, -2:] = 0, 0, 0, 0, 0, 0
    obs = torch.tensor(d["obs"], device=DEV, dtype=torch.float64)

    def loss(m):
        with torch.no_grad():
            p = s(d["wavelet"], d["src"], d["rec"], models=[torch.tensor(m, device=DEV)])
        return 0.5 * float(((p.double() - obs) ** 2).sum())

    eps = 2.0
    fd = (loss(d["vp_init"] + eps * dm) - loss(d["vp_init"] - eps * dm)) / (2 * eps)
    an = float(np.sum(g.astype(np.float64) * dm))
    assert abs(fd - an) <= 2e-3 * abs(an), (fd, an)


def test_illumination_covers_the_physical_box():
    d = load("acoustic3d")
    s = _solver(d)
    s.compute_illumination = True
    _grad_run(s, d)
    assert s.source_illumination.shape == d["vp_true"].shape
    assert float(s.source_illumination.min()) >= 0 and float(s.source_illumination.max()) > 0
    assert float(s.receiver_illumination.max()) > 0
