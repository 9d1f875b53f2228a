"""2-D acoustic parity on the GPU, through the public API and the C ABI.

Bars (written here, from the task's tolerance): records within 1e-4 and
gradients within 1e-3 relative L2 of the reference's impl='c' (golden
fixtures made by the reference itself) and of the float32 CPU oracle; the
error against the float64 oracle is asserted at the same bars."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3


def _solver(d, **kw):
    from sweep_b200 import Acoustic, PropTorch
    return PropTorch(Acoustic(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape[-2:]),
                     dh=float(d["dh"]), dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, **kw)


def _grad_run(solver, d, wavelet_grad=True):
    vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
    w = torch.tensor(d["wavelet"], device=DEV, requires_grad=wavelet_grad)
    pred = solver(w, d["src"], d["rec"], models=[vp])
    loss = 0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    gw = w.grad.cpu().numpy() if wavelet_grad else None
    return pred.detach().cpu().numpy(), float(loss), vp.grad.cpu().numpy(), gw


@pytest.mark.parametrize("case", ["acoustic2d_c1", "acoustic2d_multi", "acoustic2d_pershot"])
def test_matches_reference_golden(case):
    d = load(case)
    s = _solver(d)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d["vp_true"], device=DEV)]).cpu().numpy()
    assert obs.shape == d["obs"].shape
    assert rel(obs, d["obs"]) < REC_TOL
    wg = "grad_wavelet" in d
    pred, loss, g, gw = _grad_run(s, d, wavelet_grad=wg)
    assert rel(pred, d["pred"]) < REC_TOL
    assert rel(g, d["grad_vp"]) < GRAD_TOL
    if wg:
        assert rel(gw, d["grad_wavelet"]) < GRAD_TOL


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_matches_oracle(prec):
    d = load("acoustic2d_multi")
    pred_o, loss_o, g_o, gw_o = O.acoustic_gradient(
        d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"], float(d["dh"]), float(d["dt"]),
        int(d["abcn"]), prec=prec)
    pred, loss, g, gw = _grad_run(_solver(d), d)
    print(f"vs oracle {prec}: record {rel(pred, pred_o):.2e} grad {rel(g, g_o):.2e} wavelet {rel(gw, gw_o):.2e}")
    assert rel(pred, pred_o) < REC_TOL
    assert rel(g, g_o) < GRAD_TOL
    assert rel(gw, gw_o) < GRAD_TOL


def test_off_grid_receivers_record_zero():
    d = load("acoustic2d_multi")
    pred, *_ = _grad_run(_solver(d), d)
    assert np.all(pred[1, :, 7:, 0] == 0)


def test_run_to_run_bit_exact():
    d = load("acoustic2d_multi")
    a = _grad_run(_solver(d), d)
    b = _grad_run(_solver(d), d)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[2], b[2])
    assert np.array_equal(a[3], b[3])


def test_second_backward_is_refused():
    d = load("acoustic2d_pershot")
    s = _solver(d)
    vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
    pred = s(d["wavelet"], d["src"], d["rec"], models=[vp])
    loss = pred.square().sum()
    loss.backward(retain_graph=True)
    with pytest.raises(RuntimeError, match="second backward"):
        loss.backward()


def test_gradient_matches_central_differences():
    """<g, dm> against (L(m + e dm) - L(m - e dm)) / 2e, with the loss in float64.

    The perturbation spares the outermost ring of the physical model: those
    cells are replicated across the PML pad, and the reference's gradient --
    like this one -- is the crop of a runtime-grid gradient that is zero in the
    pad (reference utils/torch.py:20-41), so it leaves the pad's share out."""
    d = load("acoustic2d_multi")
    s = _solver(d)
    _, _, g, _ = _grad_run(s, d, wavelet_grad=False)
    rng = np.random.default_rng(0)
    dm = rng.standard_normal(g.shape).astype(np.float32)
    dm[:2], dm[-2:], dm[:, :2], dm[:, -2:] = 0, 0, 0, 0
    obs = torch.tensor(d["obs"], device=DEV, dtype=torch.float64)

    def loss(m):
        with torch.no_grad():
            p = s(d["wavelet"], d["src"], d["rec"], models=[torch.tensor(m, device=DEV)])
        return 0.5 * float(((p.double() - obs) ** 2).sum())

    eps = 2.0
    fd = (loss(d["vp_init"] + eps * dm) - loss(d["vp_init"] - eps * dm)) / (2 * eps)
    an = float(np.sum(g.astype(np.float64) * dm))
    assert abs(fd - an) <= 2e-3 * abs(an), (fd, an)


def test_c2_geometry_against_oracle():
    """The 256 x 768 geometry (CPML 40, dh 12.5, dt 1 ms), one shot, 400 steps:
    record and gradient against the float32 oracle."""
    from sweep_b200 import Acoustic, PropTorch, ricker
    rng = np.random.default_rng(1)
    nz, nx, nt, dt, dh, abcn = 256, 768, 400, 0.001, 12.5, 40
    vp_true = (1500 + 2000 * np.arange(nz)[:, None] / nz + np.zeros((1, nx))).astype(np.float32)
    vp0 = (vp_true + 50 * rng.standard_normal(vp_true.shape)).astype(np.float32)
    w = ricker(np.arange(nt) * dt - 0.1, 15.0).astype(np.float32)
    src = np.array([[300, 2]])
    rec = np.stack([np.arange(20, 740, 3), np.full(240, 2)], -1)[None]
    obs = O.acoustic_forward(vp_true, w, src, rec, dh, dt, abcn)
    pred_o, _, g_o, _ = O.acoustic_gradient(vp0, w, src, rec, obs, dh, dt, abcn)
    s = PropTorch(Acoustic(8, device=DEV), shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, device=DEV)
    vp = torch.tensor(vp0, device=DEV, requires_grad=True)
    pred = s(w, src, rec, models=[vp])
    (0.5 * ((pred - torch.tensor(obs, device=DEV)) ** 2).sum()).backward()
    assert rel(pred.detach().cpu().numpy(), pred_o) < REC_TOL
    assert rel(vp.grad.cpu().numpy(), g_o) < GRAD_TOL


def test_wavelet_linearity():
    """Scaling the wavelet by 2 scales the record by 2: every operation is
    linear in the field and a power-of-two scale commutes with rounding, except
    where values are subnormal (ahead of the wavefront), so the bar is 1e-6."""
    d = load("acoustic2d_multi")
    s = _solver(d)
    vp = torch.tensor(d["vp_true"], device=DEV)
    with torch.no_grad():
        a = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=[vp])
        b = s(2 * torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=[vp])
    assert rel((2 * a).cpu().numpy(), b.cpu().numpy()) < 1e-6
