"""Edge cases on the GPU, checked against the CPU oracle (itself pinned to
the reference's outputs): one- and two-step time axes, a shot whose
receivers all lie off the grid next to a shot with receivers, sources off the
grid, and physical boxes thinner than two boundary strips (the strip widths
shrink so that no cell is saved twice, as the reference's bs_strip_widths).
Bars: records 1e-4, gradients 1e-3 relative L2, as everywhere."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3


def _acoustic(shape, dh, dt, abcn):
    from sweep_b200 import Acoustic, Acoustic3D, PropTorch
    eq = (Acoustic if len(shape) == 2 else Acoustic3D)(spatial_order=8, device=DEV)
    return PropTorch(eq, shape=shape, dh=dh, dt=dt, abcn=abcn, device=DEV)


def _gpu_grad(s, vp0, w, src, rec, obs):
    vp = torch.tensor(vp0, device=DEV, requires_grad=True)
    pred = s(torch.tensor(w, device=DEV), src, rec, models=[vp])
    (0.5 * ((pred - torch.tensor(obs, device=DEV)) ** 2).sum()).backward()
    torch.cuda.synchronize()
    return pred.detach().cpu().numpy(), vp.grad.cpu().numpy()


def _wavelet(nt, dt, f=15.0, delay=0.0):
    t = np.arange(nt) * dt - delay
    a = (np.pi * f * t) ** 2
    return ((1 - 2 * a) * np.exp(-a)).astype(np.float32)


def _check(shape, src, rec, nt, dh=10.0, dt=0.001, abcn=6, seed=0):
    rng = np.random.default_rng(seed)
    vp_true = (2000.0 + 300.0 * rng.random(shape)).astype(np.float32)
    vp0 = np.full(shape, 2100.0, np.float32)
    w = _wavelet(nt, dt, delay=0.0 if nt < 20 else 0.03)
    obs = O.acoustic_forward(vp_true, w, src, rec, dh, dt, abcn)
    pred_o, _, g_o, _ = O.acoustic_gradient(vp0, w, src, rec, obs, dh, dt, abcn)
    pred, g = _gpu_grad(_acoustic(shape, dh, dt, abcn), vp0, w, src, rec, obs)
    assert np.all(np.isfinite(pred)) and np.all(np.isfinite(g))
    if np.linalg.norm(pred_o) > 0:
        assert rel(pred, pred_o) < REC_TOL
    else:
        assert np.all(pred == 0)
    if np.linalg.norm(g_o) > 0:
        assert rel(g, g_o) < GRAD_TOL
    else:
        assert np.all(g == 0)
    return pred, g


@pytest.mark.parametrize("nt", [1, 2, 3])
def test_acoustic2d_very_short_time_axes(nt):
    _check((24, 30), np.array([[12, 10]]), np.array([[[13, 10], [5, 3]]]), nt)


@pytest.mark.parametrize("nt", [1, 2])
def test_acoustic3d_very_short_time_axes(nt):
    _check((16, 14, 18), np.array([[8, 7, 6]]), np.array([[[9, 7, 6], [3, 4, 5]]]), nt)


def test_a_shot_with_every_receiver_off_the_grid():
    src = np.array([[10, 8], [20, 12]])
    rec = np.full((2, 5, 2), -1000, np.int64)
    rec[1] = [[3, 2], [8, 2], [15, 2], [22, 2], [28, 2]]
    pred, g = _check((32, 32), src, rec, 120)
    assert np.all(pred[0] == 0) and np.abs(pred[1]).max() > 0


def test_sources_off_the_grid_give_zero_records_and_gradient():
    src = np.array([[-500, 8], [10, 10 ** 6]])
    rec = np.array([[[3, 2], [8, 2]], [[15, 2], [22, 2]]])
    pred, g = _check((32, 32), src, rec, 80)
    assert np.all(pred == 0) and np.all(g == 0)


@pytest.mark.parametrize("shape", [(4, 40), (40, 3), (6, 7)])
def test_acoustic2d_boxes_thinner_than_two_strips(shape):
    _check(shape, np.array([[1, 1]]), np.array([[[0, 0], [shape[1] - 1, shape[0] - 1]]]), 90)


def test_acoustic3d_box_thinner_than_two_strips():
    _check((5, 12, 7), np.array([[3, 6, 2]]), np.array([[[1, 2, 1], [5, 9, 3]]]), 60)


def test_elastic2d_short_axis_and_thin_box():
    from sweep_b200 import Elastic, PropTorch
    for shape, nt in (((30, 36), 2), ((7, 40), 80)):
        rng = np.random.default_rng(4)
        vp_t = (2200.0 + 200.0 * rng.random(shape)).astype(np.float32)
        ms_t = [vp_t, (vp_t / 1.73).astype(np.float32), (310.0 * vp_t ** 0.25).astype(np.float32)]
        vp0 = np.full(shape, 2300.0, np.float32)
        ms0 = [vp0, (vp0 / 1.73).astype(np.float32), (310.0 * vp0 ** 0.25).astype(np.float32)]
        dh, dt, abcn = 5.0, 0.0005, 6
        w = _wavelet(nt, dt, f=30.0, delay=0.0 if nt < 20 else 0.02)
        src = np.array([[shape[1] // 2, shape[0] // 2]])
        rec = np.array([[[1, 1], [shape[1] - 2, shape[0] - 1]]])
        obs = O.elastic_forward(*ms_t, w, src, rec, dh, dt, abcn, 8)
        pred_o, _, g_o = O.elastic_gradient(*ms0, w, src, rec, obs, dh, dt, abcn, 8)
        s = PropTorch(Elastic(spatial_order=8, device=DEV), shape=shape, dh=dh, dt=dt, abcn=abcn, device=DEV)
        ms = [torch.tensor(m, device=DEV, requires_grad=True) for m in ms0]
        pred = s(torch.tensor(w, device=DEV), src, rec, models=ms)
        (0.5 * ((pred - torch.tensor(obs, device=DEV)) ** 2).sum()).backward()
        torch.cuda.synchronize()
        pred = pred.detach().cpu().numpy()
        if np.linalg.norm(pred_o) > 0:
            assert rel(pred, pred_o) < REC_TOL, (shape, nt)
        for m, go in zip(ms, g_o):
            gg = m.grad.cpu().numpy()
            assert np.all(np.isfinite(gg))
            if np.linalg.norm(go) > 0:
                assert rel(gg, go) < GRAD_TOL, (shape, nt)
