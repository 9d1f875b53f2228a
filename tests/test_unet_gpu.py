"""The learned preconditioner on the GPU: the BF16 tensor-core convolutions
against float64 conv2d on the same (bf16-representable) inputs, the U-Net's
training, and a small FWI where the learned step is the first choice and the
plain illumination-preconditioned step the fallback."""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

from tests._util import rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _bf16(shape, gen, scale=1.0):
    return (torch.randn(shape, generator=gen) * scale).to(torch.bfloat16)


def _ref_conv(x_nhwc, w):                       # float64, NCHW conv2d
    x = x_nhwc.double().permute(0, 3, 1, 2)
    wt = w.double().permute(0, 3, 1, 2)         # (Co, 3, 3, C) -> (Co, C, 3, 3)
    return F.conv2d(x, wt, padding=1).permute(0, 2, 3, 1)


@pytest.mark.parametrize("n,h,w,c,co", [(2, 16, 24, 16, 24), (1, 9, 13, 8, 8), (3, 32, 40, 96, 64),
                                        (2, 16, 48, 256, 128)])
def test_conv_kernels_match_float64(n, h, w, c, co):
    from sweep_b200 import _lib
    gen = torch.Generator().manual_seed(n * 100 + c)
    x = _bf16((n, h, w, c), gen)
    wt = _bf16((co, 3, 3, c), gen, 0.1)
    dy = _bf16((n, h, w, co), gen)
    bias = torch.randn(co, generator=gen)
    xd, wd, dyd, bd = x.to(DEV), wt.to(DEV), dy.to(DEV), bias.to(DEV)
    st = torch.cuda.current_stream().cuda_stream
    # forward
    out = torch.empty((n, h, w, co), device=DEV)
    _lib.call("sweep_b200_conv3x3_gemm", xd.data_ptr(), wd.data_ptr(), bd.data_ptr(), out.data_ptr(),
              n, h, w, c, co, 1, st)
    _lib.call("sweep_b200_conv3x3_status", st)
    ref = _ref_conv(x, wt) + bias.double()
    assert rel(out.cpu(), ref) < 1e-5
    # data gradient: the adjoint of the forward
    wtt = wd.permute(3, 1, 2, 0).contiguous()
    gx = torch.empty((n, h, w, c), device=DEV)
    _lib.call("sweep_b200_conv3x3_gemm", dyd.data_ptr(), wtt.data_ptr(), None, gx.data_ptr(),
              n, h, w, co, c, -1, st)
    _lib.call("sweep_b200_conv3x3_status", st)
    xr = x.double().requires_grad_(True)
    yr = _ref_conv(xr, wt)
    yr.backward(dy.double())
    assert rel(gx.cpu(), xr.grad) < 1e-5
    # weight gradient
    gw = torch.empty((co, 3, 3, c), device=DEV)
    _lib.call("sweep_b200_conv3x3_wgrad", xd.data_ptr(), dyd.data_ptr(), gw.data_ptr(), n, h, w, c, co, st)
    _lib.call("sweep_b200_conv3x3_status", st)
    wr = wt.double().requires_grad_(True)
    _ref_conv(x, wr).backward(dy.double())
    torch.cuda.synchronize()
    assert rel(gw.cpu(), wr.grad) < 1e-5


def test_unet_trains():
    from sweep_b200.unet import UNet
    torch.manual_seed(0)
    net = UNet(base=16, levels=3).to(DEV)
    x = torch.randn(8, 3, 32, 48, device=DEV)
    y = torch.nn.functional.avg_pool2d(x[:, :1], 3, 1, 1)       # a learnable smooth map of the input
    opt = torch.optim.Adam(net.parameters(), lr=2e-3)
    losses = []
    for _ in range(150):
        loss = ((net(x) - y) ** 2).mean()
        opt.zero_grad()
        loss.backward()
        opt.step()
        losses.append(float(loss))
    print(f"U-Net training loss {losses[0]:.4f} -> {losses[-1]:.4f}")
    assert losses[-1] < 0.3 * losses[0]
    for p in net.parameters():
        assert p.grad is not None and torch.isfinite(p.grad).all()


def test_learned_fwi_small():
    """A small learned-preconditioned FWI: the network is trained on pairs the
    solver makes, then FWI runs with and without it from the same start on a
    held-out model.  Every step either kind takes lowers the data misfit (the
    learned step is kept only when it does), and the trained network gains:
    the learned run reaches the plain run's final misfit in fewer iterations.
    Model RMS errors are printed beside the misfits."""
    from sweep_b200.precondition import Survey, fwi, layered_model, make_pairs, smooth, train
    from sweep_b200.unet import UNet
    sv = Survey(nz=64, nx=128, nt=700, nshot=4, abcn=16, device="cuda:0")
    xs, ys = make_pairs(sv, 96, seed=1)
    net = UNet(base=16, levels=4, seed=0).to(DEV)
    hist = train(net, xs, ys, steps=800, batch=8, lr=1e-3)
    assert np.mean(hist[-20:]) < np.mean(hist[:20])
    rng = np.random.default_rng(12345)
    vt = torch.tensor(layered_model(sv.nz, sv.nx, rng), device=DEV)
    v0 = torch.tensor(smooth(vt.cpu().numpy()), device=DEV)
    with torch.no_grad():
        obs = sv.model(vt)
    iters = 8
    vp_p, hp, tp, _ = fwi(sv, v0, obs, iters)
    vp_l, hl, tl, nl = fwi(sv, v0, obs, iters, net=net)
    rms = lambda v: float(((v - vt) ** 2).mean().sqrt())
    reach = next((i for i, f in enumerate(hl) if f <= hp[-1]), None)
    print(f"plain: misfit {hp[0]:.4e} -> {hp[-1]:.4e} in {len(hp) - 1} iterations, {tp[-1]:.2f} s, model RMS "
          f"{rms(v0):.1f} -> {rms(vp_p):.1f} m/s; learned ({nl} learned steps): {hl[-1]:.4e}, model RMS "
          f"{rms(vp_l):.1f} m/s; reaches the plain final misfit after {reach} iterations")
    assert all(b < a for a, b in zip(hp, hp[1:]))
    assert all(b < a for a, b in zip(hl, hl[1:]))
    assert nl >= 1
    assert reach is not None and reach < len(hp) - 1
