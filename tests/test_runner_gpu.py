"""Stepped runners on the GPU: a forward advanced in uneven segments and its
reverse in uneven segments give exactly what one call and one backward give
(records, model gradients, wavelet gradient, illumination: bit for bit), for
2-D and 3-D acoustic and elastic, device and host tapes and a scaled strip
format; segments out of order, step_phase != 0 and checkpoint memories are
refused (reference runner contract, src/sweep/csrc/core/capi.h:236-243)."""
import numpy as np
import pytest
import torch

from tests._util import load

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _solver(d, memory=None):
    from sweep_b200 import Acoustic, Acoustic3D, Elastic, PropTorch
    if "vs_true" in d:
        eq = Elastic(spatial_order=8, device=DEV)
    else:
        eq = (Acoustic if d["vp_true"].ndim == 2 else Acoustic3D)(spatial_order=8, device=DEV)
    kw = {} if memory is None else {"memory": memory}
    return PropTorch(eq, shape=tuple(d["vp_true"].shape), dh=float(d["dh"]), dt=float(d["dt"]),
                     abcn=int(d["abcn"]), device=DEV, **kw)


def _models(d):
    keys = ("vp_init", "vs_init", "rho_init") if "vs_true" in d else ("vp_init",)
    return [torch.tensor(d[k], device=DEV) for k in keys]


def _one_call(d, memory, illum):
    s = _solver(d, memory)
    s.compute_illumination = illum
    ms = [m.clone().requires_grad_(True) for m in _models(d)]
    elastic = "vs_true" in d
    w = torch.tensor(d["wavelet"], device=DEV, requires_grad=not elastic)
    pred = s(w, d["src"], d["rec"], models=ms)
    res = pred - torch.tensor(d["obs"], device=DEV)
    (0.5 * (res ** 2).sum()).backward()
    torch.cuda.synchronize()
    out = {"pred": pred.detach(), "res": res.detach(), "grads": [m.grad for m in ms],
           "gw": None if elastic else w.grad, "illum": None}
    if illum:
        out["illum"] = (s.source_illumination, s.receiver_illumination)
    return out


def _segmented(d, memory, illum, fwd_cuts, bwd_cuts, res):
    s = _solver(d, memory)
    s.compute_illumination = illum
    r = s.forward_runner(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=_models(d))
    nt = r.nt
    cuts = [0] + list(fwd_cuts) + [nt]
    for a, b in zip(cuts[:-1], cuts[1:]):
        r.run(a, b)
    rec = r.record.clone()
    br = r.backward_runner(res)
    cuts = [nt] + list(bwd_cuts) + [0]
    for a, b in zip(cuts[:-1], cuts[1:]):
        br.run(a, b)
    torch.cuda.synchronize()
    return rec, br.gradients(), br.illumination(), r, br


CASES = [("acoustic2d_multi", None, True), ("acoustic3d", None, True), ("elastic2d", None, False),
         ("acoustic2d_storage", "host_int8", False), ("elastic2d", "host", False)]


def _memory(tag):
    from sweep_b200 import BoundarySaving
    if tag is None:
        return None
    if tag == "host":
        return BoundarySaving(storage="cpu")
    return BoundarySaving(storage="cpu", storage_dtype="int8")


@pytest.mark.parametrize("case,mem,illum", CASES, ids=[f"{c}-{m}" for c, m, _ in CASES])
def test_segments_equal_one_call(case, mem, illum):
    d = load(case)
    nt = d["wavelet"].shape[-1]
    ref = _one_call(d, _memory(mem), illum)
    rec, grads, il, r, br = _segmented(d, _memory(mem), illum, [37, 37, nt // 2, nt - 3], [nt - 1, nt // 3, 5],
                                       ref["res"])
    assert torch.equal(rec, ref["pred"])
    n_models = len(ref["grads"])
    for g, g0 in zip(grads[:n_models], ref["grads"]):
        assert torch.equal(g, g0)
    if ref["gw"] is not None:
        gw = grads[-1]
        g0 = ref["gw"]
        if g0.dim() == 1:        # a shared wavelet: autograd sums the per-shot gradients
            gw = gw.sum(dim=(0, 1))
            assert float((gw - g0).norm() / g0.norm()) < 1e-6
        else:
            assert torch.equal(gw[:, 0, :], g0)
    if illum:
        assert torch.equal(il[0], ref["illum"][0]) and torch.equal(il[1], ref["illum"][1])
    assert r.device_index() == 0
    r.close()
    br.close()


def test_partial_gradient_is_the_sum_so_far():
    """After reversing only the last steps, the gradient is that of those
    steps: running the rest adds the remaining contribution."""
    d = load("acoustic2d_multi")
    ref = _one_call(d, None, False)
    s = _solver(d)
    r = s.forward_runner(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=_models(d))
    r.run(0, r.nt)
    br = r.backward_runner(ref["res"])
    br.run(r.nt, r.nt // 2)
    g_half = br.gradients()[0].clone()
    br.run(r.nt // 2, 0)
    g_all = br.gradients()[0]
    assert torch.equal(g_all, ref["grads"][0])
    assert not torch.equal(g_half, g_all) and float(g_half.abs().max()) > 0


def test_refusals():
    from sweep_b200 import Ckpt
    d = load("acoustic2d_multi")
    s = _solver(d)
    r = s.forward_runner(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=_models(d))
    with pytest.raises(RuntimeError, match="in order"):
        r.run(5, 10)
    with pytest.raises(RuntimeError, match="step_phase"):
        r.run(0, 1, step_phase=1)
    with pytest.raises(RuntimeError, match="nt"):
        r.run(0, r.nt + 1)
    r.run(0, 10)
    with pytest.raises(RuntimeError, match="run it to the end"):
        r.backward_runner(torch.zeros_like(r.record))
    r.run(10, r.nt)
    br = r.backward_runner(torch.zeros_like(r.record))
    with pytest.raises(RuntimeError, match="in order"):
        br.run(r.nt - 5, 0)
    r.close()
    with pytest.raises(RuntimeError, match="closed"):
        r.run(r.nt, r.nt)
    with pytest.raises(ValueError, match="boundary saving"):
        _solver(d, Ckpt(chunks=20)).forward_runner(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                                                   models=_models(d))
