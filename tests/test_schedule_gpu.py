"""Launch schedules on the GPU: CUDA-graph step loops, shot grouping and the
autotuner change how the same kernels are launched, never what they compute.

* graph vs stream launches: the captured launches are the stream path's
  launches in the same order, so records and gradients are bit-identical (a
  graph length that does not divide nt exercises the partial last chunk);
* shots per CTA: each shot's forward is computed alone, so records are
  bit-identical; the image is summed over a CTA's shots before the Kahan
  accumulation, so gradients agree to rounding (bar 1e-5 relative L2);
* the autotuner records a schedule per shape, a later solver of that shape
  reuses it, and the tuned runs still meet the reference's golden vectors at
  the parity bars (records 1e-4, gradients 1e-3 relative L2)."""
import numpy as np
import pytest
import torch

from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL, GROUP_TOL = 1e-4, 1e-3, 1e-5


@pytest.fixture(autouse=True)
def _clean_schedules():
    from sweep_b200 import autotune
    autotune.clear_schedules()
    yield
    autotune.clear_schedules()


def _acoustic(d, nd=2, **kw):
    from sweep_b200 import Acoustic, Acoustic3D, PropTorch
    eq = (Acoustic if nd == 2 else Acoustic3D)(spatial_order=8, device=DEV)
    return PropTorch(eq, shape=tuple(d["vp_true"].shape), dh=float(d["dh"]), dt=float(d["dt"]),
                     abcn=int(d["abcn"]), device=DEV, **kw)


def _elastic(d, **kw):
    from sweep_b200 import Elastic, PropTorch
    return PropTorch(Elastic(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                     dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, **kw)


def _run(case, schedule=None, **kw):
    """(record, [model gradients], wavelet gradient or None) of one golden case."""
    d = load(case)
    if case.startswith("elastic"):
        s = _elastic(d, schedule=schedule, **kw)
        ms = [torch.tensor(d[k], device=DEV, requires_grad=True) for k in ("vp_init", "vs_init", "rho_init")]
        w = torch.tensor(d["wavelet"], device=DEV)
    else:
        s = _acoustic(d, nd=d["vp_true"].ndim, schedule=schedule, **kw)
        ms = [torch.tensor(d["vp_init"], device=DEV, requires_grad=True)]
        w = torch.tensor(d["wavelet"], device=DEV)
        if w.dim() == 1:
            w = w[None].expand(len(d["src"]), -1).clone()
        w.requires_grad_(True)
    pred = s(w, d["src"], d["rec"], models=ms)
    loss = 0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    gw = w.grad.cpu().numpy() if w.grad is not None else None
    return pred.detach().cpu().numpy(), [m.grad.cpu().numpy() for m in ms], gw, s


CASES = {
    "acoustic2d": ("acoustic2d_multi", {}),
    "acoustic2d_ckpt": ("acoustic2d_multi", {"ckpt": 40}),
    "acoustic3d": ("acoustic3d", {}),
    "elastic2d": ("elastic2d", {}),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_graph_and_stream_launches_agree(name):
    from sweep_b200 import Ckpt
    case, opt = CASES[name]
    kw = {"memory": Ckpt(chunks=opt["ckpt"])} if "ckpt" in opt else {}
    a = _run(case, {"graph_steps": 0}, **kw)
    b = _run(case, {"graph_steps": 7}, **kw)
    assert np.array_equal(a[0], b[0])
    for ga, gb in zip(a[1], b[1]):
        assert np.array_equal(ga, gb)
    if a[2] is not None:
        assert np.array_equal(a[2], b[2])
    d = load(case)
    assert rel(b[0], d["pred"]) < REC_TOL
    assert rel(b[1][0], d["grad_vp"]) < GRAD_TOL


@pytest.mark.parametrize("case,scheds", [
    ("acoustic2d_multi", [{"shots_fwd": 1, "shots_rev": 1}, {"shots_fwd": 3, "shots_rev": 2},
                          {"shots_fwd": 2, "shots_rev": 3}]),
    ("elastic2d", [{"shots_fwd": 1, "shots_rev": 1}, {"shots_fwd": 2, "shots_rev": 2}]),
])
def test_shot_grouping_changes_no_result(case, scheds):
    base = _run(case)
    for sc in scheds:
        r = _run(case, sc)
        got = r[3].launch_schedule(load(case)["wavelet"].shape[-1], load(case)["src"], load(case)["rec"],
                                   [torch.tensor(load(case)["vp_init"], device=DEV)] * len(r[1]))
        assert (got["shots_fwd"], got["shots_rev"]) == (sc["shots_fwd"], sc["shots_rev"])
        assert np.array_equal(r[0], base[0]), sc
        for g, g0 in zip(r[1], base[1]):
            assert rel(g, g0) < GROUP_TOL, sc
        if r[2] is not None:
            assert np.array_equal(r[2], base[2]), sc


@pytest.mark.parametrize("case", ["acoustic2d_multi", "acoustic3d", "elastic2d"])
def test_autotune_records_a_schedule_and_keeps_parity(case):
    from sweep_b200 import autotune
    pred, grads, gw, s = _run(case, autotune=True)
    rep = s.tune_report
    assert rep is not None and set(rep["trials"]) >= {"graph_steps"}
    assert rep["schedule"]["graph_steps"] in rep["trials"]["graph_steps"]
    for knob, res in rep["trials"].items():
        assert rep["schedule"][knob] == min(res, key=res.get), knob
    d = load(case)
    assert rel(pred, d["pred"]) < REC_TOL
    assert rel(grads[0], d["grad_vp"]) < GRAD_TOL
    # a second solver of the same shape runs the recorded schedule without tuning again
    _, _, _, s2 = _run(case, autotune=True)
    assert s2.tune_report is None
    n_models = len(grads)
    got = s2.launch_schedule(d["wavelet"].shape[-1], d["src"], d["rec"],
                             [torch.tensor(d["vp_init"], device=DEV)] * n_models)
    assert got == rep["schedule"]
    autotune.clear_schedules()
