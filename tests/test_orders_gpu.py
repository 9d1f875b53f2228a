"""Acoustic propagation at spatial orders other than 8 on the GPU (the
reference's Acoustic / Acoustic3D default to order 4).

Bars: records within 1e-4 and vp / wavelet gradients within 1e-3 relative L2
of the reference's own runs (fixture ``acoustic_orders``, made by the
reference's impl='c'); per-shot models, illumination and every shot's 3-D
wavelet gradient against the float32 oracle, the float64 oracle printed
beside."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3


def _solver(order, shape, dh, dt, abcn, **kw):
    from sweep_b200 import Acoustic, Acoustic3D, PropTorch
    eq = (Acoustic if len(shape) == 2 else Acoustic3D)(spatial_order=order, device=DEV)
    return PropTorch(eq, shape=shape, dh=dh, dt=dt, abcn=abcn, device=DEV, **kw)


def _grad_run(s, w, src, rec, vp, obs, wavelet_grad=True, illum=False):
    vp = torch.tensor(vp, device=DEV, requires_grad=True)
    wt = torch.tensor(w, device=DEV, requires_grad=wavelet_grad)
    s.compute_illumination = illum
    pred = s(wt, src, rec, models=[vp])
    (0.5 * ((pred - torch.tensor(obs, device=DEV)) ** 2).sum()).backward()
    torch.cuda.synchronize()
    out = [pred.detach().cpu().numpy(), vp.grad.cpu().numpy(), wt.grad.cpu().numpy() if wavelet_grad else None]
    if illum:
        out += [s.source_illumination.cpu().numpy(), s.receiver_illumination.cpu().numpy()]
    return out


@pytest.mark.parametrize("order", [2, 4, 6, 12])
def test_acoustic2d_orders_match_reference(order):
    d = load("acoustic_orders")
    s = _solver(order, tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d["vp_true"], device=DEV)]).cpu().numpy()
    assert rel(obs, d[f"obs_o{order}"]) < REC_TOL
    pred, g, gw = _grad_run(s, d["wavelet"], d["src"], d["rec"], d["vp_init"], d[f"obs_o{order}"])
    print(f"order {order}: record {rel(pred, d[f'pred_o{order}']):.2e}, vp {rel(g, d[f'grad_vp_o{order}']):.2e}, "
          f"wavelet {rel(gw, d[f'grad_wavelet_o{order}']):.2e}")
    assert rel(pred, d[f"pred_o{order}"]) < REC_TOL
    assert rel(g, d[f"grad_vp_o{order}"]) < GRAD_TOL
    assert rel(gw, d[f"grad_wavelet_o{order}"]) < GRAD_TOL


@pytest.mark.parametrize("order", [4, 6])
def test_acoustic3d_orders_match_reference(order):
    d = load("acoustic_orders")
    a = (float(d["dh"]), float(d["dt3"]), int(d["abcn3"]))
    s = _solver(order, tuple(d["vp3_true"].shape), *a)
    pred, g, gw = _grad_run(s, d["wavelet3"], d["src3"], d["rec3"], d["vp3_init"], d[f"obs3_o{order}"])
    run = O.Acoustic3D(d["vp3_init"], d["wavelet3"], d["src3"], d["rec3"], *a, order=order)
    p_o = run.forward()
    _, gw_o = run.backward(p_o - d[f"obs3_o{order}"])
    print(f"3-D order {order}: record {rel(pred, d[f'pred3_o{order}']):.2e}, "
          f"vp {rel(g, d[f'grad3_vp_o{order}']):.2e}, wavelet (every shot) vs oracle {rel(gw, gw_o.sum(0)):.2e}")
    assert rel(pred, d[f"pred3_o{order}"]) < REC_TOL
    assert rel(g, d[f"grad3_vp_o{order}"]) < GRAD_TOL
    # every shot's wavelet gradient (the reference keeps shot 0 only in 3-D)
    assert rel(gw, gw_o.sum(0)) < GRAD_TOL


def _layered(nz, nx, rng):
    z = np.arange(nz)[:, None] + 0 * np.arange(nx)[None, :]
    return (1600.0 + 900.0 * (z > nz // 3) + 500.0 * (z > 2 * nz // 3)
            + 15.0 * rng.standard_normal((nz, nx))).astype(np.float32)


@pytest.mark.parametrize("order", [4, 6])
def test_per_shot_models_and_illumination_match_oracle(order):
    """Three shots, each in its own model, with illumination, against the
    oracle (per-shot gradients and illuminations)."""
    rng = np.random.default_rng(17 + order)
    nz, nx, nt, dt, dh, abcn = 36, 52, 240, 0.001, 10.0, 8
    vps = np.stack([_layered(nz, nx, rng) for _ in range(3)])
    v0 = np.full((3, nz, nx), 1900.0, np.float32)
    w = np.stack([np.sin(np.arange(nt) * dt * 2 * np.pi * f) * np.exp(-((np.arange(nt) * dt - 0.05) / 0.02) ** 2)
                  for f in (12.0, 15.0, 18.0)]).astype(np.float32)
    src = np.array([[10, 6], [26, 1], [40, 12]], np.int64)
    rec = np.zeros((3, 8, 2), np.int64)
    for b in range(3):
        rec[b, :, 0] = np.linspace(1, nx - 2, 8).astype(np.int64)
        rec[b, :, 1] = 2 + b
    obs = np.ascontiguousarray(O.acoustic_forward(vps, w, src, rec, dh, dt, abcn, order=order))
    s = _solver(order, (nz, nx), dh, dt, abcn)
    pred, g, gw, i_s, i_r = _grad_run(s, w, src, rec, v0, obs, illum=True)
    assert i_s.shape == v0.shape                # per-shot models give per-shot illuminations
    i_s, i_r = i_s.sum(0), i_r.sum(0)           # the oracle sums them over shots
    for prec in ("f32", "f64"):
        po, _, go, gwo, iso, iro = O.acoustic_gradient(v0, w, src, rec, obs, dh, dt, abcn, order=order, prec=prec,
                                                       illum=True)
        print(f"order {order} per-shot vs {prec} oracle: record {rel(pred, po):.2e} vp {rel(g, go):.2e} "
              f"wavelet {rel(gw, gwo):.2e} illum src {rel(i_s, iso):.2e} rec {rel(i_r, iro):.2e}")
        if prec == "f32":
            assert rel(pred, po) < REC_TOL
            for a, b in ((g, go), (gw, gwo), (i_s, iso), (i_r, iro)):
                assert rel(a, b) < GRAD_TOL


def test_other_memory_modes_are_refused_at_order_4():
    from sweep_b200 import BoundarySaving, Ckpt
    d = load("acoustic_orders")
    for memory in (Ckpt(chunks=50), BoundarySaving(storage_dtype="bf16"), BoundarySaving(storage="cpu")):
        s = _solver(4, tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]), memory=memory)
        vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
        with pytest.raises(RuntimeError, match="boundary saving with fp32 strips"):
            s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=[vp]).sum().backward()


# ------------------------------------------------------------------ elastic
@pytest.mark.parametrize("tag,order,kw", [("o2", 2, {}), ("o4", 4, {}), ("o6", 6, {}),
                                          ("o4_fs", 4, dict(free_surface=True, receiver_type=["vx", "vz", "sxx"]))])
def test_elastic_orders_match_reference(tag, order, kw):
    """2-D elastic at orders 2, 4, 6 and at order 4 with a traction-free top
    face (a shot and receivers on the surface row) against the reference."""
    from sweep_b200 import Elastic, PropTorch
    d = load("elastic_orders")
    s = PropTorch(Elastic(spatial_order=order, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                  dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, **kw)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d[f"{n}_true"], device=DEV) for n in ("vp", "vs", "rho")]).cpu().numpy()
    assert rel(obs, d[f"obs_{tag}"]) < REC_TOL
    ms = [torch.tensor(d[f"{n}_init"], device=DEV, requires_grad=True) for n in ("vp", "vs", "rho")]
    pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms)
    (0.5 * ((pred - torch.tensor(d[f"obs_{tag}"], device=DEV)) ** 2).sum()).backward()
    torch.cuda.synchronize()
    pred = pred.detach().cpu().numpy()
    errs = [rel(m.grad.cpu().numpy(), d[f"grad_{n}_{tag}"]) for m, n in zip(ms, ("vp", "vs", "rho"))]
    print(f"elastic {tag}: record {rel(pred, d[f'pred_{tag}']):.2e}, vp / vs / rho "
          + " / ".join(f"{e:.2e}" for e in errs))
    assert rel(pred, d[f"pred_{tag}"]) < REC_TOL
    assert max(errs) < GRAD_TOL


def test_elastic_order4_per_shot_body_force_matches_oracle():
    """Order 4, per-shot models, body-force sources on (vx, vz), (vx, vz,
    szz) receivers, against the float32 oracle (float64 printed)."""
    from sweep_b200 import Elastic, PropTorch
    rng = np.random.default_rng(41)
    nz, nx, nt, dt, dh, abcn, B = 34, 48, 220, 0.0005, 5.0, 8, 2
    vp = np.stack([_layered(nz, nx, rng) + 600.0 for _ in range(B)]).astype(np.float32)
    vs, rho = (vp / 1.8).astype(np.float32), (310.0 * vp ** 0.25).astype(np.float32)
    v0 = np.full_like(vp, 2300.0)
    v0s, r0 = (v0 / 1.8).astype(np.float32), (310.0 * v0 ** 0.25).astype(np.float32)
    w = np.stack([np.sin(np.arange(nt) * dt * 2 * np.pi * f) * np.exp(-((np.arange(nt) * dt - 0.03) / 0.012) ** 2)
                  for f in (20.0, 26.0)]).astype(np.float32)
    src = np.array([[12, 8], [30, 14]], np.int64)
    rec = np.zeros((B, 6, 2), np.int64)
    for b in range(B):
        rec[b, :, 0] = np.linspace(2, nx - 3, 6).astype(np.int64)
        rec[b, :, 1] = 3 + 2 * b
    kw = dict(source_fields=("vx", "vz"), receiver_fields=("vx", "vz", "szz"))
    obs = O.elastic_forward(vp, vs, rho, w, src, rec, dh, dt, abcn, order=4, **kw)
    s = PropTorch(Elastic(spatial_order=4, device=DEV), shape=(nz, nx), dh=dh, dt=dt, abcn=abcn, device=DEV,
                  source_type=["vx", "vz"], receiver_type=["vx", "vz", "szz"])
    ms = [torch.tensor(m, device=DEV, requires_grad=True) for m in (v0, v0s, r0)]
    pred = s(torch.tensor(w, device=DEV), src, rec, models=ms)
    (0.5 * ((pred - torch.tensor(obs, device=DEV)) ** 2).sum()).backward()
    torch.cuda.synchronize()
    pred = pred.detach().cpu().numpy()
    for prec in ("f32", "f64"):
        po, _, go = O.elastic_gradient(v0, v0s, r0, w, src, rec, obs, dh, dt, abcn, order=4, prec=prec, **kw)
        errs = [rel(m.grad.cpu().numpy(), g) for m, g in zip(ms, go)]
        print(f"elastic order 4 per-shot body force vs {prec} oracle: record {rel(pred, po):.2e}, vp / vs / rho "
              + " / ".join(f"{e:.2e}" for e in errs))
        if prec == "f32":
            assert rel(pred, po) < REC_TOL
            assert max(errs) < GRAD_TOL


def test_elastic_other_memory_modes_are_refused_at_order_4():
    from sweep_b200 import BoundarySaving, Ckpt, Elastic, PropTorch
    d = load("elastic_orders")
    for memory in (Ckpt(chunks=50), BoundarySaving(storage_dtype="int8")):
        s = PropTorch(Elastic(spatial_order=4, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                      dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, memory=memory)
        ms = [torch.tensor(d[f"{n}_init"], device=DEV, requires_grad=True) for n in ("vp", "vs", "rho")]
        with pytest.raises(RuntimeError, match="boundary saving with fp32 strips"):
            s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms).sum().backward()


@pytest.mark.parametrize("tag,order,kw", [("o2", 2, {}), ("o4", 4, {}), ("o6", 6, {}),
                                          ("o4_fs", 4, dict(free_surface=True))])
def test_elastic3d_orders_match_reference(tag, order, kw):
    """3-D elastic at orders 2, 4, 6 and at order 4 with a traction-free top
    face (a shot on the surface row) against the reference."""
    from sweep_b200 import Elastic3D, PropTorch
    d = load("elastic3d_orders")
    s = PropTorch(Elastic3D(spatial_order=order, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                  dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, **kw)
    ms = [torch.tensor(d[f"{n}_init"], device=DEV, requires_grad=True) for n in ("vp", "vs", "rho")]
    pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms)
    (0.5 * ((pred - torch.tensor(d[f"obs_{tag}"], device=DEV)) ** 2).sum()).backward()
    torch.cuda.synchronize()
    pred = pred.detach().cpu().numpy()
    errs = [rel(m.grad.cpu().numpy(), d[f"grad_{n}_{tag}"]) for m, n in zip(ms, ("vp", "vs", "rho"))]
    print(f"elastic3d {tag}: record {rel(pred, d[f'pred_{tag}']):.2e}, vp / vs / rho "
          + " / ".join(f"{e:.2e}" for e in errs))
    assert rel(pred, d[f"pred_{tag}"]) < REC_TOL
    assert max(errs) < GRAD_TOL
