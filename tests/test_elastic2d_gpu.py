"""2-D isotropic elastic parity on the GPU, through the public API and the C ABI.

Bars: records within 1e-4 and vp / vs / rho gradients within 1e-3 relative L2
of the reference's impl='c' (golden fixture made by the reference itself) and
of the float32 and float64 CPU oracles.  Norms are taken in float64: the
elastic gradients are ~1e-19 in absolute value."""
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
                     device=DEV, **kw)


def _golden_solver(d):
    return _solver(tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]))


def _grad_run(s, w, src, rec, models, obs):
    ms = [torch.tensor(m, device=DEV, requires_grad=True) for m in models]
    pred = s(torch.tensor(w, device=DEV), src, rec, models=ms)
    loss = 0.5 * ((pred - torch.tensor(obs, device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return pred.detach().cpu().numpy(), [m.grad.cpu().numpy() for m in ms]


def test_matches_reference_golden():
    d = load("elastic2d")
    s = _golden_solver(d)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d[k], device=DEV) for k in ("vp_true", "vs_true", "rho_true")])
    obs = obs.cpu().numpy()
    assert obs.shape == d["obs"].shape
    assert rel(obs, d["obs"]) < REC_TOL
    pred, (gvp, gvs, grho) = _grad_run(s, d["wavelet"], d["src"], d["rec"],
                                       [d["vp_init"], d["vs_init"], d["rho_init"]], d["obs"])
    print(f"elastic vs reference: record {rel(pred, d['pred']):.2e} vp {rel(gvp, d['grad_vp']):.2e} "
          f"vs {rel(gvs, d['grad_vs']):.2e} rho {rel(grho, d['grad_rho']):.2e}")
    assert rel(pred, d["pred"]) < REC_TOL
    assert rel(gvp, d["grad_vp"]) < GRAD_TOL
    assert rel(gvs, d["grad_vs"]) < GRAD_TOL
    assert rel(grho, d["grad_rho"]) < GRAD_TOL
    # the reference's full-storage gradient differs from its boundary-saving one only by the it = 0 image
    assert rel(gvp, d["grad_vp_full"]) < GRAD_TOL


def _case(seed=3, nz=70, nx=96, B=3, nt=400, per_shot=False):
    rng = np.random.default_rng(seed)
    z = np.arange(nz)[:, None] + 3.0 * np.sin(np.arange(nx)[None, :] / 9.0)
    vp = (2000.0 + 12.0 * z + 40 * rng.standard_normal((nz, nx))).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    rho = (310.0 * vp ** 0.25).astype(np.float32)
    if per_shot:
        f = (1.0 + 0.02 * np.arange(B, dtype=np.float32))[:, None, None]
        vp, vs, rho = vp[None] * f, vs[None] * f, rho[None] * f
    t = np.arange(nt) * 0.0008
    w = ((1 - 2 * (np.pi * 18 * (t - 0.06)) ** 2) * np.exp(-(np.pi * 18 * (t - 0.06)) ** 2)).astype(np.float32)
    src = np.stack([np.linspace(10, nx - 11, B), np.full(B, 7)], 1).astype(np.int64)
    rec = np.zeros((B, 20, 2), np.int64)
    for b in range(B):
        rec[b, :, 0] = np.linspace(2, nx - 3, 20).astype(np.int64)
        rec[b, :, 1] = 4 + 2 * b
    rec[-1, -1] = (-500, 3)                         # padding receiver off the grid: records zero
    obs = (0.3 * rng.standard_normal((B, nt, 20, 2)) * 1e-9).astype(np.float32)
    return dict(vp=vp, vs=vs, rho=rho, w=w, src=src, rec=rec, obs=obs, dh=6.0, dt=0.0008, abcn=16)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("per_shot", [False, True])
def test_matches_oracle(prec, per_shot):
    c = _case(per_shot=per_shot)
    s = _solver(c["vp"].shape[-2:], c["dh"], c["dt"], c["abcn"])
    pred, g = _grad_run(s, c["w"], c["src"], c["rec"], [c["vp"], c["vs"], c["rho"]], c["obs"])
    run = O.Elastic2D(c["vp"], c["vs"], c["rho"], c["w"], c["src"], c["rec"], c["dh"], c["dt"],
                      c["abcn"], prec=prec)
    pred_o = run.forward()
    g_o = run.backward(pred_o - c["obs"])
    errs = [rel(a, b) for a, b in zip(g, g_o)]
    print(f"elastic vs oracle {prec} per_shot={per_shot}: record {rel(pred, pred_o):.2e} grads "
          + " ".join(f"{e:.2e}" for e in errs))
    assert np.all(pred[-1, :, -1] == 0)
    assert rel(pred, pred_o) < REC_TOL
    for e in errs:
        assert e < GRAD_TOL


def test_stress_receivers_and_shear_source_match_oracle():
    c = _case(seed=11, nz=60, nx=70, B=2, nt=300)
    rf = ("szz", "vx", "sxz", "sxx", "vz")
    s = _solver(c["vp"].shape, c["dh"], c["dt"], c["abcn"], source_type=["sxz"], receiver_type=list(rf))
    obs = np.zeros((2, 300, 20, len(rf)), np.float32)
    pred, g = _grad_run(s, c["w"], c["src"], c["rec"], [c["vp"], c["vs"], c["rho"]], obs)
    run = O.Elastic2D(c["vp"], c["vs"], c["rho"], c["w"], c["src"], c["rec"], c["dh"], c["dt"],
                      c["abcn"], source_fields=("sxz",), receiver_fields=rf)
    pred_o = run.forward()
    g_o = run.backward(pred_o - obs)
    assert pred.shape == (2, 300, 20, 5)
    assert rel(pred, pred_o) < REC_TOL
    for a, b in zip(g, g_o):
        assert rel(a, b) < GRAD_TOL


def test_wavelet_gradient_and_second_backward_are_refused():
    d = load("elastic2d")
    s = _golden_solver(d)
    ms = [torch.tensor(d[k], device=DEV, requires_grad=True) for k in ("vp_init", "vs_init", "rho_init")]
    w = torch.tensor(d["wavelet"], device=DEV, requires_grad=True)
    with pytest.raises(NotImplementedError, match="wavelet gradient"):
        s(w, d["src"], d["rec"], models=ms)
    pred = s(w.detach(), d["src"], d["rec"], models=ms)
    loss = (pred ** 2).sum()
    loss.backward(retain_graph=True)
    with pytest.raises(RuntimeError, match="second backward"):
        loss.backward()


@pytest.mark.parametrize("memory", ["boundary", "ckpt", "recursive"])
def test_velocity_sources_match_reference_golden(memory):
    """Body-force sources on vx and vz (shot 0's inside the boundary strips,
    with a receiver on its cell), (vx, vz, sxx) receivers: records within
    1e-4 and vp / vs / rho gradients within 1e-3 of the reference, in every
    memory mode, and against the float64 oracle."""
    from sweep_b200 import BoundarySaving, Ckpt
    d = load("elastic2d_vsrc")
    mem = {"boundary": BoundarySaving(), "ckpt": Ckpt(chunks=41),
           "recursive": Ckpt(mode="recursive", count=2)}[memory]
    s = _solver(tuple(d["vp_true"].shape), float(d["dh"]), float(d["dt"]), int(d["abcn"]),
                source_type=["vx", "vz"], receiver_type=["vx", "vz", "sxx"], memory=mem)
    with torch.no_grad():
        obs = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"],
                models=[torch.tensor(d[k], device=DEV) for k in ("vp_true", "vs_true", "rho_true")])
    assert rel(obs.cpu().numpy(), d["obs"]) < REC_TOL
    pred, grads = _grad_run(s, d["wavelet"], d["src"], d["rec"], [d["vp_init"], d["vs_init"], d["rho_init"]],
                            d["obs"])
    assert rel(pred, d["pred"]) < REC_TOL
    _, _, g64 = O.elastic_gradient(d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"], d["rec"],
                                   d["obs"], float(d["dh"]), float(d["dt"]), int(d["abcn"]), prec="f64",
                                   source_fields=("vx", "vz"), receiver_fields=("vx", "vz", "sxx"))
    for g, ref, o in zip(grads, ("grad_vp", "grad_vs", "grad_rho"), g64):
        print(f"velocity sources ({memory}) {ref}: vs reference {rel(g, d[ref]):.2e}, vs fp64 oracle {rel(g, o):.2e}")
        assert rel(g, d[ref]) < GRAD_TOL
        assert rel(g, o) < GRAD_TOL


def _fd_case():
    rng = np.random.default_rng(21)
    nz, nx, nt, dt, dh, abcn = 40, 48, 260, 0.0005, 5.0, 10
    z = np.arange(nz)[:, None] + np.zeros((1, nx))
    vp = (2000 + 20.0 * z + 30 * rng.standard_normal((nz, nx))).astype(np.float32)
    vs = (vp / 1.73).astype(np.float32)
    rho = (310 * vp ** 0.25).astype(np.float32)
    t = np.arange(nt) * dt
    w = ((1 - 2 * (np.pi * 25 * (t - 0.04)) ** 2) * np.exp(-(np.pi * 25 * (t - 0.04)) ** 2)).astype(np.float32)
    src = np.array([[24, 5]])
    rec = np.zeros((1, 12, 2), np.int64)
    rec[0, :, 0] = np.linspace(2, nx - 3, 12)
    rec[0, :, 1] = 3
    vt = vp.copy()
    vt[20:] *= 1.1
    obs = O.elastic_forward(vt, (vt / 1.73).astype(np.float32), (310 * vt ** 0.25).astype(np.float32),
                            w, src, rec, dh, dt, abcn, prec="f64").astype(np.float32)
    return dict(vp=vp, vs=vs, rho=rho, w=w, src=src, rec=rec, obs=obs, dh=dh, dt=dt, abcn=abcn, rng=rng)


def test_gradient_matches_central_differences_at_32_cells():
    """vp / vs / rho gradients at 32 random interior cells against central
    differences of the loss, taken with the float64 oracle forward (its own
    adjoint agrees with them to ~1e-6)."""
    c = _fd_case()
    s = _solver(c["vp"].shape, c["dh"], c["dt"], c["abcn"])
    _, g = _grad_run(s, c["w"], c["src"], c["rec"], [c["vp"], c["vs"], c["rho"]], c["obs"])
    nz, nx = c["vp"].shape
    cells = [(int(c["rng"].integers(2, nz - 2)), int(c["rng"].integers(2, nx - 2))) for _ in range(32)]
    base = [c[k].astype(np.float64) for k in ("vp", "vs", "rho")]

    def loss(k, iz, ix, h):
        ms = [m.copy() for m in base]
        ms[k][iz, ix] += h
        p = O.Elastic2D(*ms, c["w"], c["src"], c["rec"], c["dh"], c["dt"], c["abcn"], prec="f64").forward(False)
        return 0.5 * np.sum((p - c["obs"]) ** 2)

    for k, name in enumerate(("vp", "vs", "rho")):
        fd = np.array([(loss(k, iz, ix, 1.0) - loss(k, iz, ix, -1.0)) / 2.0 for iz, ix in cells])
        an = np.array([g[k][iz, ix] for iz, ix in cells], np.float64)
        print(f"{name}: 32-cell gradient vs central differences rel {rel(an, fd):.2e}")
        assert rel(an, fd) < 1e-3


def test_directional_derivative_through_own_forward():
    """<g, dm> against (L(m + e dm) - L(m - e dm)) / 2e with the float32 CUDA
    forward and a float64 loss, along dm = g / max|g| per model (outer 2-cell
    ring zeroed: those cells are replicated across the PML pad and the
    gradient is the crop of a runtime-grid gradient).  Along the gradient the
    first-order change has no cancellation, so it stands well above the float32
    rounding of the records."""
    c = _fd_case()
    s = _solver(c["vp"].shape, c["dh"], c["dt"], c["abcn"])
    ms0 = [c["vp"], c["vs"], c["rho"]]
    _, g = _grad_run(s, c["w"], c["src"], c["rec"], ms0, c["obs"])
    dms = []
    for gk in g:
        dm = (gk / np.abs(gk).max()).astype(np.float32)
        dm[:2], dm[-2:], dm[:, :2], dm[:, -2:] = 0, 0, 0, 0
        dms.append(dm)
    obs = torch.tensor(c["obs"], device=DEV, dtype=torch.float64)

    def loss(e):
        with torch.no_grad():
            p = s(torch.tensor(c["w"], device=DEV), c["src"], c["rec"],
                  models=[torch.tensor(m + e * dm, device=DEV) for m, dm in zip(ms0, dms)])
        return 0.5 * float(((p.double() - obs) ** 2).sum())

    eps = 0.5
    fd = (loss(eps) - loss(-eps)) / (2 * eps)
    an = float(sum(np.sum(gk.astype(np.float64) * dm) for gk, dm in zip(g, dms)))
    print(f"directional derivative: fd {fd:.6e} adjoint {an:.6e}")
    assert abs(fd - an) <= 2e-3 * abs(an), (fd, an)
