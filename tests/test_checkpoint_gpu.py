"""Checkpoint memory mode (``Ckpt(chunks=k)``) on the GPU for every equation.

The forward is the same as with boundary saving, so the records agree bit for
bit; the backward replays each chunk from its checkpoint, so its gradient
differs from the boundary-saving one only by the rounding of the shorter
reconstructions.  Both are held to the bars against the reference's
impl='c' golden fixtures (records 1e-4, gradients 1e-3 relative L2).  Chunk
lengths are chosen not to divide nt."""
import numpy as np
import pytest
import torch

from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3


def _acoustic(d, memory, eq):
    from sweep_b200 import PropTorch
    s = PropTorch(eq(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                  dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, memory=memory)
    vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
    w = torch.tensor(d["wavelet"], device=DEV)
    pred = s(w, d["src"], d["rec"], models=[vp])
    loss = 0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return pred.detach().cpu().numpy(), vp.grad.cpu().numpy()


@pytest.mark.parametrize("case,chunks", [("acoustic2d_multi", 37), ("acoustic2d_c1", 100), ("acoustic2d_c1", 799)])
def test_acoustic2d_checkpoint(case, chunks):
    from sweep_b200 import Acoustic, BoundarySaving, Ckpt
    d = load(case)
    p_bs, g_bs = _acoustic(d, BoundarySaving(), Acoustic)
    p_ck, g_ck = _acoustic(d, Ckpt(chunks=chunks), Acoustic)
    print(f"{case} chunks={chunks}: ckpt vs boundary {rel(g_ck, g_bs):.2e}, vs reference {rel(g_ck, d['grad_vp']):.2e}")
    assert np.array_equal(p_ck, p_bs)
    assert rel(p_ck, d["pred"]) < REC_TOL
    assert rel(g_ck, d["grad_vp"]) < GRAD_TOL
    assert rel(g_ck, g_bs) < 1e-4


@pytest.mark.parametrize("chunks", [13, 1])
def test_acoustic3d_checkpoint(chunks):
    from sweep_b200 import Acoustic3D, BoundarySaving, Ckpt
    d = load("acoustic3d")
    p_bs, g_bs = _acoustic(d, BoundarySaving(), Acoustic3D)
    p_ck, g_ck = _acoustic(d, Ckpt(chunks=chunks), Acoustic3D)
    print(f"3-D chunks={chunks}: ckpt vs boundary {rel(g_ck, g_bs):.2e}, vs reference {rel(g_ck, d['grad_vp']):.2e}")
    assert np.array_equal(p_ck, p_bs)
    assert rel(g_ck, d["grad_vp"]) < GRAD_TOL
    assert rel(g_ck, g_bs) < 1e-4


@pytest.mark.parametrize("chunks", [41, 300])
def test_elastic_checkpoint(chunks):
    from sweep_b200 import BoundarySaving, Ckpt, Elastic, PropTorch
    d = load("elastic2d")

    def run(memory):
        s = PropTorch(Elastic(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                      dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, memory=memory)
        ms = [torch.tensor(d[k], device=DEV, requires_grad=True) for k in ("vp_init", "vs_init", "rho_init")]
        pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms)
        (0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()).backward()
        torch.cuda.synchronize()
        return pred.detach().cpu().numpy(), [m.grad.cpu().numpy() for m in ms]

    p_bs, g_bs = run(BoundarySaving())
    p_ck, g_ck = run(Ckpt(chunks=chunks))
    assert np.array_equal(p_ck, p_bs)
    for name, a, b, ref in zip(("vp", "vs", "rho"), g_ck, g_bs, ("grad_vp", "grad_vs", "grad_rho")):
        print(f"elastic chunks={chunks} {name}: ckpt vs boundary {rel(a, b):.2e}, vs reference {rel(a, d[ref]):.2e}")
        assert rel(a, d[ref]) < GRAD_TOL
        assert rel(a, b) < 1e-4


@pytest.mark.parametrize("case,eq_name", [("acoustic2d_multi", "Acoustic"), ("acoustic3d", "Acoustic3D")])
def test_tape_budget_switches_to_checkpoints(case, eq_name):
    """BoundarySaving(budget_gb=...): a call whose boundary-saving tape fits
    runs boundary saving, one whose tape does not checkpoints every
    ckpt_chunks steps -- the same results, bit for bit, as asking for that
    mode directly."""
    import sweep_b200
    from sweep_b200 import BoundarySaving, Ckpt
    eq = getattr(sweep_b200, eq_name)
    d = load(case)
    p_bs, g_bs = _acoustic(d, BoundarySaving(), eq)
    p_ck, g_ck = _acoustic(d, Ckpt(chunks=29), eq)
    p_big, g_big = _acoustic(d, BoundarySaving(budget_gb=100.0, ckpt_chunks=29), eq)
    p_small, g_small = _acoustic(d, BoundarySaving(budget_gb=1e-6, ckpt_chunks=29), eq)
    assert np.array_equal(p_big, p_bs) and np.array_equal(g_big, g_bs)
    assert np.array_equal(p_small, p_ck) and np.array_equal(g_small, g_ck)


@pytest.mark.parametrize("case,eq_name,count", [
    ("acoustic2d_multi", "Acoustic", 1), ("acoustic2d_multi", "Acoustic", 8),
    ("acoustic2d_c1", "Acoustic", 2), ("acoustic2d_c1", "Acoustic", 3),
    ("acoustic3d", "Acoustic3D", 1), ("acoustic3d", "Acoustic3D", 4),
])
def test_acoustic_recursive_checkpointing(case, eq_name, count):
    """Ckpt(mode='recursive', count=N): the backward bisects the time axis
    with at most N snapshots and reverses 64-step leaves, the chunks of
    Ckpt(chunks=64) -- records and gradients bit-identical to that mode (a
    budget too small for the bisection depth replays leaves from the nearest
    snapshot), and within the bars of the reference."""
    import sweep_b200
    from sweep_b200 import Ckpt
    eq = getattr(sweep_b200, eq_name)
    d = load(case)
    p_ck, g_ck = _acoustic(d, Ckpt(chunks=64), eq)
    p_rc, g_rc = _acoustic(d, Ckpt(mode="recursive", count=count), eq)
    assert np.array_equal(p_rc, p_ck)
    assert np.array_equal(g_rc, g_ck)
    assert rel(g_rc, d["grad_vp"]) < GRAD_TOL


@pytest.mark.parametrize("count", [1, 3])
def test_elastic_recursive_checkpointing(count):
    from sweep_b200 import Ckpt, Elastic, PropTorch
    d = load("elastic2d")

    def run(memory):
        s = PropTorch(Elastic(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                      dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, memory=memory)
        ms = [torch.tensor(d[k], device=DEV, requires_grad=True) for k in ("vp_init", "vs_init", "rho_init")]
        pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms)
        (0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()).backward()
        torch.cuda.synchronize()
        return pred.detach().cpu().numpy(), [m.grad.cpu().numpy() for m in ms]

    p_ck, g_ck = run(Ckpt(chunks=64))
    p_rc, g_rc = run(Ckpt(mode="recursive", count=count))
    assert np.array_equal(p_rc, p_ck)
    for a, b, ref in zip(g_rc, g_ck, ("grad_vp", "grad_vs", "grad_rho")):
        assert np.array_equal(a, b)
        assert rel(a, d[ref]) < GRAD_TOL


def _elastic3d(d, memory):
    from sweep_b200 import Elastic3D, PropTorch
    s = PropTorch(Elastic3D(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                  dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV, memory=memory)
    ms = [torch.tensor(d[k], device=DEV, requires_grad=True) for k in ("vp_init", "vs_init", "rho_init")]
    pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms)
    (0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()).backward()
    torch.cuda.synchronize()
    return pred.detach().cpu().numpy(), [m.grad.cpu().numpy() for m in ms]


@pytest.mark.parametrize("chunks", [37, 1, 200])
def test_elastic3d_checkpoint(chunks):
    """Elastic3D with Ckpt(chunks=k): nine fields and 18 CPML memories per
    checkpoint; records bit-identical to boundary saving, gradients within
    1e-4 of it and within the bars of the reference (nt 160)."""
    from sweep_b200 import BoundarySaving, Ckpt
    d = load("elastic3d")
    p_bs, g_bs = _elastic3d(d, BoundarySaving())
    p_ck, g_ck = _elastic3d(d, Ckpt(chunks=chunks))
    assert np.array_equal(p_ck, p_bs)
    for name, a, b in zip(("vp", "vs", "rho"), g_ck, g_bs):
        print(f"elastic3d chunks={chunks} {name}: ckpt vs boundary {rel(a, b):.2e}, "
              f"vs reference {rel(a, d['grad_' + name]):.2e}")
        assert rel(a, d["grad_" + name]) < GRAD_TOL
        assert rel(a, b) < 1e-4


@pytest.mark.parametrize("count", [1, 3])
def test_elastic3d_recursive_checkpointing(count):
    from sweep_b200 import Ckpt
    d = load("elastic3d")
    p_ck, g_ck = _elastic3d(d, Ckpt(chunks=64))
    p_rc, g_rc = _elastic3d(d, Ckpt(mode="recursive", count=count))
    assert np.array_equal(p_rc, p_ck)
    for name, a, b in zip(("vp", "vs", "rho"), g_rc, g_ck):
        assert np.array_equal(a, b)
        assert rel(a, d["grad_" + name]) < GRAD_TOL
