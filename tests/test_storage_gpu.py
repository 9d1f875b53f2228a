"""Boundary saving with the strips held as fp16 / bf16 / int8, on the GPU,
against the reference's own runs of the same storage formats (golden fixtures
``acoustic2d_storage`` and ``acoustic3d_storage``: reference
BoundarySaving(storage_dtype=...)).

Two bars per format (written here):
  * the gradient within 1e-3 relative L2 of the reference's gradient for that
    format (the path's gradient bar);
  * the change the format makes to the gradient (format minus fp32) within
    ``PERT_TOL`` relative L2 of the reference's change.  A quantiser with other
    blocks, scales or rounding gives a change of the same size but a different
    pattern (relative error near 1), so this pins the codes themselves; the
    bound leaves room for the float32 noise between the two codes (about 7e-7
    of the gradient) against changes of 1.3e-5 (fp16) to 3.1e-4 (int8), and for
    bf16 / int8 roundings that tip the other way on values that differ in the
    last float32 bit (measured on a B200: 6.5e-2 fp16, 4.5e-2 bf16, 1.7e-2 int8)."""
import numpy as np
import pytest
import torch

from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
GRAD_TOL = 1e-3
PERT_TOL = {"fp16": 0.25, "bf16": 0.1, "int8": 0.05}


def _grad(d, storage_dtype):
    from sweep_b200 import Acoustic, Acoustic3D, BoundarySaving, PropTorch
    eq = (Acoustic3D if d["vp_true"].ndim == 3 else Acoustic)(spatial_order=8, device=DEV)
    s = PropTorch(eq, shape=tuple(d["vp_true"].shape),
                  dh=float(d["dh"]), dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV,
                  memory=BoundarySaving(storage_dtype=storage_dtype))
    vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
    pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=[vp])
    loss = 0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return vp.grad.double().cpu().numpy()


CASES = ["acoustic2d_storage", "acoustic3d_storage"]


@pytest.mark.parametrize("case", CASES)
def test_fp32_baseline_matches_reference(case):
    d = load(case)
    assert rel(_grad(d, "fp32"), d["grad_vp_fp32"]) < GRAD_TOL


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("sd", ["fp16", "bf16", "int8"])
def test_reduced_storage_matches_reference(case, sd):
    d = load(case)
    g32 = _grad(d, "fp32")
    g = _grad(d, sd)
    ref32, ref = d["grad_vp_fp32"].astype(np.float64), d[f"grad_vp_{sd}"].astype(np.float64)
    err = rel(g, ref)
    pert = rel(g - g32, ref - ref32)
    print(f"{case} {sd}: gradient vs reference {err:.2e}; change vs reference change {pert:.2e} "
          f"(change {rel(ref, ref32):.2e} of the gradient)")
    assert err < GRAD_TOL
    assert pert < PERT_TOL[sd]


def _egrads(d, storage_dtype, storage="gpu", with_pred=False):
    """vp / vs / rho gradients of the elastic case in ``d`` (2-D or 3-D by the
    model's rank) with the strips stored as ``storage_dtype``."""
    from sweep_b200 import BoundarySaving, Elastic, Elastic3D, PropTorch
    eq = (Elastic3D if d["vp_true"].ndim == 3 else Elastic)(spatial_order=8, device=DEV)
    s = PropTorch(eq, shape=tuple(d["vp_true"].shape),
                  dh=float(d["dh"]), dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV,
                  memory=BoundarySaving(storage=storage, storage_dtype=storage_dtype))
    ms = [torch.tensor(d[f"{n}_init"], device=DEV, requires_grad=True) for n in ("vp", "vs", "rho")]
    pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms)
    loss = 0.5 * ((pred.double() - torch.tensor(d["obs"], device=DEV).double()) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    grads = [m.grad.double().cpu().numpy() for m in ms]
    return (pred.detach().cpu().numpy(), grads) if with_pred else grads


# elastic changes are smaller (fp16 5e-6 .. 1.2e-5 of the gradients) against
# the same float32 noise, hence the wider bounds
E_PERT_TOL = {"fp16": 0.5, "bf16": 0.15, "int8": 0.1}


@pytest.mark.parametrize("sd", ["fp16", "bf16", "int8"])
def test_elastic_reduced_storage_matches_reference(sd):
    d = load("elastic2d_storage")
    g32 = _egrads(d, "fp32")
    g = _egrads(d, sd)
    for i, n in enumerate(("vp", "vs", "rho")):
        ref32, ref = d[f"grad_{n}_fp32"].astype(np.float64), d[f"grad_{n}_{sd}"].astype(np.float64)
        err = rel(g[i], ref)
        pert = rel(g[i] - g32[i], ref - ref32)
        print(f"elastic {sd} {n}: gradient vs reference {err:.2e}; change vs reference change {pert:.2e} "
              f"(change {rel(ref, ref32):.2e})")
        assert rel(g32[i], ref32) < GRAD_TOL
        assert err < GRAD_TOL
        assert pert < E_PERT_TOL[sd]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("sd", ["fp32", "int8"])
def test_host_tape_is_bit_identical(case, sd):
    """BoundarySaving(storage='cpu'): the same tape bytes go through pinned host
    memory, so the gradient is bit-identical to the device tape's."""
    from sweep_b200 import Acoustic, Acoustic3D, BoundarySaving, PropTorch
    d = load(case)
    grads = []
    for storage in ("gpu", "cpu"):
        eq = (Acoustic3D if d["vp_true"].ndim == 3 else Acoustic)(spatial_order=8, device=DEV)
        s = PropTorch(eq, shape=tuple(d["vp_true"].shape), dh=float(d["dh"]), dt=float(d["dt"]),
                      abcn=int(d["abcn"]), device=DEV, memory=BoundarySaving(storage=storage, storage_dtype=sd))
        vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
        pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=[vp])
        loss = 0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()
        loss.backward()
        torch.cuda.synchronize()
        grads.append(vp.grad.cpu().numpy())
    assert np.array_equal(grads[0], grads[1])


def test_elastic_host_tape_is_bit_identical():
    from sweep_b200 import BoundarySaving, Elastic, PropTorch
    d = load("elastic2d_storage")
    out = []
    for storage in ("gpu", "cpu"):
        s = PropTorch(Elastic(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                      dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV,
                      memory=BoundarySaving(storage=storage, storage_dtype="bf16"))
        ms = [torch.tensor(d[f"{n}_init"], device=DEV, requires_grad=True) for n in ("vp", "vs", "rho")]
        pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms)
        (0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()).backward()
        torch.cuda.synchronize()
        out.append([m.grad.cpu().numpy() for m in ms])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


# 3-D elastic (fixture ``elastic3d_storage``: the reference's Elastic3D run per
# format, each of the nine fields quantised per face and shot).  The format
# changes the gradients by 1.6e-6 (fp16, vp) to 2.1e-4 (int8, rho); the
# change's pattern measured on a B200 against the reference's: fp16 0.26 (vp,
# whose change is near the float32 noise) / 0.10 (vs, rho), bf16 0.024, int8
# 0.018; a quantiser with other faces or blocks gives about 1.
E3_PERT_TOL = {"fp16": 0.5, "bf16": 0.1, "int8": 0.05}


@pytest.mark.parametrize("sd", ["fp16", "bf16", "int8"])
def test_elastic3d_reduced_storage_matches_reference(sd):
    d = load("elastic3d_storage")
    p32, g32 = _egrads(d, "fp32", with_pred=True)
    p, g = _egrads(d, sd, with_pred=True)
    assert np.array_equal(p, p32)                   # the strip format leaves the forward alone
    assert rel(p32, d["pred_fp32"]) < 1e-4
    for i, n in enumerate(("vp", "vs", "rho")):
        ref32, ref = d[f"grad_{n}_fp32"].astype(np.float64), d[f"grad_{n}_{sd}"].astype(np.float64)
        err = rel(g[i], ref)
        pert = rel(g[i] - g32[i], ref - ref32)
        print(f"elastic3d {sd} {n}: gradient vs reference {err:.2e}; change vs reference change {pert:.2e} "
              f"(change {rel(ref, ref32):.2e})")
        assert rel(g32[i], ref32) < GRAD_TOL
        assert err < GRAD_TOL
        assert pert < E3_PERT_TOL[sd]


@pytest.mark.parametrize("sd", ["fp32", "int8"])
def test_elastic3d_host_tape_is_bit_identical(sd):
    d = load("elastic3d_storage")
    a = _egrads(d, sd, storage="gpu")
    b = _egrads(d, sd, storage="cpu")
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
