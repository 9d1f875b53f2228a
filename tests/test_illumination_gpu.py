"""Source / receiver illumination (``solver.compute_illumination = True``:
``sum_t u_tt^2`` and ``sum_t lambda^2`` on the physical box, summed over
shots) on the GPU.

* Parity with the reference's own run of the same case (boundary saving,
  golden fixtures made by the reference's impl='c'), bar 1e-3 relative L2 as
  for gradients, and with the float64 oracle (printed).
* The reference's three pins (its test/test_illumination_pin.py:66-160):
  turning illumination on moves neither the record nor the gradient by one
  bit; it is off by default and populated (model-shaped, finite, >= 0, not
  all zero) when asked for; and it does not depend on the memory mode."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
GRAD_TOL = 1e-3
CASES = ["acoustic2d_illum", "acoustic3d_illum"]


def _memories():
    from sweep_b200 import BoundarySaving, Ckpt, Full
    return {"boundary": BoundarySaving(), "full": Full(), "ckpt": Ckpt(chunks=40),
            "recursive": Ckpt(mode="recursive", count=2)}


def _run(case, memory=None, illum=True):
    from sweep_b200 import Acoustic, Acoustic3D, PropTorch
    d = load(case)
    eq = (Acoustic if d["vp_true"].ndim == 2 else Acoustic3D)(spatial_order=8, device=DEV)
    kw = {} if memory is None else {"memory": memory}
    s = PropTorch(eq, shape=tuple(d["vp_true"].shape), dh=float(d["dh"]), dt=float(d["dt"]),
                  abcn=int(d["abcn"]), device=DEV, **kw)
    if illum is not None:
        s.compute_illumination = illum
    vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
    pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=[vp])
    (0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()).backward()
    torch.cuda.synchronize()
    out = {"pred": pred.detach().cpu().numpy(), "grad": vp.grad.cpu().numpy(),
           "src": s.source_illumination, "rec": s.receiver_illumination}
    for k in ("src", "rec"):
        if out[k] is not None:
            out[k] = out[k].cpu().numpy()
    return out


@pytest.mark.parametrize("case", CASES)
def test_matches_reference_and_oracle(case):
    d = load(case)
    r = _run(case)
    _, _, _, _, i_s, i_r = O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"],
                                               float(d["dh"]), float(d["dt"]), int(d["abcn"]), prec="f64",
                                               illum=True)
    print(f"{case}: source illumination vs reference {rel(r['src'], d['src_illum_bs']):.2e}, vs f64 oracle "
          f"{rel(r['src'], i_s):.2e}; receiver {rel(r['rec'], d['rec_illum_bs']):.2e} / {rel(r['rec'], i_r):.2e}")
    assert r["src"].shape == d["vp_true"].shape
    assert rel(r["src"], d["src_illum_bs"]) < GRAD_TOL
    assert rel(r["rec"], d["rec_illum_bs"]) < GRAD_TOL
    assert rel(r["src"], i_s) < GRAD_TOL
    assert rel(r["rec"], i_r) < GRAD_TOL
    assert rel(r["grad"], d["grad_vp_bs"]) < GRAD_TOL


@pytest.mark.parametrize("mode", ["boundary", "full", "ckpt", "recursive"])
@pytest.mark.parametrize("case", CASES)
def test_illumination_does_not_move_the_gradient(case, mode):
    mem = _memories()
    off = _run(case, mem[mode], illum=False)
    on = _run(case, _memories()[mode], illum=True)
    assert np.array_equal(off["pred"], on["pred"])
    assert np.array_equal(off["grad"], on["grad"])


@pytest.mark.parametrize("mode", ["boundary", "full", "ckpt", "recursive"])
@pytest.mark.parametrize("case", CASES)
def test_off_by_default_and_populated_when_asked(case, mode):
    off = _run(case, _memories()[mode], illum=None)
    assert off["src"] is None and off["rec"] is None
    on = _run(case, _memories()[mode], illum=True)
    shape = load(case)["vp_true"].shape
    for k in ("src", "rec"):
        t = on[k]
        assert t.shape == shape
        assert np.all(np.isfinite(t))
        assert t.min() >= 0.0 and t.max() > 0.0


@pytest.mark.parametrize("case", CASES)
def test_does_not_depend_on_the_memory_mode(case):
    runs = {m: _run(case, mem) for m, mem in _memories().items()}
    base = runs["boundary"]
    for m, r in runs.items():
        grad_rel = rel(r["grad"], base["grad"])
        bar = max(20.0 * grad_rel, 1e-6)
        assert rel(r["src"], base["src"]) <= bar, m
        assert rel(r["rec"], base["rec"]) <= bar, m
