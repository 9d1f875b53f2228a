"""Parity on the code paths the benchmark workloads run, which the small
fixtures do not reach.

* 3-D, a grid whose clear box spans several 32 x 8 column blocks
  (`acoustic3d_clean`, 64 x 72 x 96, CPML 8): split into z chunks, the
  adjoint and reconstruction kernels' CTAs that lie wholly inside the clear
  box take their clean path (gw formed once per staged plane).  Every run is
  checked against the reference's own output and the float64 oracle, at
  1, 3 and 5 z chunks and at the built-in schedule.
* 2-D, 20 shots of uneven geometry (`acoustic2d_many`) at 2 / 8 shots per
  forward / reverse CTA (the survey's schedule), 4 / 16 and 1 / 1.
* Elastic, a grid with 32 x 32 tiles clear of the CPML band
  (`elastic2d_interior`), at 1 and 2 shots per CTA.

Bars: records within 1e-4 and gradients within 1e-3 relative L2 of the
reference's impl='c'; the error against the float64 oracle is printed."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL, GRAD_TOL = 1e-4, 1e-3


@pytest.fixture(autouse=True)
def _clean_schedules():
    from sweep_b200 import autotune
    autotune.clear_schedules()
    yield
    autotune.clear_schedules()


def _acoustic(d, **kw):
    from sweep_b200 import Acoustic, Acoustic3D, PropTorch
    eq = (Acoustic if d["vp_true"].ndim == 2 else Acoustic3D)(spatial_order=8, device=DEV)
    return PropTorch(eq, shape=tuple(d["vp_true"].shape), dh=float(d["dh"]), dt=float(d["dt"]),
                     abcn=int(d["abcn"]), device=DEV, **kw)


def _acoustic_grad(s, d):
    vp = torch.tensor(d["vp_init"], device=DEV, requires_grad=True)
    w = torch.tensor(d["wavelet"], device=DEV, requires_grad=True)
    pred = s(w, d["src"], d["rec"], models=[vp])
    loss = 0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return pred.detach().cpu().numpy(), vp.grad.cpu().numpy(), w.grad.cpu().numpy()


def _clean_ctas(d, nzc):
    """How many (x, y, z-chunk) column blocks of the 3-D stencil grid lie
    wholly inside the clear box (the host's chunking: zc = ceil(nz / nzc))."""
    M, pad = 4, int(d["abcn"])
    nz, ny, nx = (n + 2 * pad + 2 * M for n in d["vp_true"].shape)
    q0 = pad + 2 * M + 1
    qz1, qy1, qx1 = nz - q0, ny - q0, nx - q0
    zc = -(-nz // nzc)
    xs = sum(1 for c in range(0, nx, 32) if c >= q0 and c + 32 <= qx1)
    ys = sum(1 for c in range(0, ny, 8) if c >= q0 and c + 8 <= qy1)
    zs = sum(1 for k in range(-(-nz // zc)) if max(M, k * zc) >= q0 and min(nz - M, (k + 1) * zc) <= qz1)
    return xs * ys * zs


@pytest.fixture(scope="module")
def clean_oracle():
    d = load("acoustic3d_clean")
    return O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"], float(d["dh"]),
                               float(d["dt"]), int(d["abcn"]), prec="f64")


@pytest.mark.parametrize("z_chunks", [1, 3, 5, None])
def test_acoustic3d_clean_ctas_match_reference(z_chunks, clean_oracle):
    d = load("acoustic3d_clean")
    sched = None if z_chunks is None else {"z_chunks": z_chunks}
    s = _acoustic(d, schedule=sched)
    pred, g, gw = _acoustic_grad(s, d)
    got = s.launch_schedule(d["wavelet"].shape[-1], d["src"], d["rec"], [torch.tensor(d["vp_init"], device=DEV)])
    if z_chunks is not None:
        assert got["z_chunks"] == z_chunks
    if z_chunks != 1:
        assert _clean_ctas(d, got["z_chunks"]) > 0          # the clean path runs
    p64, _, g64, gw64 = clean_oracle
    print(f"3-D clean, {got['z_chunks']} z chunks ({_clean_ctas(d, got['z_chunks'])} clean blocks per shot): "
          f"vs reference record {rel(pred, d['pred']):.2e} grad {rel(g, d['grad_vp']):.2e}; vs f64 oracle "
          f"record {rel(pred, p64):.2e} grad {rel(g, g64):.2e} wavelet {rel(gw, gw64):.2e}")
    assert rel(pred, d["pred"]) < REC_TOL
    assert rel(g, d["grad_vp"]) < GRAD_TOL
    # the reference's 3-D wavelet gradient holds shot 0 only (a reference defect)
    assert rel(gw[0], d["grad_wavelet"][0]) < GRAD_TOL
    assert rel(pred, p64) < REC_TOL
    assert rel(g, g64) < GRAD_TOL
    assert rel(gw, gw64) < GRAD_TOL


@pytest.mark.parametrize("z_chunks", [1, 3])
def test_acoustic3d_tile_height_changes_nothing(z_chunks):
    """16-row column blocks (512-thread CTAs) compute every cell with the same
    taps in the same order as 8-row ones: records and gradients bit-identical,
    and within the bars of the reference."""
    d = load("acoustic3d_clean")
    runs = {}
    for ty in (8, 16):
        s = _acoustic(d, schedule={"z_chunks": z_chunks, "tile_y": ty})
        runs[ty] = _acoustic_grad(s, d)
        got = s.launch_schedule(d["wavelet"].shape[-1], d["src"], d["rec"],
                                [torch.tensor(d["vp_init"], device=DEV)])
        assert got["tile_y"] == ty
    for a, b in zip(runs[8], runs[16]):
        assert np.array_equal(a, b)
    assert rel(runs[16][0], d["pred"]) < REC_TOL
    assert rel(runs[16][1], d["grad_vp"]) < GRAD_TOL


def test_acoustic3d_z_chunking_changes_nothing_but_rounding():
    d = load("acoustic3d_clean")
    runs = [_acoustic_grad(_acoustic(d, schedule={"z_chunks": k}), d) for k in (1, 5)]
    assert np.array_equal(runs[0][0], runs[1][0])           # records: same arithmetic per cell
    assert rel(runs[1][1], runs[0][1]) < 1e-5


@pytest.fixture(scope="module")
def many_oracle():
    d = load("acoustic2d_many")
    return O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"], float(d["dh"]),
                               float(d["dt"]), int(d["abcn"]), prec="f64")


@pytest.mark.parametrize("fwd,rev", [(2, 8), (4, 16), (1, 1)])
def test_acoustic2d_shot_groups_match_reference(fwd, rev, many_oracle):
    d = load("acoustic2d_many")
    s = _acoustic(d, schedule={"shots_fwd": fwd, "shots_rev": rev})
    pred, g, gw = _acoustic_grad(s, d)
    got = s.launch_schedule(d["wavelet"].shape[-1], d["src"], d["rec"], [torch.tensor(d["vp_init"], device=DEV)])
    assert (got["shots_fwd"], got["shots_rev"]) == (fwd, rev)
    p64, _, g64, gw64 = many_oracle
    print(f"2-D 20 shots, {fwd}/{rev} shots per CTA: vs reference record {rel(pred, d['pred']):.2e} "
          f"grad {rel(g, d['grad_vp']):.2e} wavelet {rel(gw, d['grad_wavelet']):.2e}; vs f64 oracle "
          f"record {rel(pred, p64):.2e} grad {rel(g, g64):.2e} wavelet {rel(gw, gw64):.2e}")
    assert rel(pred, d["pred"]) < REC_TOL
    assert rel(g, d["grad_vp"]) < GRAD_TOL
    assert rel(gw, d["grad_wavelet"]) < GRAD_TOL
    assert rel(g, g64) < GRAD_TOL
    # padded receivers (off the grid) record zero
    for b in range(len(d["src"])):
        off = d["rec"][b, :, 0] < 0
        assert np.all(pred[b, :, off] == 0)


@pytest.fixture(scope="module")
def interior_oracle():
    d = load("elastic2d_interior")
    return O.elastic_gradient(d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"], d["rec"], d["obs"],
                              float(d["dh"]), float(d["dt"]), int(d["abcn"]), int(d["order"]), prec="f64")


@pytest.mark.parametrize("fwd,rev", [(1, 1), (2, 2), (2, 4)])
def test_elastic2d_interior_tiles_match_reference(fwd, rev, interior_oracle):
    from sweep_b200 import Elastic, PropTorch
    d = load("elastic2d_interior")
    s = PropTorch(Elastic(spatial_order=8, device=DEV), shape=tuple(d["vp_true"].shape), dh=float(d["dh"]),
                  dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV,
                  schedule={"shots_fwd": fwd, "shots_rev": rev})
    ms = [torch.tensor(d[k], device=DEV, requires_grad=True) for k in ("vp_init", "vs_init", "rho_init")]
    pred = s(torch.tensor(d["wavelet"], device=DEV), d["src"], d["rec"], models=ms)
    (0.5 * ((pred - torch.tensor(d["obs"], device=DEV)) ** 2).sum()).backward()
    torch.cuda.synchronize()
    pred = pred.detach().cpu().numpy()
    gs = [m.grad.cpu().numpy() for m in ms]
    p64, _, g64 = interior_oracle
    errs = [rel(g, d[f"grad_{k}"]) for g, k in zip(gs, ("vp", "vs", "rho"))]
    errs64 = [rel(g, o) for g, o in zip(gs, g64)]
    print(f"elastic interior, {fwd}/{rev} shots per CTA: vs reference record {rel(pred, d['pred']):.2e} "
          f"grads {errs[0]:.2e} {errs[1]:.2e} {errs[2]:.2e}; vs f64 oracle record {rel(pred, p64):.2e} "
          f"grads {errs64[0]:.2e} {errs64[1]:.2e} {errs64[2]:.2e}")
    assert rel(pred, d["pred"]) < REC_TOL
    assert max(errs) < GRAD_TOL
    assert max(errs64) < GRAD_TOL
