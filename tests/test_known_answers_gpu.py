"""Known-answer checks on the GPU that do not route through the reference's
discretisation, and the bounded-wait failure path.

* The 2-D analytic Green's function (the reference's own known-answer test,
  test/test_laplacian_zero_sum.py:83-122): a 10 Hz Ricker from a point
  source in a 2000 m/s medium on a 1.25 m grid (160 points per wavelength),
  recorded 300 m away, matches the analytic pressure to 1.5e-4 relative L2.
* The bounded wait: a CTA that waits on an mbarrier nothing arrives at gives
  up after its budget and the call returns an error; the GPU context stays
  usable and the next call succeeds."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")

V, F0, T_END, SIDE, OFFSET = 2000.0, 10.0, 0.45, 1600.0, 300.0


def _ricker(t):
    """Ricker wavelet of peak frequency F0 delayed by 1.2 / F0."""
    arg = (np.pi * F0 * (np.asarray(t) - 1.2 / F0)) ** 2
    return (1.0 - 2.0 * arg) * np.exp(-arg)


def _green_2d(times, r, n=4001):
    """Pressure at distance r of p_tt = V^2 Lap p + w(t) delta(x) (zero before
    t = 0): the 2-D Green's function H(t - r/V) / (2 pi V^2 sqrt(t^2 - r^2/V^2))
    convolved with w.  With tau = (r / V) cosh(u) the singular kernel becomes
    1 / (2 pi V^2) du, so p(t) = 1 / (2 pi V^2) * int_0^{acosh(V t / r)} w(t - tau(u)) du,
    integrated with the trapezoid rule on n points."""
    out = np.zeros(len(times))
    for k, t in enumerate(times):
        if V * t <= r:
            continue
        u = np.linspace(0.0, np.arccosh(V * t / r), n)
        out[k] = np.trapezoid(_ricker(t - (r / V) * np.cosh(u)), u) / (2.0 * np.pi * V * V)
    return out


def test_fine_grid_record_matches_the_analytic_green_function():
    from sweep_b200 import Acoustic, PropTorch
    dh = 1.25
    dt = 1e-4 * dh
    nt, n = int(round(T_END / dt)), int(round(SIDE / dh)) + 1
    c = (n - 1) // 2
    s = PropTorch(Acoustic(spatial_order=8, device=DEV), shape=(n, n), dh=dh, dt=dt, abcn=30, device=DEV)
    w = torch.tensor(_ricker(np.arange(nt) * dt), dtype=torch.float32, device=DEV)
    with torch.no_grad():
        rec = s(w, np.array([[c, c]]), np.array([[[c + int(round(OFFSET / dh)), c]]]),
                models=[torch.full((n, n), V, device=DEV)])
    # the step adds w[k] to the source cell after step k: the discrete source
    # term is (dh / dt)^2 w delta, and record column k holds p at (k + 1) dt
    trace = rec[0, :, 0, 0].double().cpu().numpy() * dt ** 2 / dh ** 2
    ref = _green_2d((np.arange(nt) + 1) * dt, OFFSET)
    err = np.linalg.norm(trace - ref) / np.linalg.norm(ref)
    print(f"analytic Green's function, order 8, dh {dh}: rel L2 {err:.2e}")
    assert err < 1.5e-4


def _selftest(budget, arrive):
    from sweep_b200 import _lib
    lib = _lib.load()
    err = ctypes.create_string_buffer(_lib.ERR_CAP)
    stream = torch.cuda.current_stream(DEV).cuda_stream
    rc = lib.sweep_b200_wait_selftest(budget, arrive, stream, err, _lib.ERR_CAP)
    return rc, err.value.decode()


def test_a_wait_that_never_completes_returns_an_error_and_the_gpu_stays_usable():
    torch.cuda.set_device(DEV)
    rc, msg = _selftest(100_000, 0)
    assert rc != 0 and "did not complete in time" in msg, (rc, msg)
    rc, msg = _selftest(100_000, 1)             # the same wait, satisfied
    assert rc == 0, msg
    rc, msg = _selftest(0, 1)                   # a budget outside the range is refused
    assert rc != 0 and "budget" in msg
    # the context is intact: a normal propagation runs and gives finite records
    from sweep_b200 import Acoustic, PropTorch
    s = PropTorch(Acoustic(spatial_order=8, device=DEV), shape=(32, 40), dh=10.0, dt=0.001, abcn=8, device=DEV)
    w = torch.tensor(_ricker(np.arange(120) * 0.001), dtype=torch.float32, device=DEV)
    with torch.no_grad():
        r = s(w, np.array([[10, 10]]), np.array([[[30, 10]]]), models=[torch.full((32, 40), 2000.0, device=DEV)])
    assert torch.isfinite(r).all() and float(r.abs().max()) > 0
