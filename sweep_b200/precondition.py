"""Learned preconditioning of acoustic FWI: training pairs made by this
solver, U-Net training, and the FWI loop with the plain illumination-
preconditioned gradient as the fallback: a learned step is kept only when
the data misfit drops.

* ``plain_direction``: -grad / (illumination + eps max(illumination)), the
  reference's plain preconditioning (``_c.py:1050-1058``, used in
  ``examples/multi-gpu/torch/fwi_marmousi_dist.py:338-360``).
* ``make_pairs``: seeded random layered models, a smoothed start, the solver's
  own gradient and source illumination at the start, and the target
  (true - start) scaled to unit RMS.
* ``train``: Adam on the U-Net (BF16 tensor-core convolutions, FP32 masters).
* ``fwi``: gradient descent with a 3-point line search along the step
  direction; with a network, the learned direction is tried first and kept
  only if the data misfit drops, else the plain step is taken.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .equations import Acoustic
from .propagator import PropTorch
from .signal import ricker
from .unet import check as unet_check

__all__ = ["Survey", "layered_model", "plain_direction", "make_pairs", "train", "fwi"]


@dataclass
class Survey:
    """A 2-D acoustic FWI geometry: surface shots and a surface receiver line."""
    nz: int = 128
    nx: int = 384
    dh: float = 10.0
    dt: float = 0.001
    nt: int = 1200
    abcn: int = 20
    nshot: int = 8
    f0: float = 8.0
    delay: float = 0.12
    device: str = "cuda"
    solver: PropTorch = field(init=False, repr=False)

    def __post_init__(self):
        dev = torch.device(self.device)
        self.solver = PropTorch(Acoustic(spatial_order=8, device=dev), shape=(self.nz, self.nx), dh=self.dh,
                                dt=self.dt, abcn=self.abcn, device=dev)
        sx = np.linspace(8, self.nx - 9, self.nshot).astype(np.int64)
        self.src = np.stack([sx, np.full(self.nshot, 2)], -1)
        rx = np.arange(0, self.nx, 2)
        self.rec = np.broadcast_to(np.stack([rx, np.full(rx.size, 2)], -1), (self.nshot, rx.size, 2)).copy()
        w = ricker(np.arange(self.nt) * self.dt - self.delay, self.f0).astype(np.float32)
        self.wavelet = torch.tensor(w, device=dev)

    def model(self, vp):
        return self.solver(self.wavelet, self.src, self.rec, models=[vp])

    def misfit(self, vp, obs):
        with torch.no_grad():
            return 0.5 * float(((self.model(vp) - obs).double() ** 2).sum())

    def gradient(self, vp, obs):
        """(misfit, gradient, source illumination) at vp."""
        m = vp.detach().clone().requires_grad_(True)
        self.solver.compute_illumination = True
        try:
            pred = self.model(m)
            loss = 0.5 * ((pred - obs) ** 2).sum()
            loss.backward()
        finally:
            self.solver.compute_illumination = False
        return float(loss.detach()), m.grad.detach(), self.solver.source_illumination.detach()


def layered_model(nz, nx, rng, vmin=1500.0, vmax=4000.0, nlayers=8):
    """Seeded layered model: sorted-uniform interface depths perturbed by 3
    sinusoids, monotone velocities with 5 % noise."""
    depth = np.sort(rng.uniform(0.08 * nz, 0.95 * nz, nlayers - 1))
    x = np.arange(nx)
    surf = np.empty((nlayers - 1, nx))
    for i in range(nlayers - 1):
        amp, k, ph = rng.uniform(0, 2.5, 3), rng.uniform(1, 5, 3), rng.uniform(0, 2 * np.pi, 3)
        surf[i] = depth[i] + sum(amp[j] * np.sin(2 * np.pi * k[j] * x / nx + ph[j]) for j in range(3))
    vel = np.linspace(vmin, vmax, nlayers) * (1 + 0.05 * rng.standard_normal(nlayers))
    idx = (np.arange(nz)[:, None][None] > surf[:, None, :]).sum(0)
    return vel[idx].astype(np.float32)


def smooth(vp, sigma=8.0):
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(np.asarray(vp, np.float64), sigma).astype(np.float32)


def plain_direction(grad, illum, eps=1e-3):
    """The illumination-preconditioned descent direction."""
    return -grad / (illum + eps * illum.max())


def _standardise(a):
    return (a - a.mean()) / (a.std() + 1e-30)


def features(grad, illum, vp):
    """Network input (3, nz, nx): standardised gradient, illumination and vp."""
    return torch.stack([_standardise(grad), _standardise(illum), _standardise(vp)])


def make_pairs(survey: Survey, n, seed=0):
    """n (input, target) pairs from seeded random models."""
    rng = np.random.default_rng(seed)
    xs, ys = [], []
    dev = survey.wavelet.device
    for _ in range(n):
        vt = layered_model(survey.nz, survey.nx, rng)
        v0 = smooth(vt)
        vt_d, v0_d = torch.tensor(vt, device=dev), torch.tensor(v0, device=dev)
        with torch.no_grad():
            obs = survey.model(vt_d)
        _, g, il = survey.gradient(v0_d, obs)
        t = vt_d - v0_d
        xs.append(features(g, il, v0_d))
        ys.append((t / (t.pow(2).mean().sqrt() + 1e-30))[None])
    return torch.stack(xs), torch.stack(ys)


def train(net, xs, ys, steps, batch=16, lr=1e-3, seed=0, log_every=0):
    """Adam on 0.5 ||net(x) - y||^2 (mean); returns the loss history."""
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    for s in range(steps):
        idx = torch.randint(0, xs.shape[0], (batch,), generator=gen)
        pred = net(xs[idx])
        loss = 0.5 * ((pred - ys[idx]) ** 2).mean()
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        hist.append(float(loss))
        if log_every and s % log_every == 0:
            print(f"step {s}: loss {hist[-1]:.4f}")
    unet_check(xs.device)
    return hist


def _line_search(survey, vp, d, obs, f0, alpha0, vmin, vmax, shrink=4):
    """3-point line search along d: misfit at 0, a and 2a; the parabola's
    minimiser (clipped to [0, 4a]) if it improves, else the best tried point.
    Without a decrease the trial step shrinks 4-fold, ``shrink`` times at most.
    Every trial model is clamped to [vmin, vmax], so the misfit returned is
    the one of the model a step would take."""
    a0 = alpha0
    trial = lambda a: survey.misfit((vp + a * d).clamp(vmin, vmax), obs)  # noqa: E731
    for _ in range(shrink + 1):
        f1 = trial(a0)
        f2 = trial(2 * a0)
        den = f0 - 2 * f1 + f2
        best_a, best_f = (a0, f1) if f1 <= f2 else (2 * a0, f2)
        if den > 0:
            a = a0 * (3 * f0 - 4 * f1 + f2) / (2 * den)
            a = min(max(a, 0.0), 4 * a0)
            if a > 0:
                fa = trial(a)
                if fa < best_f:
                    best_a, best_f = a, fa
        if best_f < f0:
            return best_a, best_f
        a0 *= 0.25
    return best_a, best_f


def fwi(survey: Survey, v0, obs, iters, net=None, step_ms=20.0, vmin=1400.0, vmax=4600.0, accept=0.01):
    """Gradient-descent FWI.  Each iteration scales the direction to unit
    maximum and line-searches it (3 points); the first trial step is 1.5 times
    the last step taken along that kind of direction (``step_ms`` m/s to start
    the plain direction, 4 ``step_ms`` the learned one, which predicts the
    whole remaining update).  With a network its direction is tried first and
    kept when it lowers the data misfit by at least the fraction ``accept``;
    otherwise the plain illumination-preconditioned step is taken.  A step is
    taken only when the misfit of the (clamped) model it leads to is below the
    current one, so the misfit history decreases strictly.  Returns (vp, misfit before
    each iteration and after the last, wall-clock seconds after each
    iteration, number of learned steps taken)."""
    vp = v0.detach().clone()
    hist, times, learned = [], [], 0
    a_plain, a_learned = step_ms, 4 * step_ms
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(iters):
        f0, g, il = survey.gradient(vp, obs)
        if not hist:
            hist.append(f0)
        fcur = hist[-1]
        step = None
        if net is not None:
            with torch.no_grad():
                dl = net(features(g, il, vp)[None])[0, 0].float()
            dl = dl / (dl.abs().max() + 1e-30)
            al, fl = _line_search(survey, vp, dl, obs, f0, a_learned, vmin, vmax)
            if fl < (1.0 - accept) * fcur:
                step = (fl, vp + al * dl)
                a_learned = max(1.5 * al, step_ms)
                learned += 1
        if step is None:
            dp = plain_direction(g, il)
            dp = dp / (dp.abs().max() + 1e-30)
            ap, fp = _line_search(survey, vp, dp, obs, f0, a_plain, vmin, vmax)
            if fp >= fcur:
                break
            step = (fp, vp + ap * dp)
            a_plain = max(1.5 * ap, 0.25 * step_ms)
        vp = step[1].clamp(vmin, vmax)
        torch.cuda.synchronize()
        hist.append(step[0])
        times.append(time.perf_counter() - t0)
    return vp, hist, times, learned
