"""CPU oracle for the finite-difference hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only as the checker or the timed CPU
baseline; the product (``sweep_b200``) never imports, links or calls it.

It restates, in numpy plus the C kernels of ``fd_oracle.c`` (built by this
directory's Makefile into ``liboracle_f32.so`` / ``liboracle_f64.so``), the
reference's compiled ``impl='c'`` path:

* host-side set-up, restated from the reference's Python:
  ``fd_coefficients`` / ``second_derivative_coefficients_fp32``
  (``src/sweep/scalars.py:51-93``), ``_build_fd_coefficients``
  (``src/sweep/propagator/_c.py:1134-1156``), ``setup_pml`` /
  ``set_cpml_profiles_r`` (``src/sweep/equations/pml.py:157-269``; defaults
  ``max_vel=4500``, ``pml_freq=25``: ``src/sweep/propagator/base.py:1039-1040``),
  runtime geometry (``src/sweep/core/geometry.py:23-58``,
  ``src/sweep/propagator/_c.py:2184-2207``), replicate model padding and its
  crop adjoint (``src/sweep/utils/torch.py:8-41``);
* the per-step kernels (see ``fd_oracle.c``).

Pinned against the reference's own outputs: ``tests/golden/*.npz`` were made by
the reference itself (``tests/golden/make_golden.py``), and
``tests/test_oracle_golden.py`` checks this oracle against them.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from fractions import Fraction
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIBS: dict = {}


def build() -> None:
    """Compile the oracle's C kernels (both precisions) with the Makefile."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


class _FlushToZero:
    """The loaded oracle library with every ``oracle_*`` compute entry run
    between ``oracle_ftz(1)`` and ``oracle_ftz(0)``: subnormals flushed to
    zero in the OpenMP threads for the call, as the device does."""

    def __init__(self, lib):
        self._lib = lib
        lib.oracle_ftz.argtypes = [ctypes.c_int]
        lib.oracle_ftz.restype = None

    def __getattr__(self, name):
        fn = getattr(self._lib, name)
        if not name.startswith("oracle_") or name.endswith("_tape_len") or name == "oracle_ftz":
            return fn
        lib = self._lib

        def call(*args):
            lib.oracle_ftz(1)
            try:
                return fn(*args)
            finally:
                lib.oracle_ftz(0)
        return call


def _lib(prec: str):
    if prec not in _LIBS:
        path = HERE / f"liboracle_{prec}.so"
        if not path.exists():
            build()
        lib = ctypes.CDLL(str(path))
        real = ctypes.c_float if prec == "f32" else ctypes.c_double
        P = ctypes.c_void_p
        i, l = ctypes.c_int, ctypes.c_longlong
        geo = [i, i, i, i, i, P, real, real, real, P, P, P, P, P, P, P, P, P, l, i, P, P, i, P]
        lib.oracle_a2d_tape_len.restype = l
        lib.oracle_a2d_tape_len.argtypes = [i, i, i, i, i, P]
        lib.oracle_a2d_forward.restype = i
        lib.oracle_a2d_forward.argtypes = geo + [P, P]
        lib.oracle_a2d_backward.restype = i
        lib.oracle_a2d_backward.argtypes = geo + [P, P, P, P, P, P]
        geo3 = [i, i, i, i, i, i, P, real, real, real, real, P, P,
                P, P, P, P, P, P, P, P, P, P, l, i, P, P, i, P]
        if not hasattr(lib, "oracle_a3d_tape_len"):
            _LIBS[prec] = _FlushToZero(lib)
            return _LIBS[prec]
        lib.oracle_a3d_tape_len.restype = l
        lib.oracle_a3d_tape_len.argtypes = [i, i, i, i, i, i, P]
        lib.oracle_a3d_forward.restype = i
        lib.oracle_a3d_forward.argtypes = geo3 + [P, P]
        lib.oracle_a3d_backward.restype = i
        lib.oracle_a3d_backward.argtypes = geo3 + [P, P, P, P, P, P]
        geo_el = [i, i, i, i, i, P, real, real, real, P, P, P, P, P, l,
                  i, P, P, i, P, i, P, i, P, i]
        lib.oracle_el2d_tape_len.restype = l
        lib.oracle_el2d_tape_len.argtypes = [i, i, i, i, i, P]
        lib.oracle_el2d_forward.restype = i
        lib.oracle_el2d_forward.argtypes = geo_el + [P, P]
        lib.oracle_el2d_backward.restype = i
        lib.oracle_el2d_backward.argtypes = geo_el + [P, P, P, P, P]
        geo_el3 = [i, i, i, i, i, i, P, real, real, real, real, P, P, P, P, P, l,
                   i, P, P, i, P, i, P, i, P, i]
        lib.oracle_el3d_tape_len.restype = l
        lib.oracle_el3d_tape_len.argtypes = [i, i, i, i, i, i, P]
        lib.oracle_el3d_forward.restype = i
        lib.oracle_el3d_forward.argtypes = geo_el3 + [P, P]
        lib.oracle_el3d_backward.restype = i
        lib.oracle_el3d_backward.argtypes = geo_el3 + [P, P, P, P, P]
        geo_vti = [i, i, i, i, i, P, real, real, real, P, P, P, P, P, P, l,
                   i, P, P, i, P, i, P, i, P]
        lib.oracle_vti2d_tape_len.restype = l
        lib.oracle_vti2d_tape_len.argtypes = [i, i, i, i, i, P]
        lib.oracle_vti2d_forward.restype = i
        lib.oracle_vti2d_forward.argtypes = geo_vti + [P, P]
        lib.oracle_vti2d_backward.restype = i
        lib.oracle_vti2d_backward.argtypes = geo_vti + [P, P, P, P, P, P]
        geo_vti3 = [i, i, i, i, i, i, P, real, real, real, real, P, P, P, P, P, P, l,
                    i, P, P, i, P, i, P, i, P]
        lib.oracle_vti3d_tape_len.restype = l
        lib.oracle_vti3d_tape_len.argtypes = [i, i, i, i, i, i, P]
        lib.oracle_vti3d_forward.restype = i
        lib.oracle_vti3d_forward.argtypes = geo_vti3 + [P, P]
        lib.oracle_vti3d_backward.restype = i
        lib.oracle_vti3d_backward.argtypes = geo_vti3 + [P, P, P, P, P, P]
        _LIBS[prec] = _FlushToZero(lib)
    return _LIBS[prec]


# ----------------------------------------------------------------- scalars
def fd_coefficients(derivative_order: int, accuracy_order: int) -> np.ndarray:
    """Centred Taylor coefficients of the positive taps (``scalars.py:51-67``)."""
    n = accuracy_order // 2
    pts = np.arange(-n, n + 1, dtype=np.float64)
    mat = np.array([pts ** i for i in range(2 * n + 1)])
    rhs = np.zeros(2 * n + 1)
    rhs[derivative_order] = math.factorial(derivative_order)
    return np.linalg.solve(mat, rhs)[-n:]


def second_derivative_coefficients_fp32(order: int):
    """float32 ``(c0, c)`` with ``c0 + 2 sum(c) == 0`` exactly (``scalars.py:69-93``)."""
    c = fd_coefficients(2, order)
    c0 = np.float32(-2 * c.sum())
    c = c.astype(np.float32)
    residual = Fraction(float(c0)) + 2 * sum(Fraction(float(x)) for x in c)
    if residual:
        c[-1] = np.float32(float(Fraction(float(c[-1])) - residual / 2))
    return c0, c


def fd_tables(M: int):
    """``(lap, grad)`` float32 tables of length M+1 (``_c.py:1134-1156``)."""
    c0, c = second_derivative_coefficients_fp32(2 * M)
    lap = np.zeros(M + 1, np.float32)
    lap[0] = -c0
    lap[1:] = c
    grad = np.zeros(M + 1, np.float32)
    grad[1:] = fd_coefficients(1, 2 * M).astype(np.float32)
    return lap, grad


# -------------------------------------------------------------------- CPML
def setup_pml(width, start, max_pml, dt, n, max_vel, pml_freq, r_val=0.001, n_power=2, eps=1e-9,
              offset=0.0):
    """a, b profiles of one axis in float32 (``pml.py:216-269``); ``offset`` 0.5
    gives the half-grid profiles of the staggered CPML."""
    dtype = np.float32
    alpha0 = math.pi * pml_freq
    if max_pml == 0:
        return np.zeros(n, dtype), np.zeros(n, dtype)
    sigma0 = -(1 + n_power) * max_vel * math.log(r_val) / (2 * max_pml)
    x = np.arange(n, dtype=dtype) + dtype(offset)
    f0 = (dtype(start[0]) - x) / dtype(width[0]) if width[0] else np.zeros_like(x)
    f1 = (x - dtype(start[1])) / dtype(width[1]) if width[1] else np.zeros_like(x)
    frac = np.clip(np.maximum(f0, f1), 0.0, 1.0)
    sigma = dtype(sigma0) * (frac ** n_power)
    alpha = dtype(alpha0) * (dtype(1.0) - frac)
    sa = sigma + alpha
    sa = np.where(np.abs(sa) < eps, dtype(eps), sa)
    a = np.exp(-sa * abs(dt)).astype(dtype, copy=False)
    b = (sigma / sa) * (a - dtype(1.0))
    a = a.copy()
    a[frac == 0] = dtype(0.0)
    return a, b.astype(dtype, copy=False)


def cpml_profiles(pads, M, dt, spacing, shape, max_vel=4500.0, pml_freq=25.0):
    """Per axis (shape order) ``(a, b, db)`` on the runtime grid (``pml.py:157-214``).

    ``pads``: flat per-face PML widths ``[lo0, hi0, lo1, hi1, ...]``;
    ``shape``: the runtime shape (physical + 2 pad + 2 M per axis)."""
    out = []
    for d, n in enumerate(shape):
        w = pads[2 * d: 2 * d + 2]
        start = [float(M + w[0]), float(n - 1 - M - w[1])]
        max_pml = max(w[0] * spacing[d], w[1] * spacing[d])
        a, b = setup_pml(w, start, max_pml, dt, n, max_vel, pml_freq)
        db = np.gradient(b, spacing[d])
        out.append((a, b, db.astype(np.float32)))
    return out


def cpml_profiles_s(pads, M, dt, spacing, shape, max_vel=4500.0, pml_freq=25.0):
    """Staggered-grid profiles per axis (shape order): ``(a, b, a_half, b_half)``
    (``pml.py:81-154``; half = positions offset by half a cell)."""
    out = []
    for d, n in enumerate(shape):
        w = pads[2 * d: 2 * d + 2]
        start = [M + w[0], n - 1 - M - w[1]]
        max_pml = max(w[0] * spacing[d], w[1] * spacing[d])
        a, b = setup_pml(w, start, max_pml, dt, n, max_vel, pml_freq, offset=0.0)
        ah, bh = setup_pml(w, start, max_pml, dt, n, max_vel, pml_freq, offset=0.5)
        out.append((a, b, ah, bh))
    return out


def staggered_coefficients(M: int):
    """Exact staggered first-derivative weights ``a_1..a_M`` as Fractions
    (``scalars.py:25-49``; order 8 gives 1225/1024, -245/3072, 49/5120,
    -5/7168, the constants of ``operators/staggered.cuh:351-354``)."""
    out = []
    for m in range(1, M + 1):
        a = Fraction((-1) ** (m + 1), 2 * m - 1)
        for n in range(1, M + 1):
            if n != m:
                num = (2 * n - 1) ** 2
                a *= abs(Fraction(num, num - (2 * m - 1) ** 2))
        out.append(a)
    return out


# ---------------------------------------------------------------- geometry
def _batch_io(wavelet, src, rec, ndim):
    """``(B, 1, nt)`` wavelet, ``(B, 1, ndim)`` sources, ``(B, nrec, ndim)`` receivers."""
    src = np.asarray(src, np.int64).reshape(-1, ndim)
    B = src.shape[0]
    w = np.asarray(wavelet, np.float32)
    if w.ndim == 1:
        w = np.broadcast_to(w, (B, w.shape[0]))
    rec = np.asarray(rec, np.int64).reshape(B, -1, ndim)
    return np.ascontiguousarray(w[:, None, :]), src[:, None, :], rec


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class _Acoustic:
    """Shared set-up of the 2-D / 3-D acoustic oracle runs."""

    def __init__(self, vp, wavelet, src, rec, dh, dt, abcn, order=8, prec="f32",
                 max_vel=4500.0, pml_freq=25.0):
        self.prec = prec
        self.real = np.float32 if prec == "f32" else np.float64
        vp = np.asarray(vp, np.float32)
        self.ndim = 2 if src is not None and np.asarray(src).shape[-1] == 2 else 3
        nd = self.ndim
        self.per_shot = vp.ndim == nd + 1
        self.M = M = order // 2
        w, s, r = _batch_io(wavelet, src, rec, nd)
        self.B, self.nt = w.shape[0], w.shape[-1]
        phys = vp.shape[-nd:]
        self.phys = phys
        self.pad = abcn
        self.shape = tuple(n + 2 * abcn + 2 * M for n in phys)
        padw = [(abcn + M, abcn + M)] * nd
        lead = [(0, 0)] if self.per_shot else []
        self.vp = np.ascontiguousarray(np.pad(vp, lead + padw, mode="edge").astype(self.real))
        self.vp_stride = int(np.prod(self.shape)) if self.per_shot else 0
        sp = dh if np.ndim(dh) else [dh] * nd
        self.spacing = [float(x) for x in sp]
        self.dt = float(dt)
        prof = cpml_profiles([abcn] * (2 * nd), M, dt, self.spacing, self.shape, max_vel, pml_freq)
        self.prof = [tuple(np.ascontiguousarray(x.astype(self.real)) for x in p) for p in prof]
        lap, grad = fd_tables(M)
        self.lap, self.grad = lap.astype(self.real), grad.astype(self.real)
        off = abcn + M
        self.src = np.ascontiguousarray((s + off).astype(np.int32))
        self.rec = np.ascontiguousarray((r + off).astype(np.int32))
        self.wavelet = np.ascontiguousarray(w.astype(self.real))
        self.nrec = self.rec.shape[1]
        self.nsrc = 1

    def crop(self, g):
        M, a = self.M, self.pad
        sl = tuple(slice(a + M, a + M + n) for n in self.phys)
        return g[(Ellipsis,) + sl]


class Acoustic2D(_Acoustic):
    def _geo(self):
        nz, nx = self.shape
        (az, bz, dbz), (ax, bx, dbx) = self.prof
        pad = np.array([self.pad] * 4, np.int32)
        self._keep = (pad, az, bz, dbz, ax, bx, dbx)
        return [self.B, nz, nx, self.nt, self.M, _ptr(pad), self.dt, self.spacing[0],
                self.spacing[1], _ptr(self.lap), _ptr(self.grad), _ptr(az), _ptr(bz),
                _ptr(dbz), _ptr(ax), _ptr(bx), _ptr(dbx), _ptr(self.vp), self.vp_stride,
                self.nsrc, _ptr(self.src), _ptr(self.wavelet), self.nrec, _ptr(self.rec)]

    def forward(self, keep_tape=True):
        lib = _lib(self.prec)
        nz, nx = self.shape
        pad = np.array([self.pad] * 4, np.int32)
        rec = np.zeros((self.B, self.nrec, self.nt), self.real)
        self.tape = None
        if keep_tape:
            n = lib.oracle_a2d_tape_len(self.B, nz, nx, self.nt, self.M, _ptr(pad))
            self.tape = np.zeros(n, self.real)
        rc = lib.oracle_a2d_forward(*self._geo(), _ptr(rec),
                                    _ptr(self.tape) if keep_tape else None)
        assert rc == 0
        return rec.transpose(0, 2, 1)[..., None]                 # (B, nt, nrec, 1)

    def backward(self, adj, illum=False):
        """``adj``: record cotangent in the canonical ``(B, nt, nrec, 1)`` layout.
        With ``illum``, also the source and receiver illuminations
        (``sum_t u_tt^2``, ``sum_t lambda^2``, summed over shots, cropped)."""
        lib = _lib(self.prec)
        a = np.ascontiguousarray(np.asarray(adj)[..., 0].transpose(0, 2, 1).astype(self.real))
        g = np.zeros(((self.B,) if self.per_shot else ()) + self.shape, self.real)
        gw = np.zeros((self.B, 1, self.nt), self.real)
        i_s = np.zeros(self.shape, self.real) if illum else None
        i_r = np.zeros(self.shape, self.real) if illum else None
        rc = lib.oracle_a2d_backward(*self._geo(), _ptr(a), _ptr(self.tape), _ptr(g), _ptr(gw),
                                     _ptr(i_s) if illum else None, _ptr(i_r) if illum else None)
        assert rc == 0
        if illum:
            return self.crop(g), gw[:, 0, :], self.crop(i_s), self.crop(i_r)
        return self.crop(g), gw[:, 0, :]


class Acoustic3D(_Acoustic):
    def _geo(self):
        nz, ny, nx = self.shape
        (az, bz, dbz), (ay, by, dby), (ax, bx, dbx) = self.prof
        pad = np.array([self.pad] * 6, np.int32)
        self._keep = (pad,)
        return [self.B, nz, ny, nx, self.nt, self.M, _ptr(pad), self.dt, self.spacing[0],
                self.spacing[1], self.spacing[2], _ptr(self.lap), _ptr(self.grad),
                _ptr(az), _ptr(bz), _ptr(dbz), _ptr(ay), _ptr(by), _ptr(dby),
                _ptr(ax), _ptr(bx), _ptr(dbx), _ptr(self.vp), self.vp_stride,
                self.nsrc, _ptr(self.src), _ptr(self.wavelet), self.nrec, _ptr(self.rec)]

    def forward(self, keep_tape=True):
        lib = _lib(self.prec)
        nz, ny, nx = self.shape
        pad = np.array([self.pad] * 6, np.int32)
        rec = np.zeros((self.B, self.nrec, self.nt), self.real)
        self.tape = None
        if keep_tape:
            n = lib.oracle_a3d_tape_len(self.B, nz, ny, nx, self.nt, self.M, _ptr(pad))
            self.tape = np.zeros(n, self.real)
        rc = lib.oracle_a3d_forward(*self._geo(), _ptr(rec),
                                    _ptr(self.tape) if keep_tape else None)
        assert rc == 0
        return rec.transpose(0, 2, 1)[..., None]

    def backward(self, adj, illum=False):
        lib = _lib(self.prec)
        a = np.ascontiguousarray(np.asarray(adj)[..., 0].transpose(0, 2, 1).astype(self.real))
        g = np.zeros(self.shape, self.real)
        gw = np.zeros((self.B, 1, self.nt), self.real)
        i_s = np.zeros(self.shape, self.real) if illum else None
        i_r = np.zeros(self.shape, self.real) if illum else None
        rc = lib.oracle_a3d_backward(*self._geo(), _ptr(a), _ptr(self.tape), _ptr(g), _ptr(gw),
                                     _ptr(i_s) if illum else None, _ptr(i_r) if illum else None)
        assert rc == 0
        if illum:
            return self.crop(g), gw[:, 0, :], self.crop(i_s), self.crop(i_r)
        return self.crop(g), gw[:, 0, :]


def acoustic_gradient(vp, wavelet, src, rec, obs, dh, dt, abcn, order=8, prec="f32", illum=False, **kw):
    """Record, loss ``0.5 ||pred - obs||^2``, model gradient (cropped, summed over
    shots for a shared model) and wavelet gradient (summed over shots for a
    shared wavelet), like ``PropTorch(impl='c')`` + ``loss.backward()``.  With
    ``illum``, two more results: the source and receiver illuminations, as
    ``solver.compute_illumination = True`` gives them."""
    ndim = np.asarray(src).shape[-1]
    cls = Acoustic2D if ndim == 2 else Acoustic3D
    run = cls(vp, wavelet, src, rec, dh, dt, abcn, order, prec, **kw)
    pred = run.forward(keep_tape=True)
    res = pred - np.asarray(obs, run.real)
    loss = 0.5 * float(np.sum(res.astype(np.float64) ** 2))
    out = run.backward(res, illum=illum)
    g, gw = out[0], out[1]
    if np.asarray(wavelet).ndim == 1:
        gw = gw.sum(0)
    if illum:
        return pred, loss, g, gw, out[2], out[3]
    return pred, loss, g, gw


def acoustic_forward(vp, wavelet, src, rec, dh, dt, abcn, order=8, prec="f32", **kw):
    ndim = np.asarray(src).shape[-1]
    cls = Acoustic2D if ndim == 2 else Acoustic3D
    return cls(vp, wavelet, src, rec, dh, dt, abcn, order, prec, **kw).forward(keep_tape=False)


# ------------------------------------------------------------------ elastic
ELASTIC_FIELDS = ("vx", "vz", "sxx", "szz", "sxz")


def _el_faces(spec):
    """Free faces (z_lo, z_hi, x_lo, x_hi) from the reference's spellings."""
    names = ("top", "bottom", "left", "right")
    if spec is None or isinstance(spec, (bool, np.bool_)):
        return [bool(spec), False, False, False]
    if isinstance(spec, str):
        spec = [spec]
    spec = list(spec)
    if all(isinstance(v, str) for v in spec):
        return [n in spec for n in names]
    assert len(spec) == 4
    return [bool(v) for v in spec]


class Elastic2D:
    """2-D isotropic elastic oracle run (``fd_oracle_el.c``): models
    ``vp, vs, rho`` of shape ``(nz, nx)`` or per shot ``(B, nz, nx)``; source
    fields default to the explosive ``(sxx, szz)``, receiver fields to
    ``(vx, vz)`` (``src/sweep/equations/elastic.py:123-128``).
    ``free_surface``: traction-free faces with no PML pad, as the
    reference's ``PropTorch(free_surface=...)`` spells them: ``True`` (the
    top face), face names (``'top'``, ``'bottom'``, ``'left'``,
    ``'right'``) or four bools (z_lo, z_hi, x_lo, x_hi)."""

    def __init__(self, vp, vs, rho, wavelet, src, rec, dh, dt, abcn, order=8, prec="f32",
                 source_fields=("sxx", "szz"), receiver_fields=("vx", "vz"),
                 max_vel=4500.0, pml_freq=25.0, free_surface=False):
        self.prec = prec
        self.real = np.float32 if prec == "f32" else np.float64
        models = [np.asarray(m, np.float32) for m in (vp, vs, rho)]
        self.per_shot = models[0].ndim == 3
        self.M = M = order // 2
        w, s, r = _batch_io(wavelet, src, rec, 2)
        self.B, self.nt = w.shape[0], w.shape[-1]
        self.phys = models[0].shape[-2:]
        faces = _el_faces(free_surface)
        self.fs = sum(1 << f for f in range(4) if faces[f])
        self.pads = [0 if faces[f] else abcn for f in range(4)]   # z_lo, z_hi, x_lo, x_hi
        pz, px = self.pads[:2], self.pads[2:]
        self.shape = (self.phys[0] + sum(pz) + 2 * M, self.phys[1] + sum(px) + 2 * M)
        padw = [(pz[0] + M, pz[1] + M), (px[0] + M, px[1] + M)]
        lead = [(0, 0)] if self.per_shot else []
        self.models = [np.ascontiguousarray(np.pad(m, lead + padw, mode="edge").astype(self.real))
                       for m in models]
        self.m_stride = int(np.prod(self.shape)) if self.per_shot else 0
        sp = dh if np.ndim(dh) else [dh] * 2
        self.spacing = [float(x) for x in sp]
        self.dt = float(dt)
        prof = cpml_profiles_s(self.pads, M, dt, self.spacing, self.shape, max_vel, pml_freq)
        (az, bz, azh, bzh), (ax, bx, axh, bxh) = prof
        self.prof = np.ascontiguousarray(
            np.concatenate([az, bz, azh, bzh, ax, bx, axh, bxh]).astype(self.real))
        c = staggered_coefficients(M)
        self.coef = np.array([0.0] + [float(x) for x in c], np.float64).astype(self.real)
        if self.real is np.float32:
            self.coef = np.array([0.0] + [np.float32(float(x)) for x in c], np.float32)
        off = np.array([px[0] + M, pz[0] + M])          # (x, z)
        self.src = np.ascontiguousarray((s + off).astype(np.int32))
        self.rec = np.ascontiguousarray((r + off).astype(np.int32))
        self.wavelet = np.ascontiguousarray(w.astype(self.real))
        self.nrec = self.rec.shape[1]
        self.sf = np.array([ELASTIC_FIELDS.index(f) for f in source_fields], np.int32)
        self.rf = np.array([ELASTIC_FIELDS.index(f) for f in receiver_fields], np.int32)

    def _geo(self):
        nz, nx = self.shape
        self._pad = np.array(self.pads, np.int32)
        return [self.B, nz, nx, self.nt, self.M, _ptr(self._pad), self.dt, self.spacing[0],
                self.spacing[1], _ptr(self.coef), _ptr(self.prof), _ptr(self.models[0]),
                _ptr(self.models[1]), _ptr(self.models[2]), self.m_stride,
                1, _ptr(self.src), _ptr(self.wavelet), len(self.sf), _ptr(self.sf),
                self.nrec, _ptr(self.rec), len(self.rf), _ptr(self.rf), self.fs]

    def crop(self, g):
        M = self.M
        lo = (self.pads[0], self.pads[2])
        sl = tuple(slice(a + M, a + M + n) for a, n in zip(lo, self.phys))
        return g[(Ellipsis,) + sl]

    def forward(self, keep_tape=True):
        """Records ``(B, nt, nrec, nfield)``."""
        lib = _lib(self.prec)
        nz, nx = self.shape
        rec = np.zeros((self.B, self.nt, self.nrec, len(self.rf)), self.real)
        self.tape = None
        if keep_tape:
            pad = np.array(self.pads, np.int32)
            n = lib.oracle_el2d_tape_len(self.B, nz, nx, self.nt, self.M, _ptr(pad))
            self.tape = np.zeros(n, self.real)
        rc = lib.oracle_el2d_forward(*self._geo(), _ptr(rec),
                                     _ptr(self.tape) if keep_tape else None)
        assert rc == 0
        return rec

    def backward(self, adj):
        """``adj``: record cotangent ``(B, nt, nrec, nfield)``; returns the
        cropped ``(grad_vp, grad_vs, grad_rho)``."""
        lib = _lib(self.prec)
        a = np.ascontiguousarray(np.asarray(adj).astype(self.real))
        shp = ((self.B,) if self.per_shot else ()) + self.shape
        g = [np.zeros(shp, self.real) for _ in range(3)]
        rc = lib.oracle_el2d_backward(*self._geo(), _ptr(a), _ptr(self.tape),
                                      _ptr(g[0]), _ptr(g[1]), _ptr(g[2]))
        assert rc == 0
        return tuple(self.crop(x) for x in g)


def elastic_gradient(vp, vs, rho, wavelet, src, rec, obs, dh, dt, abcn, order=8, prec="f32", **kw):
    """Record, loss ``0.5 ||pred - obs||^2`` and cropped ``(vp, vs, rho)``
    gradients (summed over shots for shared models)."""
    run = Elastic2D(vp, vs, rho, wavelet, src, rec, dh, dt, abcn, order, prec, **kw)
    pred = run.forward(keep_tape=True)
    res = pred - np.asarray(obs, run.real)
    loss = 0.5 * float(np.sum(res.astype(np.float64) ** 2))
    return pred, loss, run.backward(res)


def elastic_forward(vp, vs, rho, wavelet, src, rec, dh, dt, abcn, order=8, prec="f32", **kw):
    return Elastic2D(vp, vs, rho, wavelet, src, rec, dh, dt, abcn, order, prec, **kw).forward(
        keep_tape=False)


ELASTIC3D_FIELDS = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")


class Elastic3D:
    """3-D isotropic elastic oracle run (``fd_oracle_el3d.c``): models
    ``vp, vs, rho`` of shape ``(nz, ny, nx)`` or per shot ``(B, nz, ny, nx)``;
    coordinates ``(x, y, z)``; source fields default to the explosive
    ``(sxx, syy, szz)``, receiver fields to ``(vx, vy, vz)``
    (``src/sweep/equations/elastic3d.py:326-332``).  ``free_surface=True``:
    a traction-free top face with no PML pad."""

    def __init__(self, vp, vs, rho, wavelet, src, rec, dh, dt, abcn, order=8, prec="f32",
                 source_fields=("sxx", "syy", "szz"), receiver_fields=("vx", "vy", "vz"),
                 max_vel=4500.0, pml_freq=25.0, free_surface=False):
        self.prec = prec
        self.real = np.float32 if prec == "f32" else np.float64
        models = [np.asarray(m, np.float32) for m in (vp, vs, rho)]
        self.per_shot = models[0].ndim == 4
        self.M = M = order // 2
        w, s, r = _batch_io(wavelet, src, rec, 3)
        self.B, self.nt = w.shape[0], w.shape[-1]
        self.phys = models[0].shape[-3:]
        self.fs = 1 if free_surface else 0
        self.pads = [0 if free_surface else abcn] + [abcn] * 5   # z_lo, z_hi, y_lo, y_hi, x_lo, x_hi
        self.shape = tuple(n + self.pads[2 * a] + self.pads[2 * a + 1] + 2 * M for a, n in enumerate(self.phys))
        padw = [(self.pads[2 * a] + M, self.pads[2 * a + 1] + M) for a in range(3)]
        lead = [(0, 0)] if self.per_shot else []
        self.models = [np.ascontiguousarray(np.pad(m, lead + padw, mode="edge").astype(self.real))
                       for m in models]
        self.m_stride = int(np.prod(self.shape)) if self.per_shot else 0
        sp = dh if np.ndim(dh) else [dh] * 3
        self.spacing = [float(x) for x in sp]
        self.dt = float(dt)
        prof = cpml_profiles_s(self.pads, M, dt, self.spacing, self.shape, max_vel, pml_freq)
        self.prof = np.ascontiguousarray(np.concatenate([np.concatenate(p) for p in prof]).astype(self.real))
        c = staggered_coefficients(M)
        self.coef = np.array([0.0] + [float(x) for x in c], np.float64).astype(self.real)
        if self.real is np.float32:
            self.coef = np.array([0.0] + [np.float32(float(x)) for x in c], np.float32)
        off = np.array([self.pads[4] + M, self.pads[2] + M, self.pads[0] + M])   # (x, y, z)
        self.src = np.ascontiguousarray((s + off).astype(np.int32))
        self.rec = np.ascontiguousarray((r + off).astype(np.int32))
        self.wavelet = np.ascontiguousarray(w.astype(self.real))
        self.nrec = self.rec.shape[1]
        self.sf = np.array([ELASTIC3D_FIELDS.index(f) for f in source_fields], np.int32)
        self.rf = np.array([ELASTIC3D_FIELDS.index(f) for f in receiver_fields], np.int32)

    def _geo(self):
        nz, ny, nx = self.shape
        self._pad = np.array(self.pads, np.int32)
        return [self.B, nz, ny, nx, self.nt, self.M, _ptr(self._pad), self.dt, self.spacing[0],
                self.spacing[1], self.spacing[2], _ptr(self.coef), _ptr(self.prof), _ptr(self.models[0]),
                _ptr(self.models[1]), _ptr(self.models[2]), self.m_stride,
                1, _ptr(self.src), _ptr(self.wavelet), len(self.sf), _ptr(self.sf),
                self.nrec, _ptr(self.rec), len(self.rf), _ptr(self.rf), self.fs]

    def crop(self, g):
        M = self.M
        sl = tuple(slice(self.pads[2 * a] + M, self.pads[2 * a] + M + n) for a, n in enumerate(self.phys))
        return g[(Ellipsis,) + sl]

    def forward(self, keep_tape=True):
        """Records ``(B, nt, nrec, nfield)``."""
        lib = _lib(self.prec)
        nz, ny, nx = self.shape
        rec = np.zeros((self.B, self.nt, self.nrec, len(self.rf)), self.real)
        self.tape = None
        if keep_tape:
            pad = np.array(self.pads, np.int32)
            n = lib.oracle_el3d_tape_len(self.B, nz, ny, nx, self.nt, self.M, _ptr(pad))
            self.tape = np.zeros(n, self.real)
        rc = lib.oracle_el3d_forward(*self._geo(), _ptr(rec), _ptr(self.tape) if keep_tape else None)
        assert rc == 0
        return rec

    def backward(self, adj):
        """``adj``: record cotangent ``(B, nt, nrec, nfield)``; returns the
        cropped ``(grad_vp, grad_vs, grad_rho)``."""
        lib = _lib(self.prec)
        a = np.ascontiguousarray(np.asarray(adj).astype(self.real))
        shp = ((self.B,) if self.per_shot else ()) + self.shape
        g = [np.zeros(shp, self.real) for _ in range(3)]
        rc = lib.oracle_el3d_backward(*self._geo(), _ptr(a), _ptr(self.tape), _ptr(g[0]), _ptr(g[1]),
                                      _ptr(g[2]))
        assert rc == 0
        return tuple(self.crop(x) for x in g)


def elastic3d_gradient(vp, vs, rho, wavelet, src, rec, obs, dh, dt, abcn, order=8, prec="f32", **kw):
    """Record, loss ``0.5 ||pred - obs||^2`` and cropped ``(vp, vs, rho)``
    gradients of the 3-D elastic oracle (summed over shots for shared models)."""
    run = Elastic3D(vp, vs, rho, wavelet, src, rec, dh, dt, abcn, order, prec, **kw)
    pred = run.forward(keep_tape=True)
    res = pred - np.asarray(obs, run.real)
    loss = 0.5 * float(np.sum(res.astype(np.float64) ** 2))
    return pred, loss, run.backward(res)


def elastic3d_forward(vp, vs, rho, wavelet, src, rec, dh, dt, abcn, order=8, prec="f32", **kw):
    return Elastic3D(vp, vs, rho, wavelet, src, rec, dh, dt, abcn, order, prec, **kw).forward(keep_tape=False)


# --------------------------------------------------------------- acoustic VTI
VTI_FIELDS = ("vx", "vz", "sH", "sV")


class VTI2D:
    """One float32 / float64 run of the 2-D first-order acoustic VTI oracle
    (``fd_oracle_vti.c``; reference ``sweep.equations.AcousticVTI1st``).

    Models ``vp, epsilon, delta, rho`` of shape ``(nz, nx)`` or per shot
    ``(B, nz, nx)``; source fields default to ``(sH, sV)``, receiver fields
    to ``(vz,)`` (``src/sweep/equations/acoustic_vti_1st.py:324-330``)."""

    def __init__(self, vp, eps, delta, rho, wavelet, src, rec, dh, dt, abcn, order=8, prec="f32",
                 source_fields=("sH", "sV"), receiver_fields=("vz",), max_vel=4500.0, pml_freq=25.0):
        self.prec = prec
        self.real = np.float32 if prec == "f32" else np.float64
        models = [np.asarray(m, np.float32) for m in (vp, eps, delta, rho)]
        self.per_shot = models[0].ndim == 3
        self.M = M = order // 2
        w, s, r = _batch_io(wavelet, src, rec, 2)
        self.B, self.nt = w.shape[0], w.shape[-1]
        self.phys = models[0].shape[-2:]
        self.pads = [abcn] * 4
        self.shape = (self.phys[0] + 2 * abcn + 2 * M, self.phys[1] + 2 * abcn + 2 * M)
        padw = [(abcn + M, abcn + M)] * 2
        lead = [(0, 0)] if self.per_shot else []
        self.models = [np.ascontiguousarray(np.pad(m, lead + padw, mode="edge").astype(self.real))
                       for m in models]
        self.m_stride = int(np.prod(self.shape)) if self.per_shot else 0
        sp = dh if np.ndim(dh) else [dh] * 2
        self.spacing = [float(x) for x in sp]
        self.dt = float(dt)
        prof = cpml_profiles_s(self.pads, M, dt, self.spacing, self.shape, max_vel, pml_freq)
        (az, bz, azh, bzh), (ax, bx, axh, bxh) = prof
        self.prof = np.ascontiguousarray(
            np.concatenate([az, bz, azh, bzh, ax, bx, axh, bxh]).astype(self.real))
        c = staggered_coefficients(M)
        if self.real is np.float32:
            self.coef = np.array([0.0] + [np.float32(float(x)) for x in c], np.float32)
        else:
            self.coef = np.array([0.0] + [float(x) for x in c], np.float64)
        off = np.array([abcn + M, abcn + M])
        self.src = np.ascontiguousarray((s + off).astype(np.int32))
        self.rec = np.ascontiguousarray((r + off).astype(np.int32))
        self.wavelet = np.ascontiguousarray(w.astype(self.real))
        self.nrec = self.rec.shape[1]
        self.sf = np.array([VTI_FIELDS.index(f) for f in source_fields], np.int32)
        self.rf = np.array([VTI_FIELDS.index(f) for f in receiver_fields], np.int32)

    def _geo(self):
        nz, nx = self.shape
        self._pad = np.array(self.pads, np.int32)
        return [self.B, nz, nx, self.nt, self.M, _ptr(self._pad), self.dt, self.spacing[0],
                self.spacing[1], _ptr(self.coef), _ptr(self.prof)] + [_ptr(m) for m in self.models] + [
                self.m_stride, 1, _ptr(self.src), _ptr(self.wavelet), len(self.sf), _ptr(self.sf),
                self.nrec, _ptr(self.rec), len(self.rf), _ptr(self.rf)]

    def crop(self, g):
        M, a = self.M, self.pads[0]
        sl = tuple(slice(a + M, a + M + n) for n in self.phys)
        return g[(Ellipsis,) + sl]

    def forward(self, keep_tape=True):
        """Records ``(B, nt, nrec, nfield)``."""
        lib = _lib(self.prec)
        nz, nx = self.shape
        rec = np.zeros((self.B, self.nt, self.nrec, len(self.rf)), self.real)
        self.tape = None
        if keep_tape:
            pad = np.array(self.pads, np.int32)
            self.tape = np.zeros(lib.oracle_vti2d_tape_len(self.B, nz, nx, self.nt, self.M, _ptr(pad)), self.real)
        rc = lib.oracle_vti2d_forward(*self._geo(), _ptr(rec), _ptr(self.tape) if keep_tape else None)
        assert rc == 0
        return rec

    def backward(self, adj):
        """``adj``: record cotangent ``(B, nt, nrec, nfield)``; returns the
        cropped ``(grad_vp, grad_epsilon, grad_delta, grad_rho)``."""
        lib = _lib(self.prec)
        a = np.ascontiguousarray(np.asarray(adj).astype(self.real))
        shp = ((self.B,) if self.per_shot else ()) + self.shape
        g = [np.zeros(shp, self.real) for _ in range(4)]
        rc = lib.oracle_vti2d_backward(*self._geo(), _ptr(a), _ptr(self.tape),
                                       *[_ptr(x) for x in g])
        assert rc == 0
        return tuple(self.crop(x) for x in g)


def vti2d_gradient(vp, eps, delta, rho, wavelet, src, rec, obs, dh, dt, abcn, order=8, prec="f32", **kw):
    """Record, loss ``0.5 ||pred - obs||^2`` and cropped ``(vp, epsilon,
    delta, rho)`` gradients (summed over shots for shared models)."""
    run = VTI2D(vp, eps, delta, rho, wavelet, src, rec, dh, dt, abcn, order, prec, **kw)
    pred = run.forward(keep_tape=True)
    res = pred - np.asarray(obs, run.real)
    loss = 0.5 * float(np.sum(res.astype(np.float64) ** 2))
    return pred, loss, run.backward(res)


def vti2d_forward(vp, eps, delta, rho, wavelet, src, rec, dh, dt, abcn, order=8, prec="f32", **kw):
    return VTI2D(vp, eps, delta, rho, wavelet, src, rec, dh, dt, abcn, order, prec, **kw).forward(keep_tape=False)


VTI3_FIELDS = ("vx", "vy", "vz", "sH", "sV")


class VTI3D:
    """One float32 / float64 run of the 3-D first-order acoustic VTI oracle
    (``fd_oracle_vti3d.c``; reference ``sweep.equations.AcousticVTI1st3D``).

    Models ``vp, epsilon, delta, rho`` of shape ``(nz, ny, nx)`` or per shot
    ``(B, nz, ny, nx)``; coordinates ``(x, y, z)``; source fields default to
    ``(sH, sV)``, receiver fields to ``(vz,)``
    (``src/sweep/equations/acoustic_vti_1st.py:530-536``)."""

    def __init__(self, vp, eps, delta, rho, wavelet, src, rec, dh, dt, abcn, order=4, prec="f32",
                 source_fields=("sH", "sV"), receiver_fields=("vz",), max_vel=4500.0, pml_freq=25.0):
        self.prec = prec
        self.real = np.float32 if prec == "f32" else np.float64
        models = [np.asarray(m, np.float32) for m in (vp, eps, delta, rho)]
        self.per_shot = models[0].ndim == 4
        self.M = M = order // 2
        w, s, r = _batch_io(wavelet, src, rec, 3)
        self.B, self.nt = w.shape[0], w.shape[-1]
        self.phys = models[0].shape[-3:]
        self.pads = [abcn] * 6                   # z_lo, z_hi, y_lo, y_hi, x_lo, x_hi
        self.shape = tuple(n + 2 * abcn + 2 * M for n in self.phys)
        padw = [(abcn + M, abcn + M)] * 3
        lead = [(0, 0)] if self.per_shot else []
        self.models = [np.ascontiguousarray(np.pad(m, lead + padw, mode="edge").astype(self.real))
                       for m in models]
        self.m_stride = int(np.prod(self.shape)) if self.per_shot else 0
        sp = dh if np.ndim(dh) else [dh] * 3
        self.spacing = [float(x) for x in sp]
        self.dt = float(dt)
        prof = cpml_profiles_s(self.pads, M, dt, self.spacing, self.shape, max_vel, pml_freq)
        self.prof = np.ascontiguousarray(np.concatenate([np.concatenate(p) for p in prof]).astype(self.real))
        c = staggered_coefficients(M)
        if self.real is np.float32:
            self.coef = np.array([0.0] + [np.float32(float(x)) for x in c], np.float32)
        else:
            self.coef = np.array([0.0] + [float(x) for x in c], np.float64)
        off = np.full(3, abcn + M)
        self.src = np.ascontiguousarray((s + off).astype(np.int32))
        self.rec = np.ascontiguousarray((r + off).astype(np.int32))
        self.wavelet = np.ascontiguousarray(w.astype(self.real))
        self.nrec = self.rec.shape[1]
        self.sf = np.array([VTI3_FIELDS.index(f) for f in source_fields], np.int32)
        self.rf = np.array([VTI3_FIELDS.index(f) for f in receiver_fields], np.int32)
        self._pad = np.array(self.pads, np.int32)

    def _geo(self):
        nz, ny, nx = self.shape
        return [self.B, nz, ny, nx, self.nt, self.M, _ptr(self._pad), self.dt, *self.spacing,
                _ptr(self.coef), _ptr(self.prof)] + [_ptr(m) for m in self.models] + [
                self.m_stride, self.src.shape[1], _ptr(self.src), _ptr(self.wavelet), len(self.sf), _ptr(self.sf),
                self.nrec, _ptr(self.rec), len(self.rf), _ptr(self.rf)]

    def crop(self, g):
        M, a = self.M, self.pads[0]
        sl = tuple(slice(a + M, a + M + n) for n in self.phys)
        return g[(Ellipsis,) + sl]

    def forward(self, keep_tape=True):
        """Records ``(B, nt, nrec, nfield)``."""
        lib = _lib(self.prec)
        nz, ny, nx = self.shape
        rec = np.zeros((self.B, self.nt, self.nrec, len(self.rf)), self.real)
        self.tape = None
        if keep_tape:
            self.tape = np.zeros(lib.oracle_vti3d_tape_len(self.B, nz, ny, nx, self.nt, self.M, _ptr(self._pad)),
                                 self.real)
        rc = lib.oracle_vti3d_forward(*self._geo(), _ptr(rec), _ptr(self.tape) if keep_tape else None)
        assert rc == 0
        return rec

    def backward(self, adj):
        """``adj``: record cotangent ``(B, nt, nrec, nfield)``; returns the
        cropped ``(grad_vp, grad_epsilon, grad_delta, grad_rho)``."""
        lib = _lib(self.prec)
        a = np.ascontiguousarray(np.asarray(adj).astype(self.real))
        shp = ((self.B,) if self.per_shot else ()) + self.shape
        g = [np.zeros(shp, self.real) for _ in range(4)]
        rc = lib.oracle_vti3d_backward(*self._geo(), _ptr(a), _ptr(self.tape), *[_ptr(x) for x in g])
        assert rc == 0
        return tuple(self.crop(x) for x in g)


def vti3d_gradient(vp, eps, delta, rho, wavelet, src, rec, obs, dh, dt, abcn, order=4, prec="f32", **kw):
    """Record, loss ``0.5 ||pred - obs||^2`` and cropped ``(vp, epsilon,
    delta, rho)`` gradients (summed over shots for shared models)."""
    run = VTI3D(vp, eps, delta, rho, wavelet, src, rec, dh, dt, abcn, order, prec, **kw)
    pred = run.forward(keep_tape=True)
    res = pred - np.asarray(obs, run.real)
    loss = 0.5 * float(np.sum(res.astype(np.float64) ** 2))
    return pred, loss, run.backward(res)


def vti3d_forward(vp, eps, delta, rho, wavelet, src, rec, dh, dt, abcn, order=4, prec="f32", **kw):
    return VTI3D(vp, eps, delta, rho, wavelet, src, rec, dh, dt, abcn, order, prec, **kw).forward(keep_tape=False)
