"""``PropTorch``: the drop-in propagator over the B200 core.

Mirrors the reference's ``PropTorch(equation, shape, dh, dt, abcn, impl='c',
memory=...)`` and its call ``solver(wavelet, sources, receivers, models=[...])``
(reference ``src/sweep/propagator/torch.py:576-825``,
``src/sweep/propagator/_c.py:2209-2599``): the same constructor keywords,
input modes, coordinate and padding conventions and record layout
``(B, nt, nrec, nfield)``, and ``.backward()`` fills the models' (and, for the
acoustic equations, the wavelet's) gradients through a
``torch.autograd.Function`` whose forward and backward each make one call into
``libsweep_b200.so``.

Host-side conventions restated from the reference:
* runtime grid = physical + ``abcn`` PML cells + ``M = so/2`` halo per face
  (``core/geometry.py:23-58``); coordinates shift by ``abcn + M``
  (``_c.py:2196-2207``); ``free_surface=True`` drops the top face's PML
  cells, so the surface row sits M cells from the grid's top; acoustic keeps
  the halo rows above it at zero pressure, elastic makes the face traction
  free by the image method (``common/elastic_free_surface.cuh``);
* models are replicate-padded to the runtime grid and the gradient cropped back
  (``utils/torch.py:8-41``); a shared model is used by every shot and its
  gradient summed over shots (``_c.py:2110-2155``);
* the wavelet is the raw amplitude added to the field at the source cell each
  step (``common/common.cu:11-36``);
* a second backward through the same forward is refused (``_c.py:612-625``).
"""
from __future__ import annotations

import os

import numpy as np
import torch
import torch.nn.functional as F

from . import _lib
from .equations import Acoustic, Acoustic3D, AcousticVTI1st, Elastic, Elastic3D
from .options import BoundarySaving, Ckpt, Full
from .pml import cpml_profiles_r, cpml_profiles_s
from .scalars import centred_tables, staggered_grid_coes

__all__ = ["PropTorch"]


def _as_tensor(x, dtype, device):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype)
    return torch.as_tensor(np.asarray(x), dtype=dtype, device=device)


def normalize_io(wavelet, sources, receivers, ndim):
    """Input modes of the reference (``core/validation.py:35-127``).

    Returns ``(mode, B, nsrc)``: 'A1' shared wavelet ``(nt,)`` + sources
    ``(B, ndim)``; 'A2' per-shot wavelets ``(B, nt)`` + sources ``(B, ndim)``;
    'B' one super-shot of ``nsrc`` sources ``(1, nsrc, ndim)`` with a wavelet
    ``(nt,)`` or ``(nsrc, nt)``."""
    ws = tuple(wavelet.shape)
    ss = tuple(np.shape(sources))
    rs = tuple(np.shape(receivers))
    if len(rs) != 3 or rs[-1] != ndim:
        raise ValueError(f"receivers must be (B, nrec, {ndim}); got {rs}")
    if len(ss) == 2 and ss[-1] == ndim:
        B = ss[0]
        if len(ws) == 1:
            mode = "A1"
        elif len(ws) == 2 and ws[0] == B:
            mode = "A2"
        else:
            raise ValueError(f"wavelet must be (nt,) or (nshots={B}, nt); got {ws}")
        nsrc = 1
    elif len(ss) == 3 and ss[0] == 1 and ss[-1] == ndim:
        B, nsrc = 1, ss[1]
        if not (len(ws) == 1 or (len(ws) == 2 and ws[0] == nsrc)):
            raise ValueError(f"wavelet must be (nt,) or (nsrc={nsrc}, nt) in source-encoding mode; got {ws}")
        mode = "B"
    else:
        raise ValueError(f"sources must be (nshots, {ndim}) or (1, nsrc, {ndim}); got {ss}")
    if rs[0] != B:
        raise ValueError(f"receivers batch ({rs[0]}) must equal the shot count ({B})")
    return mode, B, nsrc


FACE_NAMES = {2: ("top", "bottom", "left", "right"), 3: ("top", "bottom", "front", "back", "left", "right")}


def free_faces(spec, nd):
    """Free-surface faces as a tuple of 2*nd bools in shape order (z_lo, z_hi,
    [y_lo, y_hi,] x_lo, x_hi), from the reference's spellings
    (``equations/_edges.py:66-140``): ``True`` (the top face) / ``False`` /
    ``None``, a face name or names (``'top'``, ``['top', 'left']``), a
    2*nd sequence of bools, or a dict of name -> bool."""
    names = FACE_NAMES[nd]
    n = 2 * nd
    if spec is None or isinstance(spec, (bool, np.bool_)):
        return tuple([bool(spec)] + [False] * (n - 1))
    if isinstance(spec, str):
        spec = [spec]
    if isinstance(spec, dict):
        items = [(k, bool(v)) for k, v in spec.items()]
    else:
        spec = list(spec)
        if spec and all(isinstance(v, str) for v in spec):
            items = [(k, True) for k in spec]
        elif len(spec) == n:
            return tuple(bool(v) for v in spec)
        else:
            raise ValueError(f"free_surface: give face names {names} or {n} bools, got {spec!r}")
    faces = [False] * n
    for k, v in items:
        if k not in names:
            raise ValueError(f"unknown free-surface face {k!r}; the {nd}-D faces are {names}")
        faces[names.index(k)] = v
    return tuple(faces)


class _Geometry:
    """Everything a core call needs besides the model and wavelet tensors."""

    def __init__(self, prop, B, nsrc, nrec, nt, src_rt, rec_rt, device, max_vel, pml_freq):
        eq = prop.equation
        self.ndim = eq.NDIM
        self.M = eq.M
        self.B, self.nsrc, self.nrec, self.nt = B, nsrc, nrec, nt
        self.shape = prop.runtime_shape
        self.device = device
        self.dt = prop.dt
        self.spacing = prop.spacing
        pads = list(prop.pads)
        if isinstance(eq, Elastic):
            prof = cpml_profiles_s(pads, self.M, prop.dt, self.spacing, self.shape, max_vel, pml_freq)
        else:
            prof = cpml_profiles_r(pads, self.M, prop.dt, self.spacing, self.shape, max_vel, pml_freq)
        self.prof = [[torch.from_numpy(np.ascontiguousarray(a)).to(device) for a in p] for p in prof]
        # Elastic with free faces: the cells past a surface are air, which the
        # image method overwrites, so a source or receiver there is off the
        # grid (the reference would fold its adjoint back through the images)
        self.fs_faces = tuple(prop.fs_faces) if isinstance(eq, Elastic) else (False,) * (2 * self.ndim)
        if any(self.fs_faces):
            src_rt, rec_rt = np.array(src_rt, np.int64), np.array(rec_rt, np.int64)
            nz, nx = self.shape[0], self.shape[-1]
            M = self.M
            for loc in (src_rt, rec_rt):
                x, z = loc[..., 0], loc[..., -1]
                air = np.zeros(x.shape, bool)
                faces = self.fs_faces if self.ndim == 2 else (self.fs_faces[0], False, False, False)
                for on, cut in zip(faces, (z < M, z > nz - 1 - M, x < M, x > nx - 1 - M)):
                    if on:
                        air |= cut
                loc[air] = -(1 << 20)
        self.src = torch.from_numpy(np.ascontiguousarray(src_rt, dtype=np.int32)).to(device)
        self.rec = torch.from_numpy(np.ascontiguousarray(rec_rt, dtype=np.int32)).to(device)
        self.pads = list(prop.pads)          # per face in shape order: lo, hi per axis

    def acoustic_desc(self, vp, wavelet):
        d = _lib.AcousticDesc()
        d.ndim = self.ndim
        d.B = self.B
        if self.ndim == 2:
            d.nz, d.ny, d.nx = self.shape[0], 1, self.shape[1]
        else:
            d.nz, d.ny, d.nx = self.shape
        d.nt = self.nt
        d.M = self.M
        pz, px = self.pads[0:2], self.pads[-2:]
        py = self.pads[2:4] if self.ndim == 3 else [0, 0]
        for i, p in enumerate(pz + py + px):
            d.pad[i] = p
        d.dt = self.dt
        if self.ndim == 2:
            d.dz, d.dy, d.dx = self.spacing[0], 1.0, self.spacing[1]
        else:
            d.dz, d.dy, d.dx = self.spacing
        lap, grad = centred_tables(self.M)
        for k in range(self.M + 1):
            d.lap[k] = float(lap[k])
            d.grad[k] = float(grad[k])
        if self.ndim == 2:
            (az, bz, dbz), (ax, bx, dbx) = self.prof
            ay = by = dby = None
        else:
            (az, bz, dbz), (ay, by, dby), (ax, bx, dbx) = self.prof
        for name, t in (("az", az), ("bz", bz), ("dbz", dbz), ("ay", ay), ("by", by),
                        ("dby", dby), ("ax", ax), ("bx", bx), ("dbx", dbx)):
            setattr(d, name, t.data_ptr() if t is not None else None)
        cells = int(np.prod(self.shape))
        d.vp = vp.data_ptr()
        d.vp_stride = cells if vp.dim() == self.ndim + 1 else 0
        d.nsrc = self.nsrc
        d.src_loc = self.src.data_ptr()
        d.wavelet = wavelet.data_ptr()
        d.nrec = self.nrec
        d.rec_loc = self.rec.data_ptr()
        return d


    def elastic_desc(self, models, wavelet, src_fields, rec_fields):
        if self.ndim == 3 and len(models) == 4:
            return self.vti3d_desc(models, wavelet, src_fields, rec_fields)
        if self.ndim == 3:
            return self.elastic3d_desc(models, wavelet, src_fields, rec_fields)
        if len(models) == 4:
            return self.vti_desc(models, wavelet, src_fields, rec_fields)
        vp, vs, rho = models
        d = _lib.ElasticDesc()
        d.B = self.B
        d.nz, d.nx = self.shape
        d.nt = self.nt
        d.M = self.M
        for i in range(4):
            d.pad[i] = self.pads[i]
        d.dt = self.dt
        d.dz, d.dx = self.spacing
        (az, bz, azh, bzh), (ax, bx, axh, bxh) = self.prof
        for name, t in (("az", az), ("bz", bz), ("azh", azh), ("bzh", bzh),
                        ("ax", ax), ("bx", bx), ("axh", axh), ("bxh", bxh)):
            setattr(d, name, t.data_ptr())
        d.vp, d.vs, d.rho = vp.data_ptr(), vs.data_ptr(), rho.data_ptr()
        d.model_stride = int(np.prod(self.shape)) if vp.dim() == 3 else 0
        d.nsrc = self.nsrc
        d.src_loc = self.src.data_ptr()
        d.wavelet = wavelet.data_ptr()
        d.nsrc_fields = len(src_fields)
        for k, f in enumerate(src_fields):
            d.src_fields[k] = f
        d.nrec = self.nrec
        d.rec_loc = self.rec.data_ptr()
        d.nrec_fields = len(rec_fields)
        for k, f in enumerate(rec_fields):
            d.rec_fields[k] = f
        for f in range(4):
            d.free_surface[f] = 1 if self.fs_faces[f] else 0
        return d


    def vti_desc(self, models, wavelet, src_fields, rec_fields):
        vp, eps, dlt, rho = models
        d = _lib.VTIDesc()
        d.B = self.B
        d.nz, d.nx = self.shape
        d.nt = self.nt
        d.M = self.M
        for i in range(4):
            d.pad[i] = self.pads[i]
        d.dt = self.dt
        d.dz, d.dx = self.spacing
        (az, bz, azh, bzh), (ax, bx, axh, bxh) = self.prof
        for name, t in (("az", az), ("bz", bz), ("azh", azh), ("bzh", bzh),
                        ("ax", ax), ("bx", bx), ("axh", axh), ("bxh", bxh)):
            setattr(d, name, t.data_ptr())
        d.vp, d.epsilon, d.delta, d.rho = vp.data_ptr(), eps.data_ptr(), dlt.data_ptr(), rho.data_ptr()
        d.model_stride = int(np.prod(self.shape)) if vp.dim() == 3 else 0
        d.nsrc = self.nsrc
        d.src_loc = self.src.data_ptr()
        d.wavelet = wavelet.data_ptr()
        d.nsrc_fields = len(src_fields)
        for k, f in enumerate(src_fields):
            d.src_fields[k] = f
        d.nrec = self.nrec
        d.rec_loc = self.rec.data_ptr()
        d.nrec_fields = len(rec_fields)
        for k, f in enumerate(rec_fields):
            d.rec_fields[k] = f
        return d

    def vti3d_desc(self, models, wavelet, src_fields, rec_fields):
        vp, eps, dlt, rho = models
        d = _lib.VTI3DDesc()
        d.B = self.B
        d.nz, d.ny, d.nx = self.shape
        d.nt = self.nt
        d.M = self.M
        for i in range(6):
            d.pad[i] = self.pads[i]
        d.dt = self.dt
        d.dz, d.dy, d.dx = self.spacing
        names = ("az", "bz", "azh", "bzh", "ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh")
        for k, name in enumerate(names):
            setattr(d, name, self.prof[k // 4][k % 4].data_ptr())
        d.vp, d.epsilon, d.delta, d.rho = vp.data_ptr(), eps.data_ptr(), dlt.data_ptr(), rho.data_ptr()
        d.model_stride = int(np.prod(self.shape)) if vp.dim() == 4 else 0
        d.nsrc = self.nsrc
        d.src_loc = self.src.data_ptr()
        d.wavelet = wavelet.data_ptr()
        d.nsrc_fields = len(src_fields)
        for k, f in enumerate(src_fields):
            d.src_fields[k] = f
        d.nrec = self.nrec
        d.rec_loc = self.rec.data_ptr()
        d.nrec_fields = len(rec_fields)
        for k, f in enumerate(rec_fields):
            d.rec_fields[k] = f
        return d

    def elastic3d_desc(self, models, wavelet, src_fields, rec_fields):
        vp, vs, rho = models
        d = _lib.Elastic3DDesc()
        d.B = self.B
        d.nz, d.ny, d.nx = self.shape
        d.nt = self.nt
        d.M = self.M
        for i in range(6):
            d.pad[i] = self.pads[i]
        d.dt = self.dt
        d.dz, d.dy, d.dx = self.spacing
        names = ("az", "bz", "azh", "bzh", "ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh")
        for k, name in enumerate(names):
            setattr(d, name, self.prof[k // 4][k % 4].data_ptr())
        d.vp, d.vs, d.rho = vp.data_ptr(), vs.data_ptr(), rho.data_ptr()
        d.model_stride = int(np.prod(self.shape)) if vp.dim() == 4 else 0
        d.nsrc = self.nsrc
        d.src_loc = self.src.data_ptr()
        d.wavelet = wavelet.data_ptr()
        d.nsrc_fields = len(src_fields)
        for k, f in enumerate(src_fields):
            d.src_fields[k] = f
        d.nrec = self.nrec
        d.rec_loc = self.rec.data_ptr()
        d.nrec_fields = len(rec_fields)
        for k, f in enumerate(rec_fields):
            d.rec_fields[k] = f
        d.free_surface = 1 if self.fs_faces[0] else 0
        return d


def _stream_ptr(device):
    return torch.cuda.current_stream(device).cuda_stream


class _AcousticFn(torch.autograd.Function):
    """vp (runtime grid, shared ``(*shape)`` or per-shot ``(B, *shape)``) and
    wavelet ``(B, nsrc, nt)`` -> record ``(B, nt, nrec, 1)``."""

    @staticmethod
    def forward(ctx, vp, wavelet, prop, geo, mem_mode, ckpt_every):
        vp = vp.contiguous()
        wavelet = wavelet.contiguous()
        desc = geo.acoustic_desc(vp, wavelet)
        ws_b, tape_b = _lib.c_i64(), _lib.c_i64()
        _lib.call("sweep_b200_acoustic_sizes", desc, mem_mode, ckpt_every, ws_b, tape_b)
        need_bwd = any(ctx.needs_input_grad[:2])
        ws = prop._workspace(ws_b.value, vp.device)
        if not need_bwd:
            tape = None
        elif mem_mode & _lib.MEM_HOST_TAPE:
            tape = torch.empty(tape_b.value, dtype=torch.uint8, pin_memory=True)
        else:
            tape = torch.empty(tape_b.value, dtype=torch.uint8, device=vp.device)
        record = torch.empty((geo.B, geo.nt, geo.nrec), dtype=torch.float32, device=vp.device)
        _lib.call("sweep_b200_acoustic_forward", desc, mem_mode, ckpt_every, record.data_ptr(),
                  tape.data_ptr() if tape is not None else None, ws.data_ptr(), ws.numel(),
                  _stream_ptr(vp.device))
        ctx.save_for_backward(vp, wavelet)
        ctx.tape = tape
        ctx.geo, ctx.prop, ctx.mem_mode, ctx.ckpt_every = geo, prop, mem_mode, ckpt_every
        return record[..., None]

    @staticmethod
    def backward(ctx, grad_record):
        if ctx.tape is None:
            raise RuntimeError("sweep_b200: this forward has already been back-propagated (or ran "
                               "without gradients); a second backward is refused")
        vp, wavelet = ctx.saved_tensors
        geo, prop = ctx.geo, ctx.prop
        adj = grad_record[..., 0].to(torch.float32).contiguous()
        desc = geo.acoustic_desc(vp, wavelet)
        ws_b, tape_b = _lib.c_i64(), _lib.c_i64()
        _lib.call("sweep_b200_acoustic_sizes", desc, ctx.mem_mode, ctx.ckpt_every, ws_b, tape_b)
        ws = prop._workspace(ws_b.value, vp.device)
        grad_vp = torch.empty_like(vp)
        grad_w = torch.empty_like(wavelet) if ctx.needs_input_grad[1] else None
        illum = prop.compute_illumination
        i_s = torch.empty_like(vp) if illum else None
        i_r = torch.empty_like(vp) if illum else None
        _lib.call("sweep_b200_acoustic_backward", desc, ctx.mem_mode, ctx.ckpt_every, adj.data_ptr(),
                  ctx.tape.data_ptr(), grad_vp.data_ptr(),
                  grad_w.data_ptr() if grad_w is not None else None,
                  i_s.data_ptr() if illum else None, i_r.data_ptr() if illum else None,
                  ws.data_ptr(), ws.numel(), _stream_ptr(vp.device))
        ctx.tape = None
        if illum:
            prop._set_illumination(i_s, i_r)
        return grad_vp, grad_w, None, None, None, None


class _ElasticFn(torch.autograd.Function):
    """vp, vs, rho (runtime grid, shared or per shot, all alike) and the
    wavelet ``(B, nsrc, nt)`` -> record ``(B, nt, nrec, nfield)``.  The
    backward returns the three model gradients; the wavelet gradient is not
    produced (refused up front, as the reference's impl='c' does)."""

    @staticmethod
    def forward(ctx, vp, vs, rho, wavelet, prop, geo, fields, mem_mode, ckpt_every):
        models = [m.contiguous() for m in (vp, vs, rho)]
        wavelet = wavelet.contiguous()
        sf, rf = fields
        desc = geo.elastic_desc(models, wavelet, sf, rf)
        pre = "sweep_b200_elastic3d" if geo.ndim == 3 else "sweep_b200_elastic"
        ws_b, tape_b = _lib.c_i64(), _lib.c_i64()
        _lib.call(pre + "_sizes", desc, mem_mode, ckpt_every, ws_b, tape_b)
        need_bwd = any(ctx.needs_input_grad[:3])
        dev = vp.device
        ws = prop._workspace(ws_b.value, dev)
        if not need_bwd:
            tape = None
        elif mem_mode & _lib.MEM_HOST_TAPE:
            tape = torch.empty(tape_b.value, dtype=torch.uint8, pin_memory=True)
        else:
            tape = torch.empty(tape_b.value, dtype=torch.uint8, device=dev)
        record = torch.empty((geo.B, geo.nt, geo.nrec, len(rf)), dtype=torch.float32, device=dev)
        _lib.call(pre + "_forward", desc, mem_mode, ckpt_every, record.data_ptr(),
                  tape.data_ptr() if tape is not None else None, ws.data_ptr(), ws.numel(),
                  _stream_ptr(dev))
        ctx.save_for_backward(*models, wavelet)
        ctx.tape = tape
        ctx.geo, ctx.prop, ctx.fields = geo, prop, fields
        ctx.mem_mode, ctx.ckpt_every = mem_mode, ckpt_every
        return record

    @staticmethod
    def backward(ctx, grad_record):
        if ctx.tape is None:
            raise RuntimeError("sweep_b200: this forward has already been back-propagated (or ran "
                               "without gradients); a second backward is refused")
        vp, vs, rho, wavelet = ctx.saved_tensors
        geo, prop = ctx.geo, ctx.prop
        adj = grad_record.to(torch.float32).contiguous()
        desc = geo.elastic_desc([vp, vs, rho], wavelet, *ctx.fields)
        pre = "sweep_b200_elastic3d" if geo.ndim == 3 else "sweep_b200_elastic"
        ws_b, tape_b = _lib.c_i64(), _lib.c_i64()
        _lib.call(pre + "_sizes", desc, ctx.mem_mode, ctx.ckpt_every, ws_b, tape_b)
        ws = prop._workspace(ws_b.value, vp.device)
        g = [torch.empty_like(vp) for _ in range(3)]
        _lib.call(pre + "_backward", desc, ctx.mem_mode, ctx.ckpt_every, adj.data_ptr(),
                  ctx.tape.data_ptr(), g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr(),
                  ws.data_ptr(), ws.numel(), _stream_ptr(vp.device))
        ctx.tape = None
        return g[0], g[1], g[2], None, None, None, None, None, None


class _VTIFn(torch.autograd.Function):
    """vp, epsilon, delta, rho (runtime grid, shared or per shot, all alike)
    and the wavelet ``(B, nsrc, nt)`` -> record ``(B, nt, nrec, nfield)``; the
    backward returns the four model gradients (no wavelet gradient, as for
    Elastic)."""

    @staticmethod
    def forward(ctx, vp, eps, dlt, rho, wavelet, prop, geo, fields, mem_mode, ckpt_every):
        models = [m.contiguous() for m in (vp, eps, dlt, rho)]
        wavelet = wavelet.contiguous()
        sf, rf = fields
        desc = geo.elastic_desc(models, wavelet, sf, rf)
        pre = "sweep_b200_vti3d" if geo.ndim == 3 else "sweep_b200_vti"
        ws_b, tape_b = _lib.c_i64(), _lib.c_i64()
        _lib.call(pre + "_sizes", desc, mem_mode, ckpt_every, ws_b, tape_b)
        dev = vp.device
        ws = prop._workspace(ws_b.value, dev)
        tape = torch.empty(tape_b.value, dtype=torch.uint8, device=dev) if any(ctx.needs_input_grad[:4]) else None
        record = torch.empty((geo.B, geo.nt, geo.nrec, len(rf)), dtype=torch.float32, device=dev)
        _lib.call(pre + "_forward", desc, mem_mode, ckpt_every, record.data_ptr(),
                  tape.data_ptr() if tape is not None else None, ws.data_ptr(), ws.numel(), _stream_ptr(dev))
        ctx.save_for_backward(*models, wavelet)
        ctx.tape = tape
        ctx.geo, ctx.prop, ctx.fields = geo, prop, fields
        ctx.mem_mode, ctx.ckpt_every = mem_mode, ckpt_every
        return record

    @staticmethod
    def backward(ctx, grad_record):
        if ctx.tape is None:
            raise RuntimeError("sweep_b200: this forward has already been back-propagated (or ran "
                               "without gradients); a second backward is refused")
        vp, eps, dlt, rho, wavelet = ctx.saved_tensors
        geo, prop = ctx.geo, ctx.prop
        adj = grad_record.to(torch.float32).contiguous()
        desc = geo.elastic_desc([vp, eps, dlt, rho], wavelet, *ctx.fields)
        pre = "sweep_b200_vti3d" if geo.ndim == 3 else "sweep_b200_vti"
        ws_b, tape_b = _lib.c_i64(), _lib.c_i64()
        _lib.call(pre + "_sizes", desc, ctx.mem_mode, ctx.ckpt_every, ws_b, tape_b)
        ws = prop._workspace(ws_b.value, vp.device)
        g = [torch.empty_like(vp) for _ in range(4)]
        _lib.call(pre + "_backward", desc, ctx.mem_mode, ctx.ckpt_every, adj.data_ptr(),
                  ctx.tape.data_ptr(), *[x.data_ptr() for x in g], ws.data_ptr(), ws.numel(),
                  _stream_ptr(vp.device))
        ctx.tape = None
        return g[0], g[1], g[2], g[3], None, None, None, None, None, None


class PropTorch(torch.nn.Module):
    """Propagator over the B200 core (``impl='c'``; the only implementation).

    Args mirror the reference's ``PropBase`` (``propagator/base.py:31-120``):
    ``equation``, ``shape`` (physical ``(nz, nx)`` / ``(nz, ny, nx)``), ``dh``
    (scalar or per axis in shape order), ``dt``, ``abcn`` (PML cells per face,
    default 50), ``memory`` (``BoundarySaving()`` default, ``Full()``,
    ``Ckpt(chunks)``), ``device``/``dev``, ``source_type`` /
    ``receiver_type`` (field names; elastic only).

    Launch schedule (no counterpart in the reference, whose launch shapes are
    fixed): ``autotune=True`` times candidate schedules on the first call of
    each problem shape (``sweep_b200.autotune.tune``) and records the fastest
    for every later call of that shape; ``schedule={...}`` records the given
    fields instead (``shots_fwd``, ``shots_rev``, ``z_chunks``,
    ``graph_steps``).  ``tune_report`` holds the tuner's last report."""

    def __init__(self, equation, shape, dh=10.0, dt=0.002, abcn=50, impl="c", memory=None,
                 device=None, dev=None, source_type=None, receiver_type=None,
                 use_ckpt=None, ckpt_chunks=100, free_surface=False, autotune=False, schedule=None,
                 **kwargs):
        super().__init__()
        if impl not in (None, "c", "auto"):
            raise NotImplementedError(f"sweep_b200 implements impl='c' only (got impl={impl!r})")
        unknown = set(kwargs) - {"nt", "B", "pml_type", "backend"}
        if unknown:
            raise TypeError(f"PropTorch got unexpected keyword arguments {sorted(unknown)}")
        self.equation = equation
        self.impl = "c"
        nd = equation.NDIM
        if isinstance(equation, Elastic3D):
            if equation.M > 4:
                raise NotImplementedError(f"sweep_b200: Elastic3D is built at spatial orders 2, 4, 6 and 8 "
                                          f"(got {equation.spatial_order})")
        elif equation.M > 7:
            raise NotImplementedError(f"sweep_b200: spatial orders 2 to 14 are built (got {equation.spatial_order})")
        if len(shape) != nd:
            raise ValueError(f"{type(equation).__name__} needs a {nd}-D shape, got {shape}")
        self.shape = tuple(int(s) for s in shape)
        self.spacing = [float(x) for x in (dh if np.ndim(dh) else [dh] * nd)]
        self.dt = float(dt)
        self.abcn = int(abcn)
        if self.abcn < 1:
            raise NotImplementedError("sweep_b200: the absorbing faces need a layer (abcn >= 1)")
        self.fs_faces = free_faces(free_surface, nd)
        if isinstance(equation, AcousticVTI1st) and any(self.fs_faces):
            raise NotImplementedError(f"{type(equation).__name__} has no free surface (the reference refuses it too: the VTI "
                                      "traction-free condition needs an anisotropic image method)")
        if nd == 3 and any(self.fs_faces[1:]):
            raise NotImplementedError("per-face free surfaces are 2-D only (as in the reference); "
                                      "3-D takes free_surface=True (the top face)")
        self.free_surface = any(self.fs_faces)
        # PML cells per face in shape order (lo, hi per axis); a free surface
        # takes its face's pad away and leaves the M halo cells beyond it at
        # zero pressure (reference ``PropTorch(free_surface=...)``: pad 0 on
        # the free faces, ``propagator/base.py:181-240``)
        self.pads = [0 if f else self.abcn for f in self.fs_faces]
        M = equation.M
        self.runtime_shape = tuple(n + self.pads[2 * a] + self.pads[2 * a + 1] + 2 * M
                                   for a, n in enumerate(self.shape))
        if memory is None:
            memory = Ckpt(chunks=ckpt_chunks) if use_ckpt else BoundarySaving()
        if not isinstance(memory, (BoundarySaving, Full, Ckpt)):
            raise TypeError("memory must be BoundarySaving(), Full() or Ckpt(chunks)")
        self.memory = memory
        self.device = torch.device(device or dev or equation.device or "cuda")
        self.source_type = list(source_type or equation.default_source_fields)
        self.receiver_type = list(receiver_type or equation.default_receiver_fields)
        self.compute_illumination = False
        self.source_illumination = None
        self.receiver_illumination = None
        self._ws = None
        self.last_memory = None
        self.autotune = bool(autotune)
        self.schedule = dict(schedule) if schedule is not None else None
        self.tune_report = None

    # ---------------------------------------------------------------- helpers
    def _workspace(self, nbytes, device):
        """The core's scratch (reused between calls).  With the environment
        variable SWEEP_B200_POISON_WORKSPACE=1 it is filled with 0xFF bytes
        (float NaN) before every call, so a read of scratch that the call
        never wrote shows up in its results."""
        if self._ws is None or self._ws.numel() < nbytes or self._ws.device != device:
            self._ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device)
        if os.environ.get("SWEEP_B200_POISON_WORKSPACE") == "1":
            self._ws.fill_(255)
        return self._ws

    def _set_illumination(self, i_s, i_r):
        crop = self._crop
        if i_s.dim() == self.equation.NDIM + 1 and i_s.shape[0] == 1:
            i_s, i_r = i_s[0], i_r[0]
        self.source_illumination = crop(i_s)
        self.receiver_illumination = crop(i_r)

    def _crop(self, g):
        M = self.equation.M
        sl = tuple(slice(self.pads[2 * a] + M, self.pads[2 * a] + M + n) for a, n in enumerate(self.shape))
        return g[(Ellipsis,) + sl]

    def _pad_model(self, m):
        """Replicate-pad a physical model to the runtime grid (autograd crops back)."""
        M = self.equation.M
        nd = self.equation.NDIM
        per_shot = m.dim() == nd + 1
        x = m if per_shot else m[None]
        widths = []
        for a in reversed(range(nd)):            # F.pad runs from the last axis
            widths += [self.pads[2 * a] + M, self.pads[2 * a + 1] + M]
        x = F.pad(x[:, None], widths, mode="replicate")[:, 0]
        return x if per_shot else x[0]

    def _shift(self):
        """Runtime-grid offset of a coordinate, in the coordinate order (x[, y], z)."""
        nd, M = self.equation.NDIM, self.equation.M
        return np.array([self.pads[2 * (nd - 1 - c)] + M for c in range(nd)], np.int64)

    def _elastic_fields(self):
        """Source / receiver field indices (reference ``_c.py:1163-1176``)."""
        names = list(self.equation.FIELDS)
        for role, kinds in (("source_type", self.source_type), ("receiver_type", self.receiver_type)):
            missing = [k for k in kinds if k not in names]
            if not kinds or missing:
                raise ValueError(f"Invalid {role} entries {missing or kinds}; available wavefields are {names}")
        sf = [names.index(k) for k in self.source_type]
        if len(set(sf)) != len(sf) or len(self.receiver_type) > len(names):
            raise ValueError("source_type / receiver_type must not repeat a field")
        return sf, [names.index(k) for k in self.receiver_type]

    def _mem_mode(self):
        if isinstance(self.memory, Ckpt):
            if self.memory.mode == "recursive":
                return _lib.MEM_RECURSIVE, int(self.memory.count)
            return _lib.MEM_CHECKPOINT, int(self.memory.chunks)
        sd = getattr(self.memory, "storage_dtype", "fp32")
        mode = {"fp32": _lib.MEM_BOUNDARY, "fp16": _lib.MEM_BOUNDARY_FP16, "bf16": _lib.MEM_BOUNDARY_BF16,
                "int8": _lib.MEM_BOUNDARY_INT8}[sd]
        if getattr(self.memory, "storage", "gpu") == "cpu":
            mode |= _lib.MEM_HOST_TAPE
        return mode, 0

    def _desc(self, geo, padded, wb, fields):
        wb = wb.contiguous()
        if fields is not None:
            return geo.elastic_desc([m.contiguous() for m in padded], wb, *fields)
        return geo.acoustic_desc(padded[0].contiguous(), wb)

    def _tape_bytes(self, desc, fields, mem_mode, ckpt_every):
        ws_b, tape_b = _lib.c_i64(), _lib.c_i64()
        name = "sweep_b200_acoustic_sizes"
        if fields is not None:
            name = ("sweep_b200_elastic3d_sizes" if isinstance(desc, _lib.Elastic3DDesc) else
                    "sweep_b200_vti_sizes" if isinstance(desc, _lib.VTIDesc) else
                    "sweep_b200_vti3d_sizes" if isinstance(desc, _lib.VTI3DDesc) else "sweep_b200_elastic_sizes")
        _lib.call(name, desc, mem_mode, ckpt_every, ws_b, tape_b)
        return int(tape_b.value)

    def _apply_budget(self, geo, padded, wb, fields, mem_mode, ckpt_every):
        """Memory mode of this call: boundary saving while its tape fits
        ``BoundarySaving.budget_gb``, else checkpoints every ``ckpt_chunks``
        steps; recorded in ``last_memory``."""
        mem = self.memory
        budget = getattr(mem, "budget_gb", None)
        if budget is None:
            self.last_memory = {"mode": {_lib.MEM_CHECKPOINT: "checkpoint",
                                         _lib.MEM_RECURSIVE: "recursive"}.get(mem_mode, "boundary"),
                                "chunks": ckpt_every or None}
            return mem_mode, ckpt_every
        desc = self._desc(geo, padded, wb, fields)
        tape = self._tape_bytes(desc, fields, mem_mode, ckpt_every)
        if tape <= float(budget) * 1e9:
            self.last_memory = {"mode": "boundary", "tape_bytes": tape, "budget_bytes": float(budget) * 1e9}
            return mem_mode, ckpt_every
        k = int(mem.ckpt_chunks)
        ck_tape = self._tape_bytes(desc, fields, _lib.MEM_CHECKPOINT, k)
        self.last_memory = {"mode": "checkpoint", "chunks": k, "tape_bytes": ck_tape,
                            "boundary_tape_bytes": tape, "budget_bytes": float(budget) * 1e9}
        return _lib.MEM_CHECKPOINT, k

    def _apply_schedule(self, geo, padded, wb, fields, mem_mode, ckpt_every):
        from . import autotune
        desc = self._desc(geo, padded, wb, fields)
        if self.schedule is not None:
            autotune.set_schedule(desc, self.schedule)
        elif not autotune.tuned(desc):
            self.tune_report = autotune.tune(self, geo, padded, wb, fields, mem_mode, ckpt_every)

    def launch_schedule(self, wavelet_len, sources, receivers, models):
        """The schedule (resolved fields) a call with these inputs would run."""
        from . import autotune
        geo, padded, wb, fields = self._probe(wavelet_len, sources, receivers, models)
        desc = self._desc(geo, padded, wb, fields)
        if isinstance(desc, _lib.Elastic3DDesc):
            return {"fixed": "one thread per cell, 32 x 4 x 2 cell blocks, two z planes of a shot per grid row"}
        if isinstance(desc, _lib.VTIDesc):
            return {"fixed": "one thread per cell, 32 x 8 cell tiles per shot"}
        if isinstance(desc, _lib.VTI3DDesc):
            return {"fixed": "one thread per cell, 32 x 4 x 2 cell blocks, two z planes of a shot per grid row"}
        if desc.M != 4:
            return {"fixed": f"order {2 * desc.M}: one thread per cell, 32 x 8 cell tiles per plane and shot"}
        return autotune.get_schedule(desc)

    def tape_bytes(self, wavelet_len, sources, receivers, models):
        """Bytes of the tape a gradient call with these inputs keeps between
        its forward and backward, under this solver's memory option as given
        (before any ``budget_gb`` switch)."""
        geo, padded, wb, fields = self._probe(wavelet_len, sources, receivers, models)
        mem_mode, ckpt_every = self._mem_mode()
        return self._tape_bytes(self._desc(geo, padded, wb, fields), fields, mem_mode, ckpt_every)

    def _probe(self, wavelet_len, sources, receivers, models):
        nd = self.equation.NDIM
        src = np.asarray(sources.detach().cpu() if isinstance(sources, torch.Tensor) else sources, np.int64)
        rec = np.asarray(receivers.detach().cpu() if isinstance(receivers, torch.Tensor) else receivers, np.int64)
        B = src.shape[0]
        src = src.reshape(B, -1, nd) + self._shift()
        rec = rec.reshape(B, -1, nd) + self._shift()
        geo = _Geometry(self, B, src.shape[1], rec.shape[1], int(wavelet_len), src, rec, self.device, 4500.0, 25.0)
        padded = [self._pad_model(m.to(self.device)) for m in models]
        wb = torch.zeros((B, src.shape[1], int(wavelet_len)), dtype=torch.float32, device=self.device)
        fields = self._elastic_fields() if isinstance(self.equation, Elastic) else None
        return geo, padded, wb, fields

    # ---------------------------------------------------------------- forward
    def forward(self, wavelet, sources, receivers, models=None, max_vel=4500.0, pml_freq=25.0):
        geo, padded, wb, fields, mem_mode, ckpt_every, wavelet = self._prepare(
            wavelet, sources, receivers, models, max_vel, pml_freq)
        eq = self.equation
        if isinstance(eq, (Acoustic, Acoustic3D)):
            return _AcousticFn.apply(padded[0], wb, self, geo, mem_mode, ckpt_every)
        if isinstance(eq, AcousticVTI1st):
            if wavelet.requires_grad and torch.is_grad_enabled():
                raise NotImplementedError(
                    f"impl='c' {type(eq).__name__} does not return the wavelet gradient (its compiled backward "
                    "returns the model gradients only). Detach the wavelet.")
            return _VTIFn.apply(*padded, wb, self, geo, fields, mem_mode, ckpt_every)
        if isinstance(eq, Elastic):
            if wavelet.requires_grad and torch.is_grad_enabled():
                raise NotImplementedError(
                    "impl='c' Elastic does not return the wavelet gradient (its compiled backward "
                    "returns the model gradients only). Detach the wavelet.")
            return _ElasticFn.apply(*padded, wb, self, geo, fields, mem_mode, ckpt_every)
        raise NotImplementedError(f"{type(eq).__name__} is not built")

    def _prepare(self, wavelet, sources, receivers, models, max_vel, pml_freq):
        """Checked inputs of a call: the geometry, the padded models, the
        per-shot wavelet view, the elastic fields, and the memory mode."""
        eq = self.equation
        nd = eq.NDIM
        dev = self.device
        if dev.type != "cuda":
            raise RuntimeError("sweep_b200 runs on a CUDA device only (no CPU path)")
        if models is None or len(models) != len(eq.MODEL_NAMES):
            raise ValueError(f"{type(eq).__name__} needs models={list(eq.MODEL_NAMES)}")
        for name, m in zip(eq.MODEL_NAMES, models):
            if not isinstance(m, torch.Tensor) or m.dtype != torch.float32:
                raise TypeError(f"model {name!r} must be a float32 torch.Tensor")
            if tuple(m.shape[-nd:]) != self.shape:
                raise ValueError(f"model {name!r} has shape {tuple(m.shape)}, expected {self.shape}")
        wavelet = _as_tensor(wavelet, torch.float32, dev) if not (
            isinstance(wavelet, torch.Tensor) and wavelet.device == dev and wavelet.dtype == torch.float32) else wavelet
        mode, B, nsrc = normalize_io(wavelet, sources, receivers, nd)
        nt = wavelet.shape[-1]
        src = np.asarray(sources.detach().cpu() if isinstance(sources, torch.Tensor) else sources, np.int64)
        rec = np.asarray(receivers.detach().cpu() if isinstance(receivers, torch.Tensor) else receivers, np.int64)
        src = src.reshape(B, nsrc, nd) + self._shift()
        rec = rec.reshape(B, -1, nd) + self._shift()
        nrec = rec.shape[1]
        if mode == "A1":
            wb = wavelet[None, None, :].expand(B, 1, nt)
        elif mode == "A2":
            wb = wavelet[:, None, :]
        else:
            wb = wavelet[None, None, :].expand(1, nsrc, nt) if wavelet.dim() == 1 else wavelet[None]
        for m in models:
            if m.dim() == nd + 1 and m.shape[0] != B:
                raise ValueError(f"per-shot model batch ({m.shape[0]}) must equal the shot count ({B})")
            if m.dim() == nd + 1 and isinstance(eq, Acoustic3D):
                raise NotImplementedError("Acoustic3D takes one shared model (no per-shot models)")
        geo = _Geometry(self, B, nsrc, nrec, nt, src, rec, dev, max_vel, pml_freq)
        mem_mode, ckpt_every = self._mem_mode()
        padded = [self._pad_model(m.to(dev)) for m in models]
        fields = self._elastic_fields() if isinstance(eq, Elastic) else None
        if (self.autotune or self.schedule is not None) and (isinstance(eq, (Elastic3D, AcousticVTI1st)) or eq.M != 4):
            raise NotImplementedError(f"sweep_b200: {type(eq).__name__} at spatial_order={eq.spatial_order} has one "
                                      f"built-in launch schedule (no autotune)")
        if self.autotune or self.schedule is not None:
            self._apply_schedule(geo, padded, wb, fields, mem_mode, ckpt_every)
        mem_mode, ckpt_every = self._apply_budget(geo, padded, wb, fields, mem_mode, ckpt_every)
        if isinstance(eq, Elastic) and len({m.dim() for m in models}) != 1:
            raise ValueError("vp, vs and rho must all be shared or all per shot")
        return geo, padded, wb, fields, mem_mode, ckpt_every, wavelet

    # ------------------------------------------------------- stepped runners
    def forward_runner(self, wavelet, sources, receivers, models=None, max_vel=4500.0, pml_freq=25.0):
        """A persistent forward over these inputs, advanced segment by segment
        (reference ``sweep.backend.c.runners.ForwardRunner``): see
        :class:`sweep_b200.runners.ForwardRunner`."""
        from .runners import ForwardRunner
        return ForwardRunner(self, wavelet, sources, receivers, models, max_vel, pml_freq)
