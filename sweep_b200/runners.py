"""Stepped runners: a forward or backward pass advanced segment by segment over
the time axis (reference ``src/sweep/backend/c/runners.py`` over
``sweep_forward_runner_*`` / ``sweep_backward_runner_*``,
``src/sweep/csrc/core/capi.h:236-243``).

``runner = solver.forward_runner(wavelet, sources, receivers, models=[...])``
sets a problem up once; ``runner.run(it_begin, it_end)`` advances steps
``[it_begin, it_end)``, segments in order from 0 to nt, and ``runner.record``
holds every step run so far.  Once the forward has reached nt,
``runner.backward_runner(grad_record)`` reverses it: ``run(bw_it_begin,
bw_it_end)`` takes the steps ``[bw_it_end, bw_it_begin)``, segments in order
from nt down to 0, and ``gradients()`` gives the model gradients (and the
wavelet gradient for acoustic) of every step reversed so far.  The segments
compute what one ``solver(...)`` call and ``backward()`` compute, bit for bit.
Boundary saving only (every strip format, device or host tape); ``step_phase``
must be 0 (the reference's 1 / 2 split a step around a domain-decomposition
halo exchange, which is not built here).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .equations import AcousticVTI1st, Elastic3D


def _check_memory(mem_mode):
    base = mem_mode & ~_lib.MEM_HOST_TAPE
    if base in (_lib.MEM_CHECKPOINT, _lib.MEM_RECURSIVE):
        raise ValueError("stepped runners take boundary saving only (the reference's runners refuse "
                         "checkpointing too)")


class _Handle:
    """One runner handle of the core; destroyed once (close() or collection)."""

    def __init__(self, create, *args):
        lib = _lib.load()
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(_lib.ERR_CAP)
        _lib.check(getattr(lib, create)(*args, ctypes.byref(h), err, _lib.ERR_CAP), err)
        self.h = h

    def run(self, entry, a, b, phase, device):
        if self.h is None:
            raise RuntimeError("sweep_b200: this runner is closed")
        lib = _lib.load()
        err = ctypes.create_string_buffer(_lib.ERR_CAP)
        stream = torch.cuda.current_stream(device).cuda_stream
        _lib.check(getattr(lib, entry)(self.h, int(a), int(b), int(phase), stream, err, _lib.ERR_CAP), err)

    def close(self):
        h, self.h = self.h, None
        if h is not None and h.value:
            _lib.load().sweep_b200_runner_destroy(h)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ForwardRunner:
    """A forward pass of ``prop`` over fixed inputs, run in segments."""

    def __init__(self, prop, wavelet, sources, receivers, models, max_vel=4500.0, pml_freq=25.0):
        if isinstance(prop.equation, (Elastic3D, AcousticVTI1st)):
            raise NotImplementedError(f"sweep_b200: stepped runners are built for Acoustic, Acoustic3D and "
                                      f"Elastic; {type(prop.equation).__name__} runs whole passes only")
        models = [m.detach() for m in models]
        geo, padded, wb, fields, mem_mode, ckpt_every, _ = prop._prepare(
            wavelet.detach() if isinstance(wavelet, torch.Tensor) else wavelet, sources, receivers, models,
            max_vel, pml_freq)
        _check_memory(mem_mode)
        self.prop, self.geo, self.fields, self.mem_mode = prop, geo, fields, mem_mode
        self.models = models
        self.padded = [p.contiguous() for p in padded]
        self.wb = wb.contiguous()
        self.device = self.padded[0].device
        self.elastic = fields is not None
        if self.elastic:
            self.desc = geo.elastic_desc(self.padded, self.wb, *fields)
            sizes, create = "sweep_b200_elastic_sizes", "sweep_b200_elastic_forward_runner_create"
            shape = (geo.B, geo.nt, geo.nrec, len(fields[1]))
        else:
            self.desc = geo.acoustic_desc(self.padded[0], self.wb)
            sizes, create = "sweep_b200_acoustic_sizes", "sweep_b200_acoustic_forward_runner_create"
            shape = (geo.B, geo.nt, geo.nrec)
        ws_b, tape_b = _lib.c_i64(), _lib.c_i64()
        _lib.call(sizes, self.desc, mem_mode, 0, ws_b, tape_b)
        self.ws_bytes = ws_b.value
        self.ws = torch.empty(max(self.ws_bytes, 1), dtype=torch.uint8, device=self.device)
        if mem_mode & _lib.MEM_HOST_TAPE:
            self.tape = torch.empty(tape_b.value, dtype=torch.uint8, pin_memory=True)
        else:
            self.tape = torch.empty(tape_b.value, dtype=torch.uint8, device=self.device)
        self._record = torch.empty(shape, dtype=torch.float32, device=self.device)
        self.nt = geo.nt
        self._h = _Handle(create, self.desc, mem_mode, self._record.data_ptr(), self.tape.data_ptr(),
                          self.ws.data_ptr(), self.ws.numel())
        self.next = 0

    def run(self, it_begin: int, it_end: int, step_phase: int = 0) -> None:
        """Steps ``[it_begin, it_end)``; ``it_begin`` must be where the last
        segment ended."""
        self._h.run("sweep_b200_forward_runner_run", it_begin, it_end, step_phase, self.device)
        self.next = it_end

    @property
    def record(self) -> torch.Tensor:
        """``(B, nt, nrec, nfield)``: the steps run so far (the rest is zero)."""
        return self._record if self.elastic else self._record[..., None]

    def backward_runner(self, grad_record) -> "BackwardRunner":
        if self.next != self.nt:
            raise RuntimeError(f"sweep_b200: the forward runner stands at step {self.next}, not nt = {self.nt}; "
                               "run it to the end first")
        return BackwardRunner(self, grad_record)

    def device_index(self) -> int:
        return _lib.load().sweep_b200_runner_device_index(self._h.h) if self._h.h is not None else -1

    def close(self) -> None:
        self._h.close()


class BackwardRunner:
    """The reverse of a completed :class:`ForwardRunner`, run in segments."""

    def __init__(self, fwd: ForwardRunner, grad_record):
        self.fwd = fwd
        g = grad_record.detach().to(fwd.device, torch.float32)
        self.adj = (g if fwd.elastic else g[..., 0]).contiguous()
        self.grads = [torch.empty_like(p) for p in fwd.padded]
        self.grad_w = None
        self.illum = None
        if fwd.elastic:
            args = [self.grads[0].data_ptr(), self.grads[1].data_ptr(), self.grads[2].data_ptr()]
            create = "sweep_b200_elastic_backward_runner_create"
        else:
            self.grad_w = torch.empty_like(fwd.wb)
            if fwd.prop.compute_illumination:
                self.illum = (torch.empty_like(fwd.padded[0]), torch.empty_like(fwd.padded[0]))
            args = [self.grads[0].data_ptr(), self.grad_w.data_ptr(),
                    self.illum[0].data_ptr() if self.illum else None,
                    self.illum[1].data_ptr() if self.illum else None]
            create = "sweep_b200_acoustic_backward_runner_create"
        self._h = _Handle(create, fwd.desc, fwd.mem_mode, self.adj.data_ptr(), fwd.tape.data_ptr(), *args,
                          fwd.ws.data_ptr(), fwd.ws.numel())
        self.next = fwd.nt

    def run(self, bw_it_begin: int, bw_it_end: int, step_phase: int = 0) -> None:
        """Reverse steps ``[bw_it_end, bw_it_begin)``; ``bw_it_begin`` must be
        where the last segment stopped (nt for the first)."""
        self._h.run("sweep_b200_backward_runner_run", bw_it_begin, bw_it_end, step_phase, self.fwd.device)
        self.next = bw_it_end

    def gradients(self):
        """Gradients of the loss w.r.t. the models as given (the pad folded
        back, as autograd does through the padding), and for acoustic the
        wavelet gradient ``(B, nsrc, nt)``, of every step reversed so far."""
        xs = [m.detach().requires_grad_(True) for m in self.fwd.models]
        with torch.enable_grad():
            pads = [self.fwd.prop._pad_model(x) for x in xs]
            gs = torch.autograd.grad(pads, xs, grad_outputs=self.grads)
        out = list(gs)
        if not self.fwd.elastic:
            out.append(self.grad_w)
        return out

    def illumination(self):
        """(source, receiver) illumination on the model grid, when the solver
        had ``compute_illumination`` set at the runner's creation."""
        if self.illum is None:
            return None
        crop = self.fwd.prop._crop
        i_s, i_r = self.illum
        return crop(i_s), crop(i_r)

    def close(self) -> None:
        self._h.close()
