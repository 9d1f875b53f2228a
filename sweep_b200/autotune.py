"""Per-shape launch-schedule autotuner and the schedule table's Python side.

No counterpart in the reference: its launch shapes are fixed per kernel
(reference ``src/sweep/csrc/cuda/launch/config.h:65-70``) and its time loop
issues every launch from the host (``eq_driver.cuh:357-453``).

A *schedule* (``sweep_b200_schedule`` in ``include/sweep_b200.h``) holds the
launch choices the core leaves open for one problem shape:

* ``shots_fwd`` -- shots per CTA of the forward step kernels (2-D acoustic,
  elastic);
* ``shots_rev`` -- shots per CTA of the reverse kernels that sum the image
  (2-D acoustic, elastic);
* ``z_chunks`` -- z chunks each column block of the 3-D stencil kernels is cut
  into (the grid depth per shot, 3-D acoustic);
* ``graph_steps`` -- time steps per captured CUDA graph in the step loops
  (0: plain stream launches);
* ``tile_y`` -- 3-D acoustic: rows of the 32-column block each CTA of the
  stencil kernels covers, 8 (256 threads, 4 CTAs per SM) or 16 (512 threads,
  2 CTAs per SM, less halo per cell).

The 2-D and elastic tile shapes are compile-time constants of the kernels
(they fix the shared-memory staging and register blocking), and there is no
temporal blocking to choose: every step is one pass over HBM.

:func:`tune` times the real forward and backward calls of one shape over a
truncated time axis, one knob at a time from the built-in defaults
(coordinate descent), records the fastest schedule in the core's table and
returns a report.  Every later call of that shape -- any nt, sources and
receivers -- runs the recorded schedule.  ``PropTorch(autotune=True)`` runs it
once per shape and process, on the first call.
"""
from __future__ import annotations

import copy
import time

import torch

from . import _lib

FIELDS = ("shots_fwd", "shots_rev", "z_chunks", "graph_steps", "tile_y")
BUILTIN = {"shots_fwd": 0, "shots_rev": 0, "z_chunks": 0, "graph_steps": -1, "tile_y": 0}

_tuned: dict = {}


def _family(desc) -> int:
    return _lib.FAMILY_ELASTIC if isinstance(desc, _lib.ElasticDesc) else _lib.FAMILY_ACOUSTIC


def shape_key(desc) -> tuple:
    """The fields the core keys a schedule on (nt, sources and receivers are not)."""
    if isinstance(desc, _lib.ElasticDesc):
        return ("elastic", 2, desc.B, desc.nz, 1, desc.nx, tuple(desc.pad), desc.model_stride != 0)
    return ("acoustic", desc.ndim, desc.B, desc.nz, desc.ny, desc.nx, tuple(desc.pad), desc.vp_stride != 0)


def get_schedule(desc) -> dict:
    """The schedule a call with ``desc`` runs, every field resolved."""
    lib = _lib.load()
    out = _lib.Schedule()
    err = _lib.ctypes.create_string_buffer(_lib.ERR_CAP)
    _lib.check(lib.sweep_b200_schedule_get(_family(desc), _lib.ctypes.byref(desc), _lib.ctypes.byref(out),
                                           err, _lib.ERR_CAP), err)
    return {f: int(getattr(out, f)) for f in FIELDS}


def set_schedule(desc, schedule: dict) -> None:
    """Record ``schedule`` for the shape of ``desc``; fields it omits keep the
    built-in choice."""
    bad = set(schedule) - set(FIELDS)
    if bad:
        raise ValueError(f"unknown schedule fields {sorted(bad)}; the fields are {FIELDS}")
    full = dict(BUILTIN, **schedule)
    s = _lib.Schedule(*(int(full[f]) for f in FIELDS))
    lib = _lib.load()
    err = _lib.ctypes.create_string_buffer(_lib.ERR_CAP)
    _lib.check(lib.sweep_b200_schedule_set(_family(desc), _lib.ctypes.byref(desc), _lib.ctypes.byref(s),
                                           err, _lib.ERR_CAP), err)


def clear_schedules() -> None:
    """Forget every recorded schedule (the core's table and this module's record)."""
    _lib.load().sweep_b200_schedule_clear()
    _tuned.clear()


def _candidates(desc, builtin: dict, mem_mode: int, nt_tune: int) -> list:
    """(knob, values, forward_only) in tuning order."""
    knobs = []
    if isinstance(desc, _lib.ElasticDesc):
        per_shot = desc.model_stride != 0
        B = desc.B
        if not per_shot and B > 1:
            knobs.append(("shots_fwd", sorted({g for g in (1, 2, 4, 8) if g <= B} | {builtin["shots_fwd"]}), True))
            knobs.append(("shots_rev", sorted({g for g in (1, 2, 4, 8) if g <= B} | {builtin["shots_rev"]}), False))
    elif desc.ndim == 2:
        per_shot = desc.vp_stride != 0
        B = desc.B
        if not per_shot and B > 1:
            knobs.append(("shots_fwd", sorted({g for g in (1, 2, 4, 8) if g <= B} | {builtin["shots_fwd"]}), True))
            knobs.append(("shots_rev", sorted({g for g in (2, 4, 8, 16) if g <= B} | {builtin["shots_rev"]}), False))
    else:
        # the tile height first: the z-chunk count the core picks depends on it
        knobs.append(("tile_y", [8, 16], False))
        z = builtin["z_chunks"]
        knobs.append(("z_chunks", sorted({max(1, z // 2), z, min(_zmax(desc), 2 * z)}), False))
    if not mem_mode & _lib.MEM_HOST_TAPE:
        # a graph's capture and instantiation overlap the previous graph's run:
        # the trial holds four graphs, so that it sees the steady state of a
        # long time axis rather than the first graph's set-up alone
        knobs.append(("graph_steps", [0, max(1, min(64, nt_tune // 4))], False))
    return knobs


def _zmax(desc) -> int:
    """Most z chunks the core takes for this grid (chunks of >= 16 planes)."""
    return max(1, desc.nz // 16)


def _time(run, repeats: int) -> float:
    """Best wall time of ``repeats`` calls after one untimed call (seconds)."""
    best = float("inf")
    for i in range(repeats + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run()
        torch.cuda.synchronize()
        if i:
            best = min(best, time.perf_counter() - t0)
    return best


def tune(prop, geo, padded, wavelet, fields, mem_mode: int, ckpt_every: int,
         nt_tune: int | None = None, repeats: int = 2) -> dict:
    """Tune the schedule of one shape through the propagator's own calls.

    ``prop``, ``geo``, ``padded`` (runtime-grid models), ``wavelet``
    ``(B, nsrc, nt)``, ``fields`` (elastic source / receiver field indices, or
    None), ``mem_mode`` and ``ckpt_every`` are what ``PropTorch.forward``
    passes to its autograd function; the trials run a time axis of
    ``nt_tune`` steps.  Returns ``{"schedule": ..., "trials": {knob: {value:
    seconds}}, "nt": nt_tune, "seconds": total}``."""
    from .propagator import _AcousticFn, _ElasticFn

    t_start = time.perf_counter()
    elastic = fields is not None
    if nt_tune is None:
        nt_tune = 128 if elastic else (256 if geo.ndim == 2 else 16)
    nt_tune = max(2, min(int(nt_tune), geo.nt))
    g = copy.copy(geo)
    g.nt = nt_tune
    w = wavelet[..., :nt_tune].contiguous()
    models = [m.detach() for m in padded]
    desc = g.elastic_desc(models, w, *fields) if elastic else g.acoustic_desc(models[0], w)
    builtin = get_schedule(desc)
    gen = torch.Generator(device=models[0].device).manual_seed(0)
    saved = (prop.source_illumination, prop.receiver_illumination)

    def call(grad: bool):
        ms = [m.clone().requires_grad_(grad) for m in models]
        if elastic:
            rec = _ElasticFn.apply(*ms, w, prop, g, fields, mem_mode, ckpt_every)
        else:
            rec = _AcousticFn.apply(ms[0], w, prop, g, mem_mode, ckpt_every)
        if grad:
            rec.backward(torch.randn(rec.shape, generator=gen, device=rec.device))
        return rec

    def fwd():
        with torch.no_grad():
            call(False)

    def fwd_bwd():
        with torch.enable_grad():
            call(True)

    current = dict(builtin)
    trials = {}
    try:
        for knob, values, forward_only in _candidates(desc, builtin, mem_mode, nt_tune):
            if knob == "z_chunks":
                # around the count the core picks for the tile height chosen so far
                set_schedule(desc, current)
                z = get_schedule(desc)["z_chunks"]
                values = sorted({max(1, z // 2), z, min(_zmax(desc), 2 * z)})
            res = {}
            run = fwd if forward_only else fwd_bwd
            for v in values:
                set_schedule(desc, dict(current, **{knob: v}))
                res[v] = _time(run, repeats)
            # z chunks: keep doubling while the largest count tried is the fastest
            while knob == "z_chunks" and min(res, key=res.get) == max(res) and 2 * max(res) <= _zmax(desc):
                v = 2 * max(res)
                set_schedule(desc, dict(current, **{knob: v}))
                res[v] = _time(run, repeats)
            current[knob] = min(res, key=res.get)
            trials[knob] = res
    finally:
        set_schedule(desc, current)
        prop.source_illumination, prop.receiver_illumination = saved
    _tuned[shape_key(desc)] = dict(current)
    return {"schedule": get_schedule(desc), "trials": trials, "nt": nt_tune,
            "seconds": time.perf_counter() - t_start}


def tuned(desc) -> bool:
    """Whether :func:`tune` has recorded a schedule for this shape in this process."""
    return shape_key(desc) in _tuned
