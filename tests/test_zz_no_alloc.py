"""The allocation-free forward entry point, through the C ABI.

sweep_b200_acoustic_forward_noalloc serves callers that cannot allocate device
memory: its scratch is a static array inside the library.  Its records must
equal those of the regular entry point (sweep_b200_acoustic_forward, with a
workspace the caller allocates) on two calls in a row -- the second call runs
on the array the first one left behind.  This file is named to be collected
last; it passes alone in a fresh process and after the other tests."""
import ctypes

import numpy as np
import pytest
import torch

from tests._util import load, rel

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
REC_TOL = 1e-4


def _problem(case, vp_key):
    from sweep_b200 import Acoustic, PropTorch
    from sweep_b200.propagator import _Geometry, normalize_io
    d = load(case)
    s = PropTorch(Acoustic(8, device=DEV), shape=tuple(d["vp_true"].shape[-2:]), dh=float(d["dh"]),
                  dt=float(d["dt"]), abcn=int(d["abcn"]), device=DEV)
    w = torch.tensor(d["wavelet"], device=DEV)
    mode, B, nsrc = normalize_io(w, d["src"], d["rec"], 2)
    wb = (w[None, None, :].expand(B, 1, -1) if w.dim() == 1 else w[:, None, :]).contiguous()
    off = s.abcn + 4
    src = np.asarray(d["src"]).reshape(B, 1, 2) + off
    rec = np.asarray(d["rec"]).reshape(B, -1, 2) + off
    geo = _Geometry(s, B, 1, rec.shape[1], w.shape[-1], src, rec, DEV, 4500.0, 25.0)
    vp = s._pad_model(torch.tensor(d[vp_key], device=DEV)).contiguous()
    return geo, vp, wb


def _regular(geo, vp, wb):
    from sweep_b200 import _lib
    desc = geo.acoustic_desc(vp, wb)
    ws_b, tape_b = _lib.c_i64(), _lib.c_i64()
    _lib.call("sweep_b200_acoustic_sizes", desc, _lib.MEM_BOUNDARY, 0, ws_b, tape_b)
    ws = torch.empty(ws_b.value, dtype=torch.uint8, device=DEV)
    rec = torch.empty((geo.B, geo.nt, geo.nrec), device=DEV)
    _lib.call("sweep_b200_acoustic_forward", desc, _lib.MEM_BOUNDARY, 0, rec.data_ptr(), None,
              ws.data_ptr(), ws.numel(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rec.cpu().numpy()


def _noalloc(geo, vp, wb):
    from sweep_b200 import _lib
    desc = geo.acoustic_desc(vp, wb)
    rec = torch.full((geo.B, geo.nt, geo.nrec), float("nan"), device=DEV)
    _lib.call("sweep_b200_acoustic_forward_noalloc", desc, rec.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rec.cpu().numpy()


def test_noalloc_forward_matches_regular_entry_twice():
    geo, vp, wb = _problem("acoustic2d_multi", "vp_true")
    ref = _regular(geo, vp, wb)
    first = _noalloc(geo, vp, wb)
    assert rel(first, ref) < REC_TOL
    # a different model in between, then the first problem again: the array
    # keeps the last call's contents, which the next call must clear
    geo2, vp2, wb2 = _problem("acoustic2d_c1", "vp_true")
    other = _noalloc(geo2, vp2, wb2)
    assert rel(other, _regular(geo2, vp2, wb2)) < REC_TOL
    second = _noalloc(geo, vp, wb)
    assert rel(second, ref) < REC_TOL
    assert np.array_equal(first, second)


def test_noalloc_rejects_oversized_problems():
    from sweep_b200 import _lib
    geo, vp, wb = _problem("acoustic2d_multi", "vp_true")
    desc = geo.acoustic_desc(vp, wb)
    desc.B = 4000          # scratch need far above the static array (no device work is issued)
    with pytest.raises(RuntimeError, match="static array"):
        _lib.call("sweep_b200_acoustic_forward_noalloc", desc, None, None)
