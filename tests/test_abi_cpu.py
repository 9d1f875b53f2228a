"""The C ABI without a GPU: the library loads, exports every symbol its header
declares, reports the right ABI version, and the host-side size query and
argument checks work (no device work is issued)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "sweep_b200.h"


def _declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"SWEEP_B200_API\s+\w+\s+(sweep_b200_\w+)\s*\(", text)))


def test_header_and_loader_agree():
    from sweep_b200 import _lib
    assert sorted(_lib.SYMBOLS) == _declared()


def test_library_exports_every_declared_symbol():
    from sweep_b200 import _lib
    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name), name
    assert lib.sweep_b200_abi_version() == _lib.ABI_VERSION


def _desc(B=2, nz=40, nx=60, nt=10, nsrc=1, nrec=3, M=4):
    from sweep_b200 import _lib
    d = _lib.AcousticDesc()
    d.ndim, d.B, d.nz, d.ny, d.nx, d.nt, d.M = 2, B, nz, 1, nx, nt, M
    for i, p in enumerate([5, 5, 0, 0, 5, 5]):
        d.pad[i] = p
    d.dt, d.dz, d.dy, d.dx = 1e-3, 10.0, 1.0, 10.0
    d.nsrc, d.nrec = nsrc, nrec
    return d


def test_sizes_query_is_host_only():
    from sweep_b200 import _lib
    d = _desc()
    ws, tape = _lib.c_i64(), _lib.c_i64()
    _lib.call("sweep_b200_acoustic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    n = 2 * 40 * 60
    assert ws.value >= 14 * n * 4     # 3 adjoint + 8 adjoint-CPML + 3 reconstruction fields
    # strips (M + 1 = 5 wide) of a 22 x 42 physical box, per step and shot, plus the last two states
    pz, px = 40 - 2 * 9, 60 - 2 * 9
    nstrip = 2 * 5 * px + 2 * 5 * (pz - 10)
    assert tape.value >= (10 * 2 * nstrip + 2 * n) * 4


def test_errors_come_back_as_messages():
    from sweep_b200 import _lib
    d = _desc(M=8)
    ws, tape = _lib.c_i64(), _lib.c_i64()
    with pytest.raises(RuntimeError, match="orders 2 to 14"):
        _lib.call("sweep_b200_acoustic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d = _desc(M=3)                              # order 6: the any-order kernels, boundary saving only
    _lib.call("sweep_b200_acoustic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    px, pz = 60 - 2 * 8, 40 - 2 * 8
    assert tape.value == (10 * 2 * (px * pz - (px - 8) * (pz - 8)) + 2 * 2 * 40 * 60) * 4
    for mode in (_lib.MEM_CHECKPOINT, _lib.MEM_BOUNDARY_INT8, _lib.MEM_BOUNDARY | _lib.MEM_HOST_TAPE):
        with pytest.raises(RuntimeError, match="boundary saving with fp32 strips"):
            _lib.call("sweep_b200_acoustic_sizes", d, mode, 10, ws, tape)
    d = _desc()
    d.pad[0] = d.pad[5] = 0                    # free-surface faces (2-D: any)
    _lib.call("sweep_b200_acoustic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d.pad[4] = -1
    with pytest.raises(RuntimeError, match="PML pad"):
        _lib.call("sweep_b200_acoustic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d3 = _desc(nz=30, nx=30)
    d3.ndim, d3.ny = 3, 30
    for i in range(6):
        d3.pad[i] = 5
    d3.pad[4] = 0                              # 3-D: the top face only
    with pytest.raises(RuntimeError, match="PML pad"):
        _lib.call("sweep_b200_acoustic_sizes", d3, _lib.MEM_BOUNDARY, 0, ws, tape)
    with pytest.raises(RuntimeError, match="null"):
        _lib.call("sweep_b200_acoustic_sizes", None, _lib.MEM_BOUNDARY, 0, ws, tape)


def test_spatial_orders_on_the_host():
    """Orders 2 to 14 are accepted for Acoustic, Acoustic3D and Elastic (order
    8 on the tiled kernels, the others on the any-order ones) and 2 to 8 for
    Elastic3D; higher orders are refused when the solver is built; the
    elastic core sizes an order-4 problem and refuses its checkpoints."""
    import torch
    from sweep_b200 import Acoustic, Acoustic3D, Elastic, Elastic3D, PropTorch, _lib
    for order in (2, 4, 6, 8, 10, 14):
        PropTorch(Acoustic(spatial_order=order), shape=(20, 20), abcn=5, device="cpu")
        PropTorch(Acoustic3D(spatial_order=order), shape=(12, 12, 12), abcn=4, device="cpu")
        PropTorch(Elastic(spatial_order=order), shape=(20, 20), abcn=5, device="cpu")
    for eq in (Acoustic, Elastic):
        with pytest.raises(NotImplementedError, match="orders 2 to 14"):
            PropTorch(eq(spatial_order=16), shape=(20, 20), abcn=5, device="cpu")
    for order in (2, 4, 6, 8):
        PropTorch(Elastic3D(spatial_order=order), shape=(12, 12, 12), abcn=5, device="cpu")
    with pytest.raises(NotImplementedError, match="orders 2, 4, 6 and 8"):
        PropTorch(Elastic3D(spatial_order=10), shape=(12, 12, 12), abcn=5, device="cpu")
    s = PropTorch(Elastic(), shape=(30, 40), dh=5.0, dt=5e-4, abcn=6, device="cpu")
    geo, padded, wb, fields = s._probe(50, np.array([[8, 6]]), np.zeros((1, 4, 2), np.int64), [torch.ones(30, 40)] * 3)
    d = s._desc(geo, padded, wb, fields)
    assert d.M == 2
    ws, tape = _lib.c_i64(), _lib.c_i64()
    _lib.call("sweep_b200_elastic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    assert tape.value > 50 * 5 * 4 and ws.value > 0
    with pytest.raises(RuntimeError, match="boundary saving with fp32 strips"):
        _lib.call("sweep_b200_elastic_sizes", d, _lib.MEM_CHECKPOINT, 10, ws, tape)


def test_propagator_refuses_cpu_and_other_impls():
    import torch
    from sweep_b200 import Acoustic, PropTorch
    with pytest.raises(NotImplementedError):
        PropTorch(Acoustic(8), shape=(20, 20), impl="eager")
    p = PropTorch(Acoustic(8), shape=(20, 20), abcn=5, device="cpu")
    vp = torch.full((20, 20), 2000.0)
    with pytest.raises(RuntimeError, match="CUDA"):
        p(np.zeros(10, np.float32), np.array([[5, 5]]), np.array([[[6, 6]]]), models=[vp])


def _edesc(B=2, nz=40, nx=60, nt=10, nsrc=1, nrec=3, M=4):
    from sweep_b200 import _lib
    d = _lib.ElasticDesc()
    d.B, d.nz, d.nx, d.nt, d.M = B, nz, nx, nt, M
    for i in range(4):
        d.pad[i] = 5
    d.dt, d.dz, d.dx = 1e-3, 10.0, 10.0
    d.nsrc, d.nrec = nsrc, nrec
    d.nsrc_fields, d.nrec_fields = 2, 2
    d.src_fields[0], d.src_fields[1] = 2, 3
    d.rec_fields[0], d.rec_fields[1] = 0, 1
    return d


def test_elastic_sizes_and_errors():
    from sweep_b200 import _lib
    d = _edesc()
    ws, tape = _lib.c_i64(), _lib.c_i64()
    _lib.call("sweep_b200_elastic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    n = 2 * 40 * 64                                  # pitched to 64 columns
    assert ws.value >= 17 * n * 4                    # 5 forward + 2 carriers + 5 adjoint + 3 x 2 gradient slots
    pz, px = 40 - 18, 60 - 18
    nstrip = 2 * 4 * px + 2 * (px + 8) + (pz - 2) * 10
    assert tape.value >= (10 * 2 * 5 * nstrip + 5 * n) * 4
    d.src_fields[0] = 1                               # a body-force (vz) source is built
    _lib.call("sweep_b200_elastic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d.src_fields[0] = 7
    with pytest.raises(RuntimeError, match="bad source field"):
        _lib.call("sweep_b200_elastic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d.nsrc_fields, d.src_fields[0], d.src_fields[1] = 2, 3, 3
    with pytest.raises(RuntimeError, match="repeated"):
        _lib.call("sweep_b200_elastic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d = _edesc(M=8)
    with pytest.raises(RuntimeError, match="orders 2 to 14"):
        _lib.call("sweep_b200_elastic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d = _edesc(M=2)                                   # order 4: the any-order kernels
    _lib.call("sweep_b200_elastic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d.nsrc_fields, d.src_fields[0], d.src_fields[1] = 2, 3, 3
    with pytest.raises(RuntimeError, match="repeated"):
        _lib.call("sweep_b200_elastic_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)


@pytest.mark.parametrize("kind", ["acoustic2d", "acoustic3d", "elastic2d"])
def test_checkpoint_tape_is_smaller_for_long_runs(kind):
    """A long run's checkpoint tape (state every k steps) is a fraction of the
    boundary-saving tape (strips every step); the workspace grows by the
    replay set and one chunk of strips."""
    from sweep_b200 import _lib
    nt = 4000
    if kind == "elastic2d":
        d = _edesc(nz=120, nx=160, nt=nt)
        fn = "sweep_b200_elastic_sizes"
    else:
        d = _desc(nz=120, nx=160, nt=nt)
        if kind == "acoustic3d":
            d.ndim, d.ny = 3, 48
            for i in range(6):
                d.pad[i] = 5
        fn = "sweep_b200_acoustic_sizes"
    ws_b, tape_b, ws_c, tape_c = _lib.c_i64(), _lib.c_i64(), _lib.c_i64(), _lib.c_i64()
    _lib.call(fn, d, _lib.MEM_BOUNDARY, 0, ws_b, tape_b)
    _lib.call(fn, d, _lib.MEM_CHECKPOINT, 500, ws_c, tape_c)
    assert tape_c.value < tape_b.value
    assert ws_c.value > ws_b.value
    with pytest.raises(RuntimeError, match="interval"):
        _lib.call(fn, d, _lib.MEM_CHECKPOINT, 0, ws_c, tape_c)


def test_reduced_strip_storage_tape_sizes():
    """Boundary-saving tapes by strip format (host-side sizes query): bf16
    about half of fp32, fp16 half plus one FP32 scale per 256 cells of each
    face, int8 a quarter plus the scales; fp16 / int8 refuse a physical box
    narrower than two bands, and 3-D refuses the reduced formats."""
    from sweep_b200 import _lib
    nt = 400
    d = _desc(nz=120, nx=160, nt=nt)
    got = {}
    for name, mode in (("fp32", _lib.MEM_BOUNDARY), ("fp16", _lib.MEM_BOUNDARY_FP16),
                       ("bf16", _lib.MEM_BOUNDARY_BF16), ("int8", _lib.MEM_BOUNDARY_INT8)):
        ws, tape = _lib.c_i64(), _lib.c_i64()
        _lib.call("sweep_b200_acoustic_sizes", d, mode, 0, ws, tape)
        got[name] = tape.value
    n = 2 * 120 * 160 * 4 * 2                 # the last two states, pitched rows of 160 floats
    strips = {k: v - n for k, v in got.items()}
    assert 0.49 < strips["bf16"] / strips["fp32"] < 0.52
    assert 0.5 < strips["fp16"] / strips["fp32"] < 0.56
    assert 0.25 < strips["int8"] / strips["fp32"] < 0.31
    small = _desc(nz=26, nx=160, nt=nt)        # an 8-row physical box
    ws, tape = _lib.c_i64(), _lib.c_i64()
    _lib.call("sweep_b200_acoustic_sizes", small, _lib.MEM_BOUNDARY_BF16, 0, ws, tape)
    with pytest.raises(RuntimeError, match="at least 10 cells"):
        _lib.call("sweep_b200_acoustic_sizes", small, _lib.MEM_BOUNDARY_INT8, 0, ws, tape)
    d3 = _desc(nz=40, nx=40, nt=10)
    d3.ndim, d3.ny = 3, 40
    for i in range(6):
        d3.pad[i] = 5
    t3 = {}
    for name, mode in (("fp32", _lib.MEM_BOUNDARY), ("int8", _lib.MEM_BOUNDARY_INT8)):
        _lib.call("sweep_b200_acoustic_sizes", d3, mode, 0, ws, tape)
        t3[name] = tape.value
    assert t3["int8"] < t3["fp32"]
    te = {}
    for name, mode in (("fp32", _lib.MEM_BOUNDARY), ("bf16", _lib.MEM_BOUNDARY_BF16), ("int8", _lib.MEM_BOUNDARY_INT8)):
        _lib.call("sweep_b200_elastic_sizes", _edesc(nz=60, nx=60, nt=10), mode, 0, ws, tape)
        te[name] = tape.value
    assert te["int8"] < te["bf16"] < te["fp32"]
    with pytest.raises(RuntimeError, match="memory mode"):
        _lib.call("sweep_b200_elastic_sizes", _edesc(nz=60, nx=60, nt=10), 7, 0, ws, tape)


def test_free_surface_spellings():
    """The reference's free_surface spellings (equations/_edges.py:66-140)."""
    from sweep_b200.propagator import free_faces
    assert free_faces(True, 2) == (True, False, False, False)
    assert free_faces(False, 3) == (False,) * 6
    assert free_faces(None, 2) == (False,) * 4
    assert free_faces("left", 2) == (False, False, True, False)
    assert free_faces(["top", "right"], 2) == (True, False, False, True)
    assert free_faces({"bottom": 1, "top": 0}, 2) == (False, True, False, False)
    assert free_faces([1, 0, 0, 1], 2) == (True, False, False, True)
    with pytest.raises(ValueError, match="unknown"):
        free_faces(["front"], 2)


def test_schedule_table_is_host_only_and_keyed_by_shape():
    """The per-shape schedule table: recorded fields win, the rest resolve to
    the built-in choice; nt, sources and receivers are not part of the key;
    out-of-range values are refused with a message."""
    from sweep_b200 import _lib, autotune
    autotune.clear_schedules()
    try:
        d = _desc(B=8, nz=120, nx=200)
        base = autotune.get_schedule(d)
        assert base["shots_fwd"] >= 1 and base["shots_rev"] >= 1 and base["graph_steps"] >= 0
        autotune.set_schedule(d, {"shots_rev": 4, "graph_steps": 0})
        got = autotune.get_schedule(d)
        assert got["shots_rev"] == 4 and got["graph_steps"] == 0 and got["shots_fwd"] == base["shots_fwd"]
        d.nt, d.nrec = 999, 7                   # same shape: same schedule
        assert autotune.get_schedule(d) == got
        other = _desc(B=4, nz=120, nx=200)      # another shot count: another shape
        assert autotune.get_schedule(other)["graph_steps"] == base["graph_steps"]
        d.vp_stride = 120 * 200                 # per-shot models always run one shot per CTA
        assert autotune.get_schedule(d)["shots_rev"] == 1
        with pytest.raises(RuntimeError, match="shots_fwd"):
            autotune.set_schedule(d, {"shots_fwd": 17})
        with pytest.raises(ValueError, match="unknown schedule"):
            autotune.set_schedule(d, {"tile": 3})
        d3 = _desc(B=2, nz=64, nx=64)
        d3.ndim, d3.ny = 3, 64
        for i in range(6):
            d3.pad[i] = 5
        autotune.set_schedule(d3, {"z_chunks": 2})
        assert autotune.get_schedule(d3)["z_chunks"] == 2
        assert autotune.get_schedule(d3)["tile_y"] == 8       # the built-in tile height
        autotune.set_schedule(d3, {"z_chunks": 2, "tile_y": 16})
        assert autotune.get_schedule(d3)["tile_y"] == 16
        with pytest.raises(RuntimeError, match="tile_y"):
            autotune.set_schedule(d3, {"tile_y": 12})
        e = _lib.ElasticDesc()
        e.B, e.nz, e.nx, e.nt, e.M = 6, 80, 90, 10, 4
        for i in range(4):
            e.pad[i] = 10
        e.nsrc_fields, e.src_fields[0], e.nrec_fields = 1, 2, 1
        autotune.set_schedule(e, {"shots_fwd": 3, "shots_rev": 2})
        s = autotune.get_schedule(e)
        assert (s["shots_fwd"], s["shots_rev"]) == (3, 2)
    finally:
        autotune.clear_schedules()
    assert autotune.get_schedule(_desc(B=8, nz=120, nx=200)) == base


def test_recursive_checkpoint_options_and_sizes():
    """Ckpt(mode='recursive', count=N) follows the reference's option rules;
    its tape is a token (nothing is kept from the forward) and its workspace
    grows by one snapshot per unit of budget."""
    from sweep_b200 import Ckpt, _lib
    assert Ckpt(mode="recursive", count=3).count == 3
    with pytest.raises(ValueError):
        Ckpt(mode="recursive")
    with pytest.raises(ValueError):
        Ckpt(chunks=10, count=2)
    with pytest.raises(ValueError):
        Ckpt(mode="revolve", count=2)
    d = _desc(B=2, nz=40, nx=60, nt=300)
    ws1, ws2, tape = _lib.c_i64(), _lib.c_i64(), _lib.c_i64()
    _lib.call("sweep_b200_acoustic_sizes", d, _lib.MEM_RECURSIVE, 1, ws1, tape)
    assert tape.value <= 256
    _lib.call("sweep_b200_acoustic_sizes", d, _lib.MEM_RECURSIVE, 5, ws2, tape)
    assert ws2.value > ws1.value
    with pytest.raises(RuntimeError, match="budget"):
        _lib.call("sweep_b200_acoustic_sizes", d, _lib.MEM_RECURSIVE, 0, ws1, tape)


def test_autotune_candidates_follow_the_shape():
    """The tuner's knobs: shot grouping only with several shots sharing a
    model, z chunks only in 3-D (doubling bounded by 16-plane chunks), graph
    length only without a host tape; each knob's values include the
    built-in choice."""
    from sweep_b200 import _lib, autotune
    d = _desc(B=8, nz=120, nx=200)
    base = {"shots_fwd": 2, "shots_rev": 8, "z_chunks": 0, "graph_steps": 64}
    knobs = {k: v for k, v, _ in autotune._candidates(d, base, _lib.MEM_BOUNDARY, 256)}
    assert set(knobs) == {"shots_fwd", "shots_rev", "graph_steps"}
    assert 2 in knobs["shots_fwd"] and 8 in knobs["shots_rev"] and max(knobs["shots_rev"]) <= 8
    assert knobs["graph_steps"] == [0, 64]
    host = {k for k, _, _ in autotune._candidates(d, base, _lib.MEM_BOUNDARY | _lib.MEM_HOST_TAPE, 256)}
    assert "graph_steps" not in host
    d.vp_stride = 120 * 200                          # per-shot models: one shot per CTA, nothing to group
    assert {k for k, _, _ in autotune._candidates(d, base, _lib.MEM_BOUNDARY, 256)} == {"graph_steps"}
    d3 = _desc(B=4, nz=64, nx=64)
    d3.ndim, d3.ny = 3, 64
    knobs3 = {k: v for k, v, _ in autotune._candidates(d3, dict(base, z_chunks=2), _lib.MEM_BOUNDARY, 16)}
    assert knobs3["z_chunks"] == [1, 2, 4] and autotune._zmax(d3) == 4
    assert knobs3["graph_steps"] == [0, 4]
    assert knobs3["tile_y"] == [8, 16]
    order = [k for k, _, _ in autotune._candidates(d3, dict(base, z_chunks=2), _lib.MEM_BOUNDARY, 16)]
    assert order.index("tile_y") < order.index("z_chunks")


def test_tape_budget_rule_is_host_side():
    """BoundarySaving(budget_gb=...) picks the memory mode from the host-only
    size query: boundary saving while the tape fits, else checkpoints."""
    import numpy as np
    import torch
    from sweep_b200 import Acoustic, BoundarySaving, PropTorch, _lib
    vp = torch.full((30, 40), 2000.0)
    src, rec = np.array([[5, 2], [20, 2]]), np.array([[[10, 2]], [[30, 2]]])
    for budget, mode in ((100.0, "boundary"), (1e-6, "checkpoint")):
        s = PropTorch(Acoustic(spatial_order=8, device="cpu"), shape=(30, 40), dh=10.0, dt=1e-3, abcn=10,
                      device="cpu", memory=BoundarySaving(budget_gb=budget, ckpt_chunks=25))
        tape = s.tape_bytes(200, src, rec, [vp])
        geo, padded, wb, fields = s._probe(200, src, rec, [vp])
        got = s._apply_budget(geo, padded, wb, fields, _lib.MEM_BOUNDARY, 0)
        assert s.last_memory["mode"] == mode
        if mode == "boundary":
            assert got == (_lib.MEM_BOUNDARY, 0) and s.last_memory["tape_bytes"] == tape
        else:
            assert got == (_lib.MEM_CHECKPOINT, 25) and s.last_memory["boundary_tape_bytes"] == tape


def test_recursive_sizes_every_equation():
    """The recursive mode's sizes for 3-D acoustic and elastic: a token tape,
    a workspace that grows with the snapshot budget and exceeds the
    boundary-saving one by at least one snapshot; a host tape is refused."""
    from sweep_b200 import _lib
    d3 = _desc(B=1, nz=40, nx=40, nt=200)
    d3.ndim, d3.ny = 3, 40
    for i in range(6):
        d3.pad[i] = 5
    e = _edesc(nt=200)
    for name, d in (("sweep_b200_acoustic_sizes", d3), ("sweep_b200_elastic_sizes", e)):
        ws_bs, ws1, ws4, tape = _lib.c_i64(), _lib.c_i64(), _lib.c_i64(), _lib.c_i64()
        _lib.call(name, d, _lib.MEM_BOUNDARY, 0, ws_bs, tape)
        _lib.call(name, d, _lib.MEM_RECURSIVE, 1, ws1, tape)
        assert tape.value <= 256
        _lib.call(name, d, _lib.MEM_RECURSIVE, 4, ws4, tape)
        assert ws4.value > ws1.value > ws_bs.value
        with pytest.raises(RuntimeError, match="host tape"):
            _lib.call(name, d, _lib.MEM_RECURSIVE | _lib.MEM_HOST_TAPE, 2, ws1, tape)


def test_elastic_free_surface_faces_checked():
    """The elastic core takes traction-free faces with no pad on them and an
    absorbing pad on every other face (host-side checks, no device work);
    the public API drops a free face's pad."""
    from sweep_b200 import Elastic, PropTorch, _lib
    e = _lib.ElasticDesc()
    e.B, e.nz, e.nx, e.nt, e.M = 2, 60, 80, 10, 4
    e.pad[0], e.pad[1], e.pad[2], e.pad[3] = 0, 10, 10, 10
    e.nsrc_fields, e.src_fields[0], e.nrec_fields = 1, 2, 1
    ws, tape = _lib.c_i64(), _lib.c_i64()
    with pytest.raises(RuntimeError, match="pad"):
        _lib.call("sweep_b200_elastic_sizes", e, _lib.MEM_BOUNDARY, 0, ws, tape)
    e.free_surface[0] = 1
    _lib.call("sweep_b200_elastic_sizes", e, _lib.MEM_BOUNDARY, 0, ws, tape)
    assert ws.value > 0 and tape.value > 0
    e.pad[0] = 3
    with pytest.raises(RuntimeError, match="free face has no PML pad"):
        _lib.call("sweep_b200_elastic_sizes", e, _lib.MEM_BOUNDARY, 0, ws, tape)
    e.pad[0], e.free_surface[3] = 0, 1
    with pytest.raises(RuntimeError, match="free face has no PML pad"):
        _lib.call("sweep_b200_elastic_sizes", e, _lib.MEM_BOUNDARY, 0, ws, tape)
    e.pad[3] = 0
    _lib.call("sweep_b200_elastic_sizes", e, _lib.MEM_BOUNDARY, 0, ws, tape)
    eq = Elastic(spatial_order=8, device="cpu")
    s = PropTorch(eq, shape=(30, 40), dh=5.0, dt=0.0005, abcn=8, device="cpu", free_surface=True)
    assert s.pads == [0, 8, 8, 8] and s.runtime_shape == (30 + 8 + 8, 40 + 16 + 8)
    s = PropTorch(eq, shape=(30, 40), dh=5.0, dt=0.0005, abcn=8, device="cpu", free_surface=["left", "bottom"])
    assert s.pads == [8, 0, 0, 8] and s.runtime_shape == (30 + 8 + 8, 40 + 8 + 8)


def test_elastic3d_sizes_and_refusals():
    """The 3-D elastic core sizes its workspace and tape on the host for every
    memory mode and refuses bad ones (a host tape with checkpoints, unknown
    modes, a zero interval, faces other than the top one as free surfaces)
    before any device work."""
    import numpy as np
    import torch
    from sweep_b200 import Ckpt, Elastic3D, PropTorch, _lib
    eq = Elastic3D(spatial_order=8, device="cpu")
    s = PropTorch(eq, shape=(20, 22, 24), dh=5.0, dt=0.0005, abcn=6, device="cpu")
    assert s.runtime_shape == (40, 42, 44) and eq.default_source_fields == ["sxx", "syy", "szz"]
    src, rec = np.array([[8, 10, 6]]), np.zeros((1, 4, 3), np.int64)
    geo, padded, wb, fields = s._probe(50, src, rec, [torch.ones(20, 22, 24)] * 3)
    d = s._desc(geo, padded, wb, fields)
    ws, tape = _lib.c_i64(), _lib.c_i64()
    _lib.call("sweep_b200_elastic3d_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    assert ws.value > 0 and tape.value > 50 * 9 * 4
    tapes = {}
    for mode in (_lib.MEM_BOUNDARY, _lib.MEM_BOUNDARY_FP16, _lib.MEM_BOUNDARY_BF16, _lib.MEM_BOUNDARY_INT8,
                 _lib.MEM_BOUNDARY | _lib.MEM_HOST_TAPE, _lib.MEM_CHECKPOINT, _lib.MEM_RECURSIVE):
        _lib.call("sweep_b200_elastic3d_sizes", d, mode, 10, ws, tape)
        tapes[mode] = tape.value
    state = 9 * 40 * 42 * 44 * 4                     # the final nine-field state closes the tape
    strips = tapes[_lib.MEM_BOUNDARY] - state
    assert tapes[_lib.MEM_BOUNDARY | _lib.MEM_HOST_TAPE] == tapes[_lib.MEM_BOUNDARY]
    assert abs((tapes[_lib.MEM_BOUNDARY_BF16] - state) / strips - 0.5) < 0.01
    assert (tapes[_lib.MEM_BOUNDARY_INT8] - state) < (tapes[_lib.MEM_BOUNDARY_FP16] - state) < strips
    assert tapes[_lib.MEM_CHECKPOINT] < tapes[_lib.MEM_BOUNDARY] and tapes[_lib.MEM_RECURSIVE] == 256
    for mode, every, msg in ((_lib.MEM_CHECKPOINT | _lib.MEM_HOST_TAPE, 10, "host tape"), (77, 10, "unknown"),
                             (_lib.MEM_CHECKPOINT, 0, "interval"), (_lib.MEM_RECURSIVE, 0, "budget")):
        with pytest.raises(RuntimeError, match=msg):
            _lib.call("sweep_b200_elastic3d_sizes", d, mode, every, ws, tape)
    d.M = 2                                            # order 4: the same sizes rule, its own strips
    _lib.call("sweep_b200_elastic3d_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d.M = 5
    with pytest.raises(RuntimeError, match="orders 2, 4, 6 and 8"):
        _lib.call("sweep_b200_elastic3d_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    fs = PropTorch(eq, shape=(20, 22, 24), dh=5.0, dt=0.0005, abcn=6, device="cpu", free_surface=True)
    assert fs.pads == [0, 6, 6, 6, 6, 6]
    geo, padded, wb, fields = fs._probe(50, src, rec, [torch.ones(20, 22, 24)] * 3)
    d = fs._desc(geo, padded, wb, fields)
    assert d.free_surface == 1 and d.pad[0] == 0
    _lib.call("sweep_b200_elastic3d_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d.pad[0] = 2
    with pytest.raises(RuntimeError, match="free top face"):
        _lib.call("sweep_b200_elastic3d_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    with pytest.raises(NotImplementedError, match="per-face"):
        PropTorch(eq, shape=(20, 22, 24), dh=5.0, dt=0.0005, abcn=6, device="cpu", free_surface=["bottom"])
    with pytest.raises(NotImplementedError, match="Elastic3D runs whole passes"):
        s.forward_runner(torch.zeros(50), src, rec, [torch.ones(20, 22, 24)] * 3)
    with pytest.raises(ValueError, match="source_type"):
        PropTorch(eq, shape=(20, 22, 24), dh=5.0, dt=0.0005, abcn=6, device="cpu",
                  source_type=["sxz", "pressure"])._elastic_fields()


def test_vti_sizes_and_refusals():
    """The 2-D acoustic VTI core sizes its workspace and tape on the host,
    takes every order 2 to 14, and refuses other memory modes, free surfaces,
    stepped runners and tuning."""
    import torch
    from sweep_b200 import AcousticVTI1st, Ckpt, PropTorch, _lib
    eq = AcousticVTI1st(spatial_order=8)
    assert eq.default_source_fields == ["sH", "sV"] and eq.default_receiver_fields == ["vz"]
    s = PropTorch(eq, shape=(30, 40), dh=5.0, dt=5e-4, abcn=6, device="cpu")
    src, rec = np.array([[8, 6]]), np.zeros((1, 4, 2), np.int64)
    models = [torch.full((30, 40), 2000.0), torch.full((30, 40), 0.1), torch.full((30, 40), 0.05),
              torch.full((30, 40), 2000.0)]
    geo, padded, wb, fields = s._probe(50, src, rec, models)
    d = s._desc(geo, padded, wb, fields)
    assert isinstance(d, _lib.VTIDesc) and d.M == 4 and list(d.pad) == [6, 6, 6, 6]
    ws, tape = _lib.c_i64(), _lib.c_i64()
    _lib.call("sweep_b200_vti_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    assert tape.value > 50 * 4 * 4 and ws.value > 0
    assert s.launch_schedule(50, src, rec, models) == {"fixed": "one thread per cell, 32 x 8 cell tiles per shot"}
    for mode in (_lib.MEM_CHECKPOINT, _lib.MEM_BOUNDARY_FP16, _lib.MEM_BOUNDARY | _lib.MEM_HOST_TAPE):
        with pytest.raises(RuntimeError, match="boundary saving with fp32 strips"):
            _lib.call("sweep_b200_vti_sizes", d, mode, 10, ws, tape)
    d.M = 8
    with pytest.raises(RuntimeError, match="orders 2 to 14"):
        _lib.call("sweep_b200_vti_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    with pytest.raises(NotImplementedError, match="no free surface"):
        PropTorch(eq, shape=(30, 40), abcn=6, device="cpu", free_surface=True)
    with pytest.raises(NotImplementedError, match="whole passes"):
        s.forward_runner(torch.zeros(50), src, rec, models)
    with pytest.raises(ValueError, match="source_type"):
        PropTorch(eq, shape=(30, 40), abcn=6, device="cpu", source_type=["sxx"])._elastic_fields()


def test_vti3d_sizes_and_refusals():
    """The 3-D acoustic VTI core sizes its workspace and tape on the host (the
    tape: nt steps of five fields' band cells plus the five final fields),
    takes every order 2 to 14, and refuses other memory modes, B * nz above
    the grid limit, free surfaces and stepped runners."""
    import torch
    from sweep_b200 import AcousticVTI1st3D, PropTorch, _lib
    eq = AcousticVTI1st3D()
    assert eq.spatial_order == 4 and eq.FIELDS == ("vx", "vy", "vz", "sH", "sV")
    assert eq.default_source_fields == ["sH", "sV"] and eq.default_receiver_fields == ["vz"]
    shape = (10, 12, 14)
    s = PropTorch(eq, shape=shape, dh=5.0, dt=5e-4, abcn=3, device="cpu", receiver_type=["vx", "vy", "sV"])
    src, rec = np.array([[4, 5, 3]]), np.zeros((1, 4, 3), np.int64)
    models = [torch.full(shape, 2000.0), torch.full(shape, 0.1), torch.full(shape, 0.05), torch.full(shape, 2000.0)]
    geo, padded, wb, fields = s._probe(50, src, rec, models)
    d = s._desc(geo, padded, wb, fields)
    assert isinstance(d, _lib.VTI3DDesc) and d.M == 2 and list(d.pad) == [3] * 6
    assert (d.nz, d.ny, d.nx) == (20, 22, 24) and list(d.rec_fields)[:3] == [0, 1, 4]
    ws, tape = _lib.c_i64(), _lib.c_i64()
    _lib.call("sweep_b200_vti3d_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    # band cells: the three face pairs (M + 1 = 3 deep) over the 10 x 12 x 14 box, each cell once
    box = np.zeros((20, 22, 24), bool)
    z0, y0, x0 = 5, 5, 5
    for lo, hi in ((z0 - 2, z0 + 1), (z0 + 9, z0 + 12)):
        box[lo:hi, y0:y0 + 12, x0:x0 + 14] = True
    for lo, hi in ((y0 - 2, y0 + 1), (y0 + 11, y0 + 14)):
        box[z0:z0 + 10, lo:hi, x0:x0 + 14] = True
    for lo, hi in ((x0 - 2, x0 + 1), (x0 + 13, x0 + 16)):
        box[z0:z0 + 10, y0:y0 + 12, lo:hi] = True
    assert tape.value == 4 * (50 * 5 * int(box.sum()) + 5 * 20 * 22 * 24)
    assert s.launch_schedule(50, src, rec, models) == {
        "fixed": "one thread per cell, 32 x 4 x 2 cell blocks, two z planes of a shot per grid row"}
    for mode in (_lib.MEM_CHECKPOINT, _lib.MEM_BOUNDARY_FP16):
        with pytest.raises(RuntimeError, match="boundary saving with fp32 strips"):
            _lib.call("sweep_b200_vti3d_sizes", d, mode, 10, ws, tape)
    d.B = 4000
    with pytest.raises(RuntimeError, match="65535"):
        _lib.call("sweep_b200_vti3d_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    d.B, d.M = 1, 8
    with pytest.raises(RuntimeError, match="orders 2 to 14"):
        _lib.call("sweep_b200_vti3d_sizes", d, _lib.MEM_BOUNDARY, 0, ws, tape)
    with pytest.raises(NotImplementedError, match="no free surface"):
        PropTorch(eq, shape=shape, abcn=3, device="cpu", free_surface=True)
    with pytest.raises(NotImplementedError, match="whole passes"):
        s.forward_runner(torch.zeros(50), src, rec, models)
    with pytest.raises(NotImplementedError, match="orders 2 to 14"):
        PropTorch(AcousticVTI1st3D(spatial_order=16), shape=shape, abcn=3, device="cpu")
