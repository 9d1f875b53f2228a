"""ctypes binding of ``libsweep_b200.so`` (declared in ``include/sweep_b200.h``).

The Python side of the C ABI, in the role of the reference's ctypes layer
(reference ``src/sweep/backend/c/entries.py:119-146``, ``loader.py:29-138``):
load the core once, check its ABI version and that every declared symbol is
exported, pack plain descriptors, run each call on torch's current stream and
turn a non-zero return into ``RuntimeError`` with the core's message.

There is no fallback: if the library is missing or fails to load, every call
raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("SWEEP_B200_LIB", HERE / "libsweep_b200.so"))
ABI_VERSION = 8
ERR_CAP = 4096

c_i32, c_i64, c_f32, c_p = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_void_p

# Every symbol include/sweep_b200.h declares.
SYMBOLS = (
    "sweep_b200_abi_version",
    "sweep_b200_acoustic_sizes",
    "sweep_b200_acoustic_forward",
    "sweep_b200_acoustic_backward",
    "sweep_b200_acoustic_forward_noalloc",
    "sweep_b200_elastic_sizes",
    "sweep_b200_elastic_forward",
    "sweep_b200_elastic_backward",
    "sweep_b200_elastic3d_sizes",
    "sweep_b200_elastic3d_forward",
    "sweep_b200_elastic3d_backward",
    "sweep_b200_vti_sizes",
    "sweep_b200_vti_forward",
    "sweep_b200_vti_backward",
    "sweep_b200_vti3d_sizes",
    "sweep_b200_vti3d_forward",
    "sweep_b200_vti3d_backward",
    "sweep_b200_conv3x3_gemm",
    "sweep_b200_conv3x3_wgrad",
    "sweep_b200_conv3x3_status",
    "sweep_b200_schedule_set",
    "sweep_b200_schedule_get",
    "sweep_b200_schedule_clear",
    "sweep_b200_wait_selftest",
    "sweep_b200_acoustic_forward_runner_create",
    "sweep_b200_acoustic_backward_runner_create",
    "sweep_b200_elastic_forward_runner_create",
    "sweep_b200_elastic_backward_runner_create",
    "sweep_b200_forward_runner_run",
    "sweep_b200_backward_runner_run",
    "sweep_b200_runner_device_index",
    "sweep_b200_runner_destroy",
)

MEM_BOUNDARY = 0
MEM_CHECKPOINT = 1
MEM_BOUNDARY_FP16 = 2            # boundary saving, strips stored as scaled fp16 / bf16 / scaled int8
MEM_BOUNDARY_BF16 = 3
MEM_BOUNDARY_INT8 = 4
MEM_HOST_TAPE = 0x100           # OR'ed into a boundary-saving mode: the tape is pinned host memory
MEM_RECURSIVE = 5               # recursive checkpointing, ckpt_every = snapshot budget
RECURSIVE_LEAF = 64

FAMILY_ACOUSTIC = 0
FAMILY_ELASTIC = 1


class AcousticDesc(ctypes.Structure):
    """Mirror of ``sweep_acoustic_desc``."""
    _fields_ = [
        ("ndim", c_i32), ("B", c_i32), ("nz", c_i32), ("ny", c_i32), ("nx", c_i32),
        ("nt", c_i32), ("M", c_i32), ("pad", c_i32 * 6),
        ("dt", c_f32), ("dz", c_f32), ("dy", c_f32), ("dx", c_f32),
        ("lap", c_f32 * 8), ("grad", c_f32 * 8),
        ("az", c_p), ("bz", c_p), ("dbz", c_p),
        ("ay", c_p), ("by", c_p), ("dby", c_p),
        ("ax", c_p), ("bx", c_p), ("dbx", c_p),
        ("vp", c_p), ("vp_stride", c_i64),
        ("nsrc", c_i32), ("src_loc", c_p), ("wavelet", c_p),
        ("nrec", c_i32), ("rec_loc", c_p),
    ]


class ElasticDesc(ctypes.Structure):
    """Mirror of ``sweep_elastic_desc``."""
    _fields_ = [
        ("B", c_i32), ("nz", c_i32), ("nx", c_i32), ("nt", c_i32), ("M", c_i32),
        ("pad", c_i32 * 4),
        ("dt", c_f32), ("dz", c_f32), ("dx", c_f32),
        ("az", c_p), ("bz", c_p), ("azh", c_p), ("bzh", c_p),
        ("ax", c_p), ("bx", c_p), ("axh", c_p), ("bxh", c_p),
        ("vp", c_p), ("vs", c_p), ("rho", c_p), ("model_stride", c_i64),
        ("nsrc", c_i32), ("src_loc", c_p), ("wavelet", c_p),
        ("nsrc_fields", c_i32), ("src_fields", c_i32 * 5),
        ("nrec", c_i32), ("rec_loc", c_p),
        ("nrec_fields", c_i32), ("rec_fields", c_i32 * 5),
        ("free_surface", c_i32 * 4),
    ]


class Elastic3DDesc(ctypes.Structure):
    """Mirror of ``sweep_elastic3d_desc``."""
    _fields_ = [
        ("B", c_i32), ("nz", c_i32), ("ny", c_i32), ("nx", c_i32), ("nt", c_i32), ("M", c_i32),
        ("pad", c_i32 * 6),
        ("dt", c_f32), ("dz", c_f32), ("dy", c_f32), ("dx", c_f32),
        ("az", c_p), ("bz", c_p), ("azh", c_p), ("bzh", c_p),
        ("ay", c_p), ("by", c_p), ("ayh", c_p), ("byh", c_p),
        ("ax", c_p), ("bx", c_p), ("axh", c_p), ("bxh", c_p),
        ("vp", c_p), ("vs", c_p), ("rho", c_p), ("model_stride", c_i64),
        ("nsrc", c_i32), ("src_loc", c_p), ("wavelet", c_p),
        ("nsrc_fields", c_i32), ("src_fields", c_i32 * 9),
        ("nrec", c_i32), ("rec_loc", c_p),
        ("nrec_fields", c_i32), ("rec_fields", c_i32 * 9),
        ("free_surface", c_i32),
    ]


class VTIDesc(ctypes.Structure):
    """Mirror of ``sweep_vti_desc``."""
    _fields_ = [
        ("B", c_i32), ("nz", c_i32), ("nx", c_i32), ("nt", c_i32), ("M", c_i32), ("pad", c_i32 * 4),
        ("dt", c_f32), ("dz", c_f32), ("dx", c_f32),
        ("az", c_p), ("bz", c_p), ("azh", c_p), ("bzh", c_p),
        ("ax", c_p), ("bx", c_p), ("axh", c_p), ("bxh", c_p),
        ("vp", c_p), ("epsilon", c_p), ("delta", c_p), ("rho", c_p), ("model_stride", c_i64),
        ("nsrc", c_i32), ("src_loc", c_p), ("wavelet", c_p),
        ("nsrc_fields", c_i32), ("src_fields", c_i32 * 4),
        ("nrec", c_i32), ("rec_loc", c_p),
        ("nrec_fields", c_i32), ("rec_fields", c_i32 * 4),
    ]


class VTI3DDesc(ctypes.Structure):
    """Mirror of ``sweep_vti3d_desc``."""
    _fields_ = [
        ("B", c_i32), ("nz", c_i32), ("ny", c_i32), ("nx", c_i32), ("nt", c_i32), ("M", c_i32),
        ("pad", c_i32 * 6), ("dt", c_f32), ("dz", c_f32), ("dy", c_f32), ("dx", c_f32),
        ("az", c_p), ("bz", c_p), ("azh", c_p), ("bzh", c_p),
        ("ay", c_p), ("by", c_p), ("ayh", c_p), ("byh", c_p),
        ("ax", c_p), ("bx", c_p), ("axh", c_p), ("bxh", c_p),
        ("vp", c_p), ("epsilon", c_p), ("delta", c_p), ("rho", c_p), ("model_stride", c_i64),
        ("nsrc", c_i32), ("src_loc", c_p), ("wavelet", c_p),
        ("nsrc_fields", c_i32), ("src_fields", c_i32 * 5),
        ("nrec", c_i32), ("rec_loc", c_p),
        ("nrec_fields", c_i32), ("rec_fields", c_i32 * 5),
    ]


class Schedule(ctypes.Structure):
    """Mirror of ``sweep_b200_schedule``."""
    _fields_ = [("shots_fwd", c_i32), ("shots_rev", c_i32), ("z_chunks", c_i32), ("graph_steps", c_i32),
                ("tile_y", c_i32)]


_lib = None


def load():
    """The loaded core; raises if it is missing, stale or incomplete."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"sweep_b200: the CUDA core {LIB_PATH} is not built; run "
            "`python -c 'import __graft_entry__ as g; g.build()'` (or make -C sweep_b200/csrc)")
    lib = ctypes.CDLL(str(LIB_PATH))
    missing = [s for s in SYMBOLS if not hasattr(lib, s)]
    if missing:
        raise RuntimeError(f"sweep_b200: {LIB_PATH} lacks symbols {missing}")
    lib.sweep_b200_abi_version.restype = ctypes.c_int
    ver = lib.sweep_b200_abi_version()
    if ver != ABI_VERSION:
        raise RuntimeError(f"sweep_b200: core ABI {ver} != expected {ABI_VERSION}; rebuild it")
    P = ctypes.POINTER(AcousticDesc)
    lib.sweep_b200_acoustic_sizes.argtypes = [P, c_i32, c_i32, ctypes.POINTER(c_i64),
                                              ctypes.POINTER(c_i64), ctypes.c_char_p, c_i32]
    lib.sweep_b200_acoustic_forward.argtypes = [P, c_i32, c_i32, c_p, c_p, c_p, c_i64, c_p,
                                                ctypes.c_char_p, c_i32]
    lib.sweep_b200_acoustic_backward.argtypes = [P, c_i32, c_i32, c_p, c_p, c_p, c_p, c_p, c_p,
                                                 c_p, c_i64, c_p, ctypes.c_char_p, c_i32]
    lib.sweep_b200_acoustic_forward_noalloc.argtypes = [P, c_p, c_p, ctypes.c_char_p, c_i32]
    E = ctypes.POINTER(ElasticDesc)
    lib.sweep_b200_elastic_sizes.argtypes = [E, c_i32, c_i32, ctypes.POINTER(c_i64),
                                             ctypes.POINTER(c_i64), ctypes.c_char_p, c_i32]
    lib.sweep_b200_elastic_forward.argtypes = [E, c_i32, c_i32, c_p, c_p, c_p, c_i64, c_p,
                                               ctypes.c_char_p, c_i32]
    lib.sweep_b200_elastic_backward.argtypes = [E, c_i32, c_i32, c_p, c_p, c_p, c_p, c_p, c_p,
                                                c_i64, c_p, ctypes.c_char_p, c_i32]
    E3 = ctypes.POINTER(Elastic3DDesc)
    lib.sweep_b200_elastic3d_sizes.argtypes = [E3, c_i32, c_i32, ctypes.POINTER(c_i64),
                                               ctypes.POINTER(c_i64), ctypes.c_char_p, c_i32]
    lib.sweep_b200_elastic3d_forward.argtypes = [E3, c_i32, c_i32, c_p, c_p, c_p, c_i64, c_p,
                                                 ctypes.c_char_p, c_i32]
    lib.sweep_b200_elastic3d_backward.argtypes = [E3, c_i32, c_i32, c_p, c_p, c_p, c_p, c_p, c_p,
                                                  c_i64, c_p, ctypes.c_char_p, c_i32]
    V = ctypes.POINTER(VTIDesc)
    lib.sweep_b200_vti_sizes.argtypes = [V, c_i32, c_i32, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64),
                                         ctypes.c_char_p, c_i32]
    lib.sweep_b200_vti_forward.argtypes = [V, c_i32, c_i32, c_p, c_p, c_p, c_i64, c_p, ctypes.c_char_p, c_i32]
    lib.sweep_b200_vti_backward.argtypes = [V, c_i32, c_i32, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, c_p,
                                            ctypes.c_char_p, c_i32]
    V3 = ctypes.POINTER(VTI3DDesc)
    lib.sweep_b200_vti3d_sizes.argtypes = [V3, c_i32, c_i32, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64),
                                           ctypes.c_char_p, c_i32]
    lib.sweep_b200_vti3d_forward.argtypes = [V3, c_i32, c_i32, c_p, c_p, c_p, c_i64, c_p, ctypes.c_char_p, c_i32]
    lib.sweep_b200_vti3d_backward.argtypes = [V3, c_i32, c_i32, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, c_p,
                                              ctypes.c_char_p, c_i32]
    lib.sweep_b200_conv3x3_gemm.argtypes = [c_p, c_p, c_p, c_p, c_i32, c_i32, c_i32, c_i32, c_i32, c_i32, c_p,
                                            ctypes.c_char_p, c_i32]
    lib.sweep_b200_conv3x3_wgrad.argtypes = [c_p, c_p, c_p, c_i32, c_i32, c_i32, c_i32, c_i32, c_p,
                                             ctypes.c_char_p, c_i32]
    lib.sweep_b200_conv3x3_status.argtypes = [c_p, ctypes.c_char_p, c_i32]
    S = ctypes.POINTER(Schedule)
    lib.sweep_b200_schedule_set.argtypes = [c_i32, c_p, S, ctypes.c_char_p, c_i32]
    lib.sweep_b200_schedule_get.argtypes = [c_i32, c_p, S, ctypes.c_char_p, c_i32]
    lib.sweep_b200_schedule_clear.argtypes = []
    lib.sweep_b200_wait_selftest.argtypes = [c_i64, c_i32, c_p, ctypes.c_char_p, c_i32]
    H = ctypes.POINTER(c_p)
    lib.sweep_b200_acoustic_forward_runner_create.argtypes = [P, c_i32, c_p, c_p, c_p, c_i64, H, ctypes.c_char_p,
                                                              c_i32]
    lib.sweep_b200_acoustic_backward_runner_create.argtypes = [P, c_i32, c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, H,
                                                               ctypes.c_char_p, c_i32]
    lib.sweep_b200_elastic_forward_runner_create.argtypes = [E, c_i32, c_p, c_p, c_p, c_i64, H, ctypes.c_char_p,
                                                             c_i32]
    lib.sweep_b200_elastic_backward_runner_create.argtypes = [E, c_i32, c_p, c_p, c_p, c_p, c_p, c_p, c_i64, H,
                                                              ctypes.c_char_p, c_i32]
    lib.sweep_b200_forward_runner_run.argtypes = [c_p, c_i32, c_i32, c_i32, c_p, ctypes.c_char_p, c_i32]
    lib.sweep_b200_backward_runner_run.argtypes = [c_p, c_i32, c_i32, c_i32, c_p, ctypes.c_char_p, c_i32]
    lib.sweep_b200_runner_device_index.argtypes = [c_p]
    lib.sweep_b200_runner_destroy.argtypes = [c_p]
    for s in SYMBOLS[1:]:
        getattr(lib, s).restype = ctypes.c_int
    lib.sweep_b200_runner_destroy.restype = None
    _lib = lib
    return lib


def check(rc: int, err) -> None:
    if rc != 0:
        raise RuntimeError("sweep_b200 core: " + err.value.decode(errors="replace"))


def call(name: str, *args) -> None:
    """Call entry ``name`` with the error buffer appended; raise on failure."""
    lib = load()
    err = ctypes.create_string_buffer(ERR_CAP)
    check(getattr(lib, name)(*args, err, ERR_CAP), err)
