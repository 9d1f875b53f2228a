"""Memory strategies of the backward, with the reference's spellings
(``src/sweep/propagator/options.py:186-246``: ``Full``, ``BoundarySaving``,
``Ckpt``; defaults ``chunks=100``)."""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class BoundarySaving:
    """Save the (M+1)-wide boundary strips of the physical box every step on
    the GPU and rebuild the forward field backwards from them (the impl='c'
    default).

    ``storage_dtype`` (reference ``options.py:194-212``) sets how the saved
    strips are held; compute stays FP32:

    * ``'fp32'``: 4 bytes per cell, exact;
    * ``'bf16'``: 2 bytes per cell, each value rounded to bfloat16;
    * ``'fp16'``: 2 bytes per cell plus one FP32 scale per 256 cells: each
      face of the strip set is normalised per shot, block by block, by the
      block's max |value| before rounding to fp16 (safe at any amplitude);
    * ``'int8'``: 1 byte per cell plus the same scales: symmetric 8-bit codes
      of the normalised values.

    Every equation takes every format (Elastic quantises each of its five
    fields on its own).

    ``storage='cpu'`` (reference ``options.py:186-192``) keeps the tape in
    pinned host memory: the step kernels write a small device ring and a copy
    stream moves each step's strips to the host (forward) and back ahead of
    their use (backward), so the tape no longer takes GPU memory (every
    equation).

    ``budget_gb`` (no counterpart in the reference) bounds the tape of one
    call: a call whose boundary-saving tape would exceed it checkpoints the
    state every ``ckpt_chunks`` steps instead (``Ckpt(chunks=ckpt_chunks)``);
    ``PropTorch.last_memory`` reports which one the last call ran."""
    storage: str = "gpu"
    storage_dtype: str = "fp32"
    budget_gb: float | None = None
    ckpt_chunks: int = 100

    def __post_init__(self):
        if self.budget_gb is not None and not float(self.budget_gb) > 0:
            raise ValueError("BoundarySaving.budget_gb must be a positive number of GB (or None)")
        if int(self.ckpt_chunks) < 1:
            raise ValueError("BoundarySaving.ckpt_chunks must be >= 1")
        if self.storage not in ("gpu", "cpu"):
            raise NotImplementedError("sweep_b200 keeps the boundary strips in GPU memory (storage='gpu') or "
                                      "in pinned host memory (storage='cpu'); disk storage is not built")
        if self.storage_dtype not in ("fp32", "fp16", "bf16", "int8"):
            raise ValueError("BoundarySaving.storage_dtype must be 'fp32', 'fp16', 'bf16', or 'int8'.")


@dataclass(frozen=True)
class Full:
    """Keep what the backward needs for every step.  The gradient equals the
    boundary-saving one (the reference holds its memory modes to agree); on
    this core it is computed by the boundary-saving backward, which needs a
    fraction of the memory and no extra passes."""


@dataclass(frozen=True)
class Ckpt:
    """Checkpointing, the reference's two modes (``options.py:346-370``):

    * ``mode='chunk'`` (default): checkpoint the forward state every
      ``chunks`` steps and re-run each chunk during the backward;
    * ``mode='recursive'``: keep nothing from the forward; the backward
      bisects the time axis holding at most ``count`` forward states at once,
      replays each 64-step leaf from the nearest one and reverses it (the
      gradient equals ``Ckpt(chunks=64)``'s; memory is ``count`` states
      instead of ``nt / chunks``, at the price of more replayed steps)."""
    chunks: int = 100
    mode: str = "chunk"
    count: int = 0

    def __post_init__(self):
        if self.mode == "chunk":
            if int(self.chunks) < 1:
                raise ValueError("Ckpt(chunks) must be >= 1")
            if int(self.count) != 0:
                raise ValueError("Ckpt.count is only valid when mode='recursive'.")
        elif self.mode == "recursive":
            if int(self.count) < 1:
                raise ValueError("Ckpt.count must be >= 1 when mode='recursive'.")
            if int(self.chunks) != 100:
                raise ValueError("Ckpt.chunks is only valid when mode='chunk'.")
        else:
            raise ValueError("Ckpt.mode must be 'chunk' or 'recursive'.")
