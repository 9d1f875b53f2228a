"""Memory strategies of the backward, with the reference's spellings
(``src/sweep/propagator/options.py:186-246``: ``Full``, ``BoundarySaving``,
``Ckpt``; defaults ``chunks=100``)."""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class BoundarySaving:
    """Save the (M+1)-wide boundary strips of the physical box every step on
    the GPU and rebuild the forward field backwards from them (the impl='c'
    default)."""
    storage: str = "gpu"

    def __post_init__(self):
        if self.storage != "gpu":
            raise NotImplementedError("sweep_b200 keeps the boundary ring in GPU memory only "
                                      "(storage='gpu')")


@dataclass(frozen=True)
class Full:
    """Keep what the backward needs for every step.  The gradient equals the
    boundary-saving one (the reference holds its memory modes to agree); on
    this core it is computed by the boundary-saving backward, which needs a
    fraction of the memory and no extra passes."""


@dataclass(frozen=True)
class Ckpt:
    """Checkpoint the forward state every ``chunks`` steps and re-run each
    chunk during the backward."""
    chunks: int = 100
    mode: str = "chunk"

    def __post_init__(self):
        if int(self.chunks) < 1:
            raise ValueError("Ckpt(chunks) must be >= 1")
        if self.mode != "chunk":
            raise NotImplementedError("sweep_b200 implements chunked checkpointing (mode='chunk')")
