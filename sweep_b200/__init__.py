"""sweep_b200: the B200-native finite-difference hot path of SWEEP's
``PropTorch(..., impl='c')`` -- 2-D/3-D acoustic and 2-D elastic propagation
with adjoint gradients, on hand-written sm_100a CUDA kernels behind a C ABI
(``include/sweep_b200.h``)."""
from . import autotune
from .equations import Acoustic, Acoustic3D, AcousticVTI1st, AcousticVTI1st3D, Elastic, Elastic3D
from .options import BoundarySaving, Ckpt, Full
from .propagator import PropTorch
from .signal import ricker

__all__ = ["autotune", "Acoustic", "Acoustic3D", "AcousticVTI1st", "AcousticVTI1st3D", "Elastic", "Elastic3D", "BoundarySaving", "Ckpt", "Full", "PropTorch", "ricker"]
