"""xrecon_b200 -- B200-native distance-driven CT projector.

Drop-in for the projector path of XRecon: ``Projector2d`` / ``Projector3d``
with projection, backprojection, weighted backprojection, their transposes
and filtered backprojection (FBP / FDK) for parallel, fan/cone-flat and
fan/cone-arc geometries, and ``HelicalProjector3d`` (helical arc-detector
scans with per-view source offsets, helical FDK), on hand-written sm_100a
CUDA kernels behind the C ABI of ``include/xrecon_b200.h``.
``xrecon_b200.backend`` replaces the native module ``xrecon_C``;
``xrecon_b200.rebin`` has the fan/helical -> parallel rebinning.
"""
from .geometry import (ConeBeam3d, Detector2d, Detector3d, FanBeam2d, HelicalConeBeam3d, ParallelBeam2d,
                       ParallelBeam3d, Volume2d, Volume3d)
from .phantom import phantom
from .projector import HelicalProjector3d, Projector2d, Projector3d, projector2d, projector3d

__version__ = "0.1.0"

__all__ = [
    "Detector2d", "Detector3d", "FanBeam2d", "ConeBeam3d", "HelicalConeBeam3d", "HelicalProjector3d",
    "ParallelBeam2d",
    "ParallelBeam3d", "Projector2d", "Projector3d", "Volume2d", "Volume3d", "projector2d", "projector3d",
    "phantom",
]
