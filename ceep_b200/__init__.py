"""ceep_b200 — B200-native batched multistatic FDTD (drop-in for ceep-v1's batched path).

Public API:
    BatchedFDTD2D                      2D TMz batched solver (fdtd_2d_batched.py)
    BatchedFDTD3D                      3D Yee batched solver (fdtd_3d_batched.py)
    FDTD2D (ceep_b200.fdtd2d)          non-batched TMz/TEz solver with CFS-CPML, PEC, Mur (fdtd_2d.py)
    MultistaticSParameters, ImagingRegion, DelayAndSumBeamformer, dft, das_time
The compute runs in ``_lib/libceep_b200.so`` (sm_100a); there is no CPU path.
"""
from .solvers import BatchedFDTD2D
from .solvers3d import BatchedFDTD3D
from .fdtd2d import FDTD2D
from .spectral import (DelayAndSumBeamformer, ImagingRegion, MultistaticSParameters, das_image, das_time,
                       dft)

__all__ = ["BatchedFDTD2D", "BatchedFDTD3D", "FDTD2D", "MultistaticSParameters", "ImagingRegion", "DelayAndSumBeamformer", "dft",
           "das_image", "das_time"]
