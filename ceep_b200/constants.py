"""SI constants with the reference's values (src/ceep/core/constants.py:21-27)."""
import math

C_0 = 299_792_458.0
EPS_0 = 8.854187817e-12
MU_0 = 4.0 * math.pi * 1e-7
ETA_0 = math.sqrt(MU_0 / EPS_0)
# Source amplitude the reference multiplies its waveform by (fdtd_2d_batched.py:177).
SOURCE_AMPLITUDE_SCALE = 1.049e10


def cfl_timestep_2d(dx: float, dy: float, courant: float = 0.5) -> float:
    """constants.py:105-140."""
    return courant * (1.0 / (C_0 * math.sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy))))


def cfl_timestep_3d(dx: float, dy: float, dz: float, courant: float = 0.5) -> float:
    """constants.py:143-175."""
    return courant * (1.0 / (C_0 * math.sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz))))
