"""photonoxide_b200: a B200-native engine for photonoxide's FDTD time step."""
from .types import (ALL_AXES, Axis, Boundaries, Boxes, Cpml, Current, Dipole, Dispersive, Field,  # noqa: F401
                    FluxPlane, GpuError, Grid3d, InvalidValue, Periodic, Pml, Pole, Source,
                    Waveform)
