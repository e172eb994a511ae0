"""cuwave_b200: a B200-native scalar-wave hot path behind cuwave's API.

The scalar (pressure) wave equation's leapfrog step with its PML, source injection and
receiver recording, and the adjoint step with the gradient accumulation, as
hand-written sm_100a kernels in libcuwave_b200.so, driven from Python on torch tensors.
"""

from .boundary import Dirichlet, Neumann, Pml, pml_nodes, pml_profiles, sponge
from .scalar import AcousticWave, PressureWave, ScalarWave
from .signals import ricker
from .stencils import cell_coefficients, stable_dt
from .wave import (
    Simulation,
    Source,
    apply_cell_weights,
    flatten_indices,
    grid_coords,
    padded_shape,
    sensor_cell_weights,
    simulate,
)

__all__ = [
    "AcousticWave",
    "Dirichlet",
    "Neumann",
    "Pml",
    "PressureWave",
    "ScalarWave",
    "Simulation",
    "Source",
    "apply_cell_weights",
    "cell_coefficients",
    "flatten_indices",
    "grid_coords",
    "padded_shape",
    "pml_nodes",
    "pml_profiles",
    "ricker",
    "sensor_cell_weights",
    "simulate",
    "sponge",
    "stable_dt",
]
