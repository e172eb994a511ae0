"""Scalar pressure wave equations: `PressureWave`, `ScalarWave`, `AcousticWave`.

The hooks the drivers call, restated from cuwave `scalar.py:140-950`: materials from
the design field (`build_materials`, `parametrization`), the per-axis step factors, the
source factor and excitation weights, and the native material block the kernels read.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _native as nat
from .stencils import cell_table
from .wave import (
    Simulation,
    apply_cell_weights,
    as_device,
    domain_cells,
    mirror_ghosts,
    sensor_cell_weights,
)


@dataclass
class PressureWave(Simulation):
    """Scalar wave equation base: nodal `stiff` / `minv` fields, optional damping (cuwave scalar.py:140-872)."""

    gradient_names = ("mass", "stiff")
    fuses_adjoint = True

    # ---------------------------------------------------------------- materials
    def build_materials(self, indicator) -> dict:
        """`indicator` to the material dict, ghosts mirrored (cuwave scalar.py:407-415).

        As in the reference, a ScalarWave's stiffness is the caller's indicator itself
        when it is already a device tensor of the simulation's dtype, so its ghost ring
        is overwritten in place.
        """
        indicator = self._indicator(indicator)
        stiff, minv = self.parametrization(indicator)
        mat = {"stiff": mirror_ghosts(self, stiff)}
        mat["minv"] = None if minv is None else mirror_ghosts(self, minv)
        mat["damping"] = None if self.damping is None else as_device(self.damping, self.dtype)
        mat["profiles"] = [None] * 3
        for d, lo, hi, profile in self.pml_slabs():
            mat["profiles"][d] = torch.as_tensor(profile, device=stiff.device)
        logical = stiff[tuple(slice(0, n) for n in self.Nx)]
        first = logical.reshape(-1)[0]
        mat["uniform"] = bool((logical == first).all())
        mat["stiff_value"] = float(first)
        mat["cells"] = mat["cell_table"] = None
        if self.masked:
            mat["cells"] = domain_cells(self)
            table = cell_table(self.space_order, self.stencil).astype(self.np_dtype)
            mat["cell_table"] = torch.as_tensor(table, device=stiff.device)
        return mat

    def _indicator(self, indicator) -> torch.Tensor:
        if isinstance(indicator, torch.Tensor) and indicator.is_cuda and indicator.dtype == self.dtype:
            if tuple(indicator.shape) != self.Nx_padded:
                raise ValueError(f"indicator shape {tuple(indicator.shape)} != {self.Nx_padded}")
            return indicator
        out = as_device(indicator, self.dtype)
        if tuple(out.shape) != self.Nx_padded:
            raise ValueError(f"indicator shape {tuple(out.shape)} != {self.Nx_padded}")
        return out

    def inverse_inertia(self, indicator) -> torch.Tensor:
        stiff, minv = self.parametrization(self._indicator(indicator))
        return 1.0 / stiff if minv is None else minv

    def material(self, mat: dict) -> nat.Material:
        """The native material block of `mat`."""
        m = nat.Material()
        m.stiff = mat["stiff"].data_ptr()
        m.minv = None if mat["minv"] is None else mat["minv"].data_ptr()
        m.damping = None if mat["damping"] is None else mat["damping"].data_ptr()
        for d in range(3):
            prof = mat["profiles"][d]
            m.profile[d] = None if prof is None else prof.data_ptr()
        m.derive_inertia = int(self.derive_inertia)
        m.stiff_uniform = int(mat["uniform"])
        m.stiff_value = mat["stiff_value"]
        if mat.get("cells") is not None:
            m.cells = mat["cells"].data_ptr()
            m.cell_table = mat["cell_table"].data_ptr()
        return m

    def excitation_weights(self, mat: dict, lin_index: torch.Tensor) -> torch.Tensor:
        """dt^2 source_factor / m at `lin_index`, over 1 + beta when damped (cuwave scalar.py:858-872)."""
        field = mat["stiff"] if self.derive_inertia else mat["minv"]
        weight = field.reshape(-1)[lin_index.long()]
        if self.derive_inertia:
            weight = 1.0 / weight
        if mat["damping"] is not None:
            beta = 0.5 * weight * mat["damping"].reshape(-1)[lin_index.long()] * self.dt
            weight = weight / (1.0 + beta)
        scale = torch.tensor(self.np_dtype(self.dt**2 * self.source_factor()), device=weight.device)
        return (scale * weight).to(self.dtype).contiguous()

    def adjoint_weights(self, sensors: torch.Tensor) -> torch.Tensor:
        """W times the source factor: what the adjoint source is divided by (cuwave scalar.py:758-760)."""
        return sensor_cell_weights(self, sensors) * self.source_factor()

    def gradient_fields(self, mat: dict) -> dict:
        return {
            name: torch.zeros(self.Nx_padded, dtype=self.dtype, device=mat["stiff"].device)
            for name in self.gradient_names
        }

    def finalize_gradients(self, grads: dict) -> dict:
        """Weight the accumulators by W (cuwave scalar.py:762-766)."""
        for f in grads.values():
            apply_cell_weights(self, f)
        return grads


@dataclass
class ScalarWave(PressureWave):
    """Constant-speed scalar wave, gamma scaling density (cuwave scalar.py:875-908)."""

    wavespeed: float = None
    density: float = None

    derive_inertia = True

    def __post_init__(self) -> None:
        super().__post_init__()
        if self.wavespeed is None or self.density is None:
            raise ValueError("ScalarWave requires wavespeed and density")

    def parametrization(self, indicator):
        return indicator, None

    def parametrization_jacobian(self, indicator=None) -> tuple:
        return 1.0, 1.0

    def step_factors(self) -> list:
        """2 c0^2 dt^2 / dx^2 per axis."""
        return [self.np_dtype(2.0 * self.wavespeed**2 * self.dt**2 / d**2) for d in self.dx]

    def source_factor(self) -> float:
        return 1.0 / self.density


@dataclass
class AcousticWave(PressureWave):
    """Two-phase acoustic wave, gamma interpolating 1/rho and 1/kappa (cuwave scalar.py:911-950).

    A velocity field c enters as rho1 = rho2 = 1, kappa1 = 1 and an indicator with
    1/kappa = 1/c^2, so that stiff = 1 and minv = c^2.
    """

    rho1: float = None
    rho2: float = None
    kappa1: float = None
    kappa2: float = None

    def __post_init__(self) -> None:
        super().__post_init__()
        if None in (self.rho1, self.rho2, self.kappa1, self.kappa2):
            raise ValueError("AcousticWave requires rho1, rho2, kappa1, kappa2")

    def parametrization(self, indicator):
        """1/rho and kappa from gamma, in the indicator's precision (cuwave scalar.py:927-934)."""
        rho_inv = 1 / self.rho1 + indicator * (1 / self.rho2 - 1 / self.rho1)
        kappa_inv = 1 / self.kappa1 + indicator * (1 / self.kappa2 - 1 / self.kappa1)
        return rho_inv, 1 / kappa_inv

    def parametrization_jacobian(self, indicator=None) -> tuple:
        """d(mass, stiff)/d gamma: both affine in gamma (cuwave scalar.py:936-942)."""
        return (1 / self.kappa2 - 1 / self.kappa1, 1 / self.rho2 - 1 / self.rho1)

    def step_factors(self) -> list:
        """2 dt^2 / dx^2 per axis."""
        return [self.np_dtype(2.0 * self.dt**2 / d**2) for d in self.dx]

    def source_factor(self) -> float:
        return 1.0

    @staticmethod
    def indicator_for_speed(c, kappa2: float):
        """The design field that makes minv = c^2 with rho1 = rho2 = kappa1 = 1."""
        c = np.asarray(c, dtype=np.float64)
        return (1.0 / c**2 - 1.0) / (1.0 / kappa2 - 1.0)
