"""Finite-difference coefficient tables of the cell-flux Laplacian.

The step forms, per axis, two cell differences

    D+ = sum_k w_k (u[a+k] - u[a+1-k]),   D- = sum_k w_k (u[a+k-1] - u[a-k]),

and the kernels take the row `w_1 .. w_R` of the full radius `R` as a runtime table
(`cwb_grid.coeffs`), so one build serves every order and both stencils.

Restated from cuwave `stencils.py:11-58` (`weights`, `cell_coefficients`, `_band_fit`)
and `wave.py:44-54` (`stable_dt`); the tables have to agree with the reference's to
the last float32 bit, since both feed the same recursion.
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np

STENCILS = ("taylor", "optimized")
# phase-velocity error a fitted row keeps over its band (cuwave stencils.py:8)
DISPERSION_TOL = 1e-3


def second_derivative_weights(radius: int) -> np.ndarray:
    """Central weights `w[-R..R]` of the order-2R second derivative (cuwave stencils.py:11-17).

    Solved from the moment conditions sum_j w_j j^p = 2 [p == 2], p = 0 .. 2R.
    """
    offsets = np.arange(-radius, radius + 1)
    moments = offsets[None, :] ** np.arange(2 * radius + 1)[:, None]
    target = np.zeros(2 * radius + 1)
    target[2] = 2.0
    return np.linalg.solve(moments, target)


@lru_cache
def _dispersion_fit(radius: int) -> np.ndarray:
    """Least-squares cell weights over the widest band meeting `DISPERSION_TOL`.

    The fitted row keeps the consistency constraint sum_k (2k - 1) w_k = 1 and matches
    the symbol of the cell flux to the exact one over [0, band], with the band shrunk
    from pi in 400 steps until the phase error stays under the tolerance
    (cuwave stencils.py:40-58, `_band_fit` with staggered=False).
    """
    k = np.arange(1, radius + 1)
    for band in np.linspace(np.pi, 0.0, 400, endpoint=False):
        theta = np.linspace(band / 400, band, 400)
        symbol = 2.0 * np.sin(np.outer(theta, k - 0.5)) / theta[:, None]
        symbol *= 2.0 * np.sin(theta / 2.0)[:, None] / theta[:, None]
        consistency = (2 * k - 1.0)[None]
        system = np.block(
            [[symbol.T @ symbol, consistency.T], [consistency, np.zeros((1, 1))]]
        )
        coef = np.linalg.solve(system, np.append(symbol.sum(axis=0), 1.0))[:radius]
        ratio = symbol @ coef
        if np.abs(np.sqrt(ratio) - 1.0).max() <= DISPERSION_TOL:
            return coef
    raise ValueError(f"no band meets the dispersion tolerance at radius {radius}")


def cell_coefficients(radius: int, stencil: str = "taylor") -> np.ndarray:
    """The cell-flux weights `w_1 .. w_R` (float64) of one radius (cuwave stencils.py:20-25).

    "taylor" takes the tail sums of the central second-derivative weights;
    "optimized" takes the dispersion fit.
    """
    if stencil not in STENCILS:
        raise ValueError(f"unknown stencil {stencil!r}, expected one of {STENCILS}")
    if stencil != "taylor":
        return _dispersion_fit(radius)
    w = second_derivative_weights(radius)
    return np.array([w[radius + 1 + k :].sum() for k in range(radius)])


def operator_row(space_order: int, stencil: str = "optimized") -> np.ndarray:
    """The full-radius row the step kernels read, `OP_W(R, 1..R)` of cuwave common.cuh:26-35.

    The reference bakes the double table of `stencils.preamble` (stencils.py:186-213)
    into a float `__constant__`, i.e. rounds each double to nearest float; this does
    the same through numpy. Rows below R only serve masked domains.
    """
    radius = space_order // 2
    return cell_coefficients(radius, stencil)


def cell_table(space_order: int, stencil: str = "optimized") -> np.ndarray:
    """(R, R) float64: row r - 1 holds OP_W(r, 1..r), the rows below R Taylor and row R
    `stencil`, zero past r (cuwave stencils.py:186-196). A masked domain grades the cells
    by its walls down these rows."""
    radius = space_order // 2
    table = np.zeros((radius, radius))
    for r in range(1, radius + 1):
        table[r - 1, :r] = cell_coefficients(r, stencil if r == radius else "taylor")
    if radius == 1:
        table[0, 0] = 1.0  # the operator weight is the literal 1 at radius 1
    return table


def stable_dt(
    dx: tuple[float, ...],
    wavespeed: float,
    space_order: int = 2,
    stencil: str = "optimized",
) -> float:
    """CFL-stable timestep: 2 / (c sqrt(lambda sum 1/dx^2)) (cuwave wave.py:44-54).

    lambda = 4 |sum_k w_k (-1)^k| is the flux symbol at the grid's Nyquist mode.
    """
    c = cell_coefficients(space_order // 2, stencil)
    lam = 4.0 * abs(float(c @ (-1.0) ** np.arange(len(c))))
    return 2.0 / (wavespeed * float(np.sqrt(lam * sum(1.0 / d**2 for d in dx))))
