"""The 2D periodic cell, mirroring the reference's ``Grid(Δx, Δy, Nx, Ny)``
(``lib/DielectricSmoothing/src/grid.jl:46-76``)."""

from __future__ import annotations

import dataclasses

import numpy as np

from . import _lib


@dataclasses.dataclass(frozen=True)
class Grid:
    """Dx × Dy μm cell on Nx × Ny pixels; pixel centres ``x_i = -Δx/2 + (i-1)Δx/Nx``."""

    Dx: float
    Dy: float
    Nx: int
    Ny: int

    @property
    def N(self) -> int:
        return self.Nx * self.Ny

    def x(self) -> np.ndarray:
        return -self.Dx / 2 + np.arange(self.Nx) * (self.Dx / self.Nx)

    def y(self) -> np.ndarray:
        return -self.Dy / 2 + np.arange(self.Ny) * (self.Dy / self.Ny)

    def c(self) -> "_lib.c_grid":
        return _lib.c_grid(int(self.Nx), int(self.Ny), float(self.Dx), float(self.Dy))
