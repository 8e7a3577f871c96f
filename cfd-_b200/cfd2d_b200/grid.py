"""Staggered MAC grid with a ghost layer and the fluid/solid cell flags.

Same indexing and attributes as the reference's ``cfd2d.grid.Grid``
(cfd2d/grid.py:26-158): cells (i, j) with ghosts 0 and nx+1 / ny+1; p-like
fields (nx+2, ny+2), u (nx+1, ny+2), v (nx+2, ny+1); ``fluid`` is a bool
(nx+2, ny+2) array whose ghost frame is False. The flags are set up on the host
once (they are setup data) and uploaded by the simulation.
"""

from __future__ import annotations

import numpy as np
from scipy import ndimage


class Grid:
    """Uniform Cartesian MAC grid with an obstacle mask (cfd2d/grid.py:26-42)."""

    def __init__(self, nx: int, ny: int, lx: float, ly: float):
        if nx < 4 or ny < 4:
            raise ValueError("Das Gitter braucht mindestens 4 Zellen pro Richtung.")
        if lx <= 0 or ly <= 0:
            raise ValueError("Gebietslängen müssen positiv sein.")
        self.nx, self.ny = int(nx), int(ny)
        self.lx, self.ly = float(lx), float(ly)
        self.dx = self.lx / self.nx
        self.dy = self.ly / self.ny
        self.fluid = np.zeros((self.nx + 2, self.ny + 2), dtype=np.bool_)
        self.fluid[1:-1, 1:-1] = True
        self.periodic_x = False

    # coordinates (cfd2d/grid.py:47-69)
    @property
    def xc(self) -> np.ndarray:
        return (np.arange(self.nx) + 0.5) * self.dx

    @property
    def yc(self) -> np.ndarray:
        return (np.arange(self.ny) + 0.5) * self.dy

    @property
    def xn(self) -> np.ndarray:
        return np.arange(self.nx + 1) * self.dx

    @property
    def yn(self) -> np.ndarray:
        return np.arange(self.ny + 1) * self.dy

    def cell_centers(self):
        return np.meshgrid(self.xc, self.yc, indexing="ij")

    # obstacles (cfd2d/grid.py:74-125)
    def interior_solid_padded(self) -> np.ndarray:
        s = ~self.fluid
        s[0, :] = s[-1, :] = s[:, 0] = s[:, -1] = False
        return s

    @property
    def solid(self) -> np.ndarray:
        return ~self.fluid[1:-1, 1:-1]

    @property
    def fluid_interior(self) -> np.ndarray:
        return self.fluid[1:-1, 1:-1]

    def add_obstacle(self, mask) -> None:
        mask = np.asarray(mask, dtype=bool)
        if mask.shape != (self.nx, self.ny):
            raise ValueError(f"Hindernismaske hat Form {mask.shape}, erwartet {(self.nx, self.ny)}")
        self.fluid[1:-1, 1:-1] &= ~mask

    def finalize(self) -> int:
        """Remove fluid regions that do not touch the domain border.

        4-connected regions of the interior fluid cells; with more than one region,
        every region without a cell on the outermost interior ring becomes solid
        (cfd2d/grid.py:100-125). Returns the number of removed cells.
        """
        inner = self.fluid[1:-1, 1:-1]
        lab, nreg = ndimage.label(inner)
        if nreg <= 1:
            return 0
        ring = np.zeros_like(inner)
        ring[0, :] = ring[-1, :] = True
        ring[:, 0] = ring[:, -1] = True
        touching = np.unique(lab[ring & inner])
        touching = touching[touching > 0]
        enclosed = inner & ~np.isin(lab, touching)
        count = int(enclosed.sum())
        if count:
            self.fluid[1:-1, 1:-1] &= ~enclosed
        return count

    def set_periodic_x(self) -> None:
        # ghost columns mirror the opposite columns (cfd2d/grid.py:127-133)
        self.periodic_x = True
        self.fluid[0, :] = self.fluid[self.nx, :]
        self.fluid[self.nx + 1, :] = self.fluid[1, :]
        self.fluid[:, 0] = False
        self.fluid[:, -1] = False

    # face classification (cfd2d/grid.py:138-148)
    def u_fluid_faces(self) -> np.ndarray:
        return self.fluid[:-1, :] & self.fluid[1:, :]

    def v_fluid_faces(self) -> np.ndarray:
        return self.fluid[:, :-1] & self.fluid[:, 1:]

    @property
    def n_fluid(self) -> int:
        return int(self.fluid.sum())

    def __repr__(self) -> str:  # pragma: no cover
        return (f"Grid(nx={self.nx}, ny={self.ny}, lx={self.lx}, ly={self.ly}, dx={self.dx:.4g}, "
                f"dy={self.dy:.4g}, Fluidzellen={self.n_fluid})")
