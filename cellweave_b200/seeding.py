"""Host-side lattice seeding: how a lattice is laid out before it is swept.

These run once, on the host, before the grid is uploaded; they are setup,
not the per-step path.  Each restates a CpmLattice method of the reference
(crates/engine/src/cpm.rs) on a numpy grid of shape (depth, height, width),
int32, with 0 the medium and -1 the obstacle (u32::MAX in the reference), and
a record table ``Records`` with the medium at id 0.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

OBSTACLE = -1


@dataclass
class Records:
    """Per-cell records indexed by id (CellRecord, cpm.rs:171-181), medium at 0."""

    type: list = field(default_factory=lambda: [0])
    volume: list = field(default_factory=lambda: [0])
    target: list = field(default_factory=lambda: [0])
    lam: list = field(default_factory=lambda: [0.0])

    def push(self, type_, volume, target=None, lam=50.0):
        self.type.append(int(type_))
        self.volume.append(int(volume))
        self.target.append(int(volume if target is None else target))
        self.lam.append(float(lam))
        return len(self.type) - 1

    def __len__(self):
        return len(self.type)

    def arrays(self):
        return (np.array(self.type, np.int32), np.array(self.volume, np.int32), np.array(self.target, np.int32),
                np.array(self.lam, np.float64))


def empty(width: int, height: int, depth: int = 1) -> np.ndarray:
    """CpmLattice::with_depth (cpm.rs:231-259): every pixel medium."""
    for side in (width, height, depth):
        if side == 0 or side > 65535:
            raise ValueError(f"invalid grid dimensions ({width}x{height}x{depth})")
    return np.zeros((depth, height, width), np.int32)


def add_ball(grid: np.ndarray, rec: Records, type_: int, centre, radius: int, lam: float = 50.0) -> int:
    """add_ball (cpm.rs:323-354): every free voxel within `radius` of `centre`."""
    d, h, w = grid.shape
    cx, cy, cz = (int(c) for c in (tuple(centre) + (0,))[:3])
    z, y, x = np.meshgrid(np.arange(d), np.arange(h), np.arange(w), indexing="ij")
    inside = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 <= radius * radius
    take = inside & (grid != OBSTACLE)
    cid = len(rec)
    grid[take] = cid
    return rec.push(type_, int(take.sum()), lam=lam)


def add_cell(grid, rec, type_, centre, radius, lam=50.0):
    """add_cell (cpm.rs:307-317): a disc in the first slice."""
    return add_ball(grid, rec, type_, (centre[0], centre[1], 0), radius, lam)


def add_block(grid: np.ndarray, rec: Records, type_: int, corner, width: int, height: int, lam: float = 50.0,
              z: int = 0, depth: int = 1) -> int:
    """add_block (cpm.rs:361-380): a rectangle (a box with `depth`) of medium pixels, clipped to the grid."""
    d, h, w = grid.shape
    x0, y0 = int(corner[0]), int(corner[1])
    sub = grid[z:min(z + depth, d), y0:min(y0 + height, h), x0:min(x0 + width, w)]
    take = sub == 0
    cid = len(rec)
    sub[take] = cid
    return rec.push(type_, int(take.sum()), lam=lam)


def add_obstacle_disc(grid: np.ndarray, rec: Records, centre, radius: int) -> None:
    """add_obstacle_disc (cpm.rs:389-413): a disc of obstacle through every slice; cells lose what it covers."""
    d, h, w = grid.shape
    cx, cy = int(centre[0]), int(centre[1])
    y, x = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
    disc = (x - cx) ** 2 + (y - cy) ** 2 <= radius * radius
    for zz in range(d):
        sl = grid[zz]
        was = sl[disc]
        for cid in was[(was != 0) & (was != OBSTACLE)]:
            rec.volume[int(cid)] -= 1
        sl[disc] = OBSTACLE


def recount(grid: np.ndarray, ncells: int) -> np.ndarray:
    """Pixel count per id, obstacles skipped (recount, cpm.rs:1262-1270)."""
    g = grid.reshape(-1)
    g = g[(g >= 0) & (g < ncells)]
    return np.bincount(g, minlength=ncells).astype(np.int32)
