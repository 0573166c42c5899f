"""Per-cell boundary rules for boundary="field" scenes.

The reference expresses irregular boundaries as scene code: a scene returns
true from GetExistIrregularBoundaryImpl() and its ProcessGridCellVelocityImpl
(cell, velocity, frame) rewrites the velocity of every grid node with mass
(include/mpm_config.h:108-117, called from include/mpm_algorithm.cuh:795-799).
Here the same rules are data: one rule per grid cell, applied on the device
after gravity (ckmpm_set_boundary_field).  The helpers below build the rules of
the reference scenes' hooks:

* slip_walls: cells within `width` of a domain face lose the velocity component
  along the normalised sum of their faces' inward normals
  (tests/fluid_with_two_longs/test_fluid_with_two_longs.cuh:133-161, the wall part
  of tests/fire_hydrant/test_fire_hydrant.cuh:148-185);
* fixed_box: v = 0 inside a box of cells (the fixed bottom of fire_hydrant);
* rotating_box: v = factor * radius * tangent about an axis through a centre,
  the driven grips of tests/twisting_bar/test_twisting_bar.cuh:126-163;
* sticky_walls: v = 0 within `width` cells of the faces (twisting_bar);
* separate_below: cells below a height keep only velocities with n . v >= 0:
  v_y >= 0 of a slip floor (n = +y), or twisting_bar's "v_y > 0 -> v_y = 0
  below y = 90 cells" (n = -y).

Rules are applied in the order the helpers are called: a later helper
overwrites the cells it covers, so build from the weakest rule to the strongest
(the reference's hooks test their fixed regions first).
"""
from __future__ import annotations

import numpy as np

from . import _capi as capi

FREE, FIXED, SLIP, VELOCITY, SEPARATE = (capi.CELL_FREE, capi.CELL_FIXED, capi.CELL_SLIP, capi.CELL_VELOCITY,
                                         capi.CELL_SEPARATE)


class BoundaryField:
    """rule[Nx, Ny, Nz] (uint8) and param[Nx, Ny, Nz, 3] (float32) over a domain's cells."""

    def __init__(self, config):
        self.dx = float(config.dx)
        self.shape = tuple(4 * int(b) for b in config.domain_blocks)
        self.rule = np.zeros(self.shape, np.uint8)
        self.param = np.zeros(self.shape + (3,), np.float32)

    def cells(self):
        """Integer cell coordinates (cx, cy, cz), each of shape (Nx, Ny, Nz)."""
        return np.meshgrid(*(np.arange(n) for n in self.shape), indexing="ij")

    def box(self, lo, hi) -> tuple[slice, slice, slice]:
        """Cells lo <= c < hi (clipped to the domain)."""
        return tuple(slice(max(0, int(a)), min(n, int(b))) for a, b, n in zip(lo, hi, self.shape))

    def slip_walls(self, width: int = 8) -> "BoundaryField":
        normal = np.zeros(self.shape + (3,), np.float64)
        for a, n in enumerate(self.shape):
            idx = np.arange(n)
            s = np.zeros(n)
            s[idx < width] = 1.0
            s[idx >= n - width] = -1.0
            shape = [1, 1, 1]
            shape[a] = n
            normal[..., a] = s.reshape(shape)
        on = np.any(normal != 0.0, axis=-1)
        # The reference normalises in FP32 (Vector::Norm, then a division).
        nf = normal.astype(np.float32)
        norm = np.sqrt((nf * nf).sum(axis=-1, dtype=np.float32), dtype=np.float32)
        unit = np.zeros_like(nf)
        unit[on] = nf[on] / norm[on, None]
        self.rule[on] = SLIP
        self.param[on] = unit[on]
        return self

    def sticky_walls(self, width: int = 8) -> "BoundaryField":
        cx, cy, cz = self.cells()
        out = np.zeros(self.shape, bool)
        for c, n in zip((cx, cy, cz), self.shape):
            out |= (c < width) | (c >= n - width)
        self.rule[out] = FIXED
        self.param[out] = 0.0
        return self

    def fixed_box(self, lo, hi) -> "BoundaryField":
        b = self.box(lo, hi)
        self.rule[b] = FIXED
        self.param[b] = 0.0
        return self

    def velocity_box(self, lo, hi, velocity) -> "BoundaryField":
        b = self.box(lo, hi)
        self.rule[b] = VELOCITY
        self.param[b] = np.asarray(velocity, np.float32)
        return self

    def rotating_box(self, lo, hi, center, axis, factor: float = 1.0) -> "BoundaryField":
        """v = factor * |r| * unit(axis x r) with r the cell corner (c dx) minus
        the centre, projected off the axis (the twisting_bar grips, whose axis is z)."""
        b = self.box(lo, hi)
        cx, cy, cz = (c[b] for c in self.cells())
        pos = np.stack([cx, cy, cz], -1).astype(np.float64) * self.dx - np.asarray(center, np.float64)
        axis = np.asarray(axis, np.float64)
        axis = axis / np.linalg.norm(axis)
        r = pos - (pos @ axis)[..., None] * axis
        t = np.cross(axis, r)
        tn = np.linalg.norm(t, axis=-1)
        v = np.zeros_like(t)
        ok = tn > 0.0
        v[ok] = factor * np.linalg.norm(r, axis=-1)[ok, None] * t[ok] / tn[ok, None]
        self.rule[b] = VELOCITY
        self.param[b] = v.astype(np.float32)
        return self

    def separate_below(self, cell_y: int, normal=(0.0, 1.0, 0.0)) -> "BoundaryField":
        """Cells with cy < cell_y keep only velocities with normal . v >= 0."""
        b = self.box((0, 0, 0), (self.shape[0], cell_y, self.shape[2]))
        self.rule[b] = SEPARATE
        self.param[b] = np.asarray(normal, np.float32)
        return self

    def arrays(self) -> tuple[np.ndarray, np.ndarray]:
        return self.rule, self.param
