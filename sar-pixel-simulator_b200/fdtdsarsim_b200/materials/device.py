"""Material models made on the device.

A ``LayeredMaterial`` is the recipe of a material block rather than its
arrays: interface height maps in cells (lowest first), the eps_r / sigma
of every layer and of the medium above, and lists of spherical inclusions.
``MainSimGpu.run_layered`` (and ``run_experiment`` for such models) has the
device fill the block (fdtd_fill_layers, fdtd_paint_spheres) and make Ca/Cb
from it, so a full-size block never exists on the host nor crosses the bus.
``to_model()`` builds the same arrays on the host.

The recipes are those of the reference's generators
(materials/materials.py:112-164 rough_dielectric, materials/soilmodels.py:
16-195 one- and two-layer soils, materials/bubbles.py:21-199 bubbles): a
cell takes the first layer k with z <= height_k(y, x); a bubble list is the
reference's own sequence of seeded draws and stopping rule, replayed
without the volume (the number of cells a sphere paints depends on its
radius only), so the same seed gives the same block.
"""
import math

import numba
import numpy as np

from .materialmodel import MaterialModel

__all__ = ['LayeredMaterial', 'bubble_spheres']


class LayeredMaterial:
    """Recipe of a (nz_mat, ny, nx) material block: ``heights`` (nlayers,
    ny, nx) in cells, ``eps_layers`` / ``sig_layers`` (nlayers + 1 values,
    the last for the medium above every interface), ``spheres`` a list of
    ((n, 5) arrays of zc, yc, xc, rc, ri in cells, eps_r, sigma)."""

    def __init__(self, shape, cell_size, heights, eps_layers, sig_layers, name, metadata=None,
                 dtype='float32'):
        self.shape = tuple(int(v) for v in shape)
        nz, ny, nx = self.shape
        self.heights = np.asarray(heights, dtype=np.float64).reshape(-1, ny, nx)
        self.eps_layers = np.asarray(eps_layers, dtype=np.float64)
        self.sig_layers = np.asarray(sig_layers, dtype=np.float64)
        if self.eps_layers.shape != (self.heights.shape[0] + 1,) or \
                self.sig_layers.shape != self.eps_layers.shape:
            raise ValueError('one eps_r / sigma value per layer and one for the medium above')
        self.cell_size = cell_size
        self.name = name
        self.metadata = metadata
        self.dtype = np.dtype(dtype)
        self.spheres = []

    def _layer_index(self):
        nz = self.shape[0]
        z = np.arange(nz)[:, None, None]
        idx = np.full(self.shape, self.heights.shape[0], np.int32)
        for k in range(self.heights.shape[0] - 1, -1, -1):   # the first k with z <= h_k wins
            idx = np.where(z <= self.heights[k][None], k, idx)
        return idx

    def to_model(self):
        """The block's arrays on the host (MaterialModel)."""
        idx = self._layer_index()
        eps = self.eps_layers[idx].astype(self.dtype)
        sig = self.sig_layers[idx].astype(self.dtype)
        for sp, e, s in self.spheres:
            _paint_list(eps, sig, np.asarray(sp, np.float64), self.dtype.type(e), self.dtype.type(s))
        return MaterialModel(eps, sig, self.cell_size, self.name, self.metadata)

    def material_volume(self):
        """Cells that are not vacuum before any sphere is painted, counted
        from the heights (what bubbles.material_volume counts on arrays)."""
        nz = self.shape[0]
        cast = self.dtype.type
        nonvac = [cast(e) != 1.0 or cast(s) != 0.0 for e, s in zip(self.eps_layers, self.sig_layers)]

        def below(h):   # cells z in [0, nz) with z <= h, per column
            return np.clip(np.floor(h) + 1.0, 0, nz)

        total = 0
        hmax = np.full(self.shape[1:], -np.inf)
        for k in range(self.heights.shape[0]):
            cnt = np.maximum(0.0, below(self.heights[k]) - below(hmax))
            if nonvac[k]:
                total += int(cnt.sum())
            hmax = np.maximum(hmax, self.heights[k])
        if nonvac[-1]:
            total += int((nz - below(hmax)).sum())
        return total

    def stage(self, native):
        """Fill the block into a NativeSim's staging buffers on the device."""
        native.fill_layers(self.shape[0], self.heights, self.eps_layers, self.sig_layers)
        for sp, e, s in self.spheres:
            native.paint_spheres(sp, e, s)


@numba.njit(cache=False, nogil=True)
def _draw(surf, rng, target, vol, r_min, r_max, fixed_radius, cell, nz, ny, nx):
    out = np.empty((64, 5))
    n = 0
    while vol > target:
        if fixed_radius:
            rc = r_min / cell
            ri = int(math.ceil(rc))
        else:
            rc = rng.uniform(r_min, r_max) / cell
            ri = int(np.rint(rc))
        zc = rng.uniform(ri, nz - ri - 1)
        yc = rng.uniform(ri, ny - ri - 1)
        xc = rng.uniform(ri, nx - ri - 1)
        if np.rint(zc + ri) > surf[int(np.rint(yc)), int(np.rint(xc))]:
            continue   # the bubble would reach above the surface
        cnt = 0
        for dz in range(-ri, ri + 1):
            for dy in range(-ri, ri + 1):
                for dx in range(-ri, ri + 1):
                    if dz * dz + dy * dy + dx * dx < rc * rc:
                        cnt += 1
        if n == out.shape[0]:
            grown = np.empty((2 * n, 5))
            grown[:n] = out
            out = grown
        out[n, 0] = zc
        out[n, 1] = yc
        out[n, 2] = xc
        out[n, 3] = rc
        out[n, 4] = ri
        n += 1
        vol -= cnt
    return out[:n]


@numba.njit(cache=False, nogil=True)
def _paint_list(eps, cond, sp, eps_b, cond_b):
    for k in range(sp.shape[0]):
        zc, yc, xc, rc = sp[k, 0], sp[k, 1], sp[k, 2], sp[k, 3]
        ri = int(sp[k, 4])
        for dz in range(-ri, ri + 1):
            for dy in range(-ri, ri + 1):
                for dx in range(-ri, ri + 1):
                    if dz * dz + dy * dy + dx * dx < rc * rc:
                        z = int(np.rint(zc + dz))
                        y = int(np.rint(yc + dy))
                        x = int(np.rint(xc + dx))
                        eps[z, y, x] = eps_b
                        cond[z, y, x] = cond_b


def bubble_spheres(shape, vol, surf_height_cells, bubble_frac, r_min, r_max, fixed, cell, seed):
    """The spheres bubbles._fill paints for a block of ``shape`` with ``vol``
    material cells: the same draws from default_rng(seed), in order, with
    the same stopping rule; (n, 5) rows of zc, yc, xc, rc, ri in cells."""
    rng = np.random.default_rng(seed=seed)
    target = int(round(vol * (1.0 - bubble_frac)))
    nz, ny, nx = shape
    return _draw(np.asarray(surf_height_cells, dtype=np.float64), rng, target, int(vol), float(r_min),
                 float(r_max), bool(fixed), float(cell), nz, ny, nx)
