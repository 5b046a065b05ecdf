"""Spherical inclusions ("bubbles") in a material model (materials/bubbles.py).

Bubbles are placed one at a time at uniformly random centres, rejected when
the bubble would reach above the soil surface, and painted cell by cell
until the painted-cell count has removed the requested fraction of the
material volume (every painted cell counts, also one painted twice). The
placement draws from ``numpy.random.default_rng(seed)`` in the reference's
order (radius first for random sizes, then z, y, x), so a seed gives the
reference's model; the sequential draw is why this stays a host loop
(compiled with numba).
"""
import math

import numba
import numpy as np

from .materialmodel import MaterialModel

__all__ = ['material_volume', 'add_bubbles', 'add_bubbles_randsize']


def material_volume(rel_permittivity, conductivity):
    """Cells that are not vacuum."""
    return np.sum(np.logical_or(rel_permittivity != 1.0, conductivity != 0.0))


@numba.njit(cache=False, nogil=True)
def _paint(eps, cond, surf, rng, target, vol, r_min, r_max, fixed_radius, cell, eps_b, cond_b):
    nz, ny, nx = eps.shape
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
        for dz in range(-ri, ri + 1):
            for dy in range(-ri, ri + 1):
                for dx in range(-ri, ri + 1):
                    if dz * dz + dy * dy + dx * dx < rc * rc:
                        z = int(np.rint(zc + dz))
                        y = int(np.rint(yc + dy))
                        x = int(np.rint(xc + dx))
                        eps[z, y, x] = eps_b
                        cond[z, y, x] = cond_b
                        vol -= 1
    return vol


def _fill(mat_model, surf_height_cells, bubble_frac, r_min, r_max, fixed, eps_b, cond_b, seed):
    from .device import LayeredMaterial, bubble_spheres
    if isinstance(mat_model, LayeredMaterial):
        # a recipe made on the device: the same draws as a sphere list
        vol = mat_model.material_volume() if not mat_model.spheres else \
            int(material_volume(*_arrays(mat_model.to_model())))
        sp = bubble_spheres(mat_model.shape, vol, surf_height_cells, bubble_frac, r_min, r_max, fixed,
                            mat_model.cell_size, seed)
        mat_model.spheres.append((sp, eps_b, cond_b))
        return
    rng = np.random.default_rng(seed=seed)
    vol = int(material_volume(mat_model.relative_permittivity, mat_model.conductivity))
    target = int(round(vol * (1.0 - bubble_frac)))
    _paint(mat_model.relative_permittivity, mat_model.conductivity,
           np.asarray(surf_height_cells, dtype=np.float64), rng, target, vol, float(r_min),
           float(r_max), fixed, float(mat_model.cell_size), eps_b, cond_b)


def _arrays(model):
    return model.relative_permittivity, model.conductivity


def add_bubbles(mat_model: MaterialModel, surf_height_cells: np.ndarray, bubble_frac: float,
                bubble_radius: float, bubble_eps_r: float, bubble_cond: float, seed: int):
    """Bubbles of radius ``bubble_radius`` [m] until ``bubble_frac`` of the
    material volume is bubble (materials/bubbles.py:21-105); the model is
    changed in place, its metadata extended, and returned."""
    out = mat_model
    if out.metadata is None:
        out.metadata = {}
    out.metadata['bubble_frac'] = bubble_frac
    out.metadata['bubble_radius'] = bubble_radius
    out.metadata['bubble_radius_cells'] = bubble_radius / out.cell_size
    out.metadata['bubble_eps_r'] = bubble_eps_r
    out.metadata['bubble_cond'] = bubble_cond
    _fill(out, surf_height_cells, bubble_frac, bubble_radius, bubble_radius, True, bubble_eps_r,
          bubble_cond, seed)
    return out


def add_bubbles_randsize(mat_model: MaterialModel, surf_height_cells: np.ndarray,
                         bubble_frac: float, bubble_radius_min: float, bubble_radius_max: float,
                         bubble_eps_r: float, bubble_cond: float, seed: int):
    """As add_bubbles with each radius uniform in [min, max) [m]
    (materials/bubbles.py:108-199)."""
    out = mat_model
    if out.metadata is None:
        out.metadata = {}
    out.metadata['bubble_frac'] = bubble_frac
    out.metadata['bubble_radius_min'] = bubble_radius_min
    out.metadata['bubble_radius_max'] = bubble_radius_max
    out.metadata['bubble_eps_r'] = bubble_eps_r
    out.metadata['bubble_cond'] = bubble_cond
    _fill(out, surf_height_cells, bubble_frac, bubble_radius_min, bubble_radius_max, False,
          bubble_eps_r, bubble_cond, seed)
    return out
