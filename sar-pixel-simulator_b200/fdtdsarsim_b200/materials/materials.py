"""Material arrays -> FDTD update coefficients, and the trivial generators.

``compute_material_arrays`` keeps the reference's arithmetic
(materials/materials.py:23-68): vacuum stacked on top of the model, every
operation in the simulation dtype, eps0 hard-coded as 8.8541878128e-12, and
Ca = (1 - s dt / 2e) / (1 + s dt / 2e), Cb = (dt / (e dx)) / (1 + s dt / 2e)
(Taflove eq. 3.31). The device computes the same coefficients from
eps_r/sigma in ``MainSimGpu.run_eps_sigma`` (fdtd_set_materials_eps_sigma).
"""
import numpy as np

from ..parameters import ParameterCollection
from .materialmodel import MaterialModel

EPS0_MATERIALS = 8.8541878128e-12


def compute_material_arrays(params: ParameterCollection, materials: MaterialModel):
    """Return (Ca, Cb), each (size_z, size_y, size_x) in the simulation dtype."""
    g = params.geom_params
    nx, ny, nz, nz_mat = g.size_x, g.size_y, g.size_z, g.size_z_material
    dx, dt = g.cell_size, g.timestep
    dtype = params.processing_params.datatype
    if materials.relative_permittivity.shape != materials.conductivity.shape:
        raise RuntimeError('Permittivity and conductivity arrays have different shapes')
    vac = nz - nz_mat
    perm = np.concatenate((materials.relative_permittivity,
                           np.ones((vac, ny, nx), dtype=dtype)), axis=0, dtype=dtype)
    perm *= EPS0_MATERIALS
    cond = np.concatenate((materials.conductivity,
                           np.zeros((vac, ny, nx), dtype=dtype)), axis=0, dtype=dtype)
    loss = (cond * dt) / (2.0 * perm)
    ca = (1 - loss) / (1 + loss)
    cb = (dt / (perm * dx)) / (1 + loss)
    if ca.dtype != dtype or cb.dtype != dtype:
        raise TypeError('material coefficient arrays lost the simulation dtype')
    return ca, cb


def all_vacuum(params: ParameterCollection):
    """One vacuum model (materials/materials.py:71-86)."""
    g = params.geom_params
    dtype = params.processing_params.datatype
    shape = (g.size_z_material, g.size_y, g.size_x)
    yield MaterialModel(np.ones(shape, dtype=dtype), np.zeros(shape, dtype=dtype),
                        g.cell_size, 'vacuum')


def flat_surface(params: ParameterCollection, epsilon_r: float, conductivity: float,
                 name='planar_surface'):
    """One homogeneous half-space model (materials/materials.py:89-109)."""
    g = params.geom_params
    dtype = params.processing_params.datatype
    shape = (g.size_z_material, g.size_y, g.size_x)
    meta = {'epsilon_r': epsilon_r, 'conductivity': conductivity}
    yield MaterialModel(epsilon_r * np.ones(shape, dtype=dtype),
                        conductivity * np.ones(shape, dtype=dtype), g.cell_size, name, meta)


def rough_dielectric(params: ParameterCollection, epsilon_r: float, conductivity: float,
                     height_rms: float, mean_depth: float, corr_len: float, count: int,
                     seed=None, device=False):
    """``count`` models of one dielectric under a Gaussian-correlated rough
    surface of mean depth ``mean_depth`` [m] (materials/materials.py:
    112-164): a cell is dielectric when its z index is at most the surface
    height in cells. The reference draws unseeded surfaces; ``seed`` (this
    package's addition) makes surface i use seed + i. With ``device`` (this
    package's addition) the models are LayeredMaterial recipes that the
    device fills."""
    from .roughsurface import gaussian_correlated_surface
    g = params.geom_params
    nx, ny, nz, dx = g.size_x, g.size_y, g.size_z_material, g.cell_size
    dtype = params.processing_params.datatype
    mean_cells = mean_depth / dx
    if mean_depth > nz * dx:
        raise ValueError('Requested mean soil depth is greater than the max height of the '
                         'simulator space.')
    meta = {'epsilon_r': epsilon_r, 'conductivity': conductivity, 'height_rms': height_rms,
            'mean_depth': mean_depth, 'mean_depth_cells': mean_cells, 'corr_len': corr_len}
    z = np.arange(nz)[:, None, None]
    for i in range(count):
        h = gaussian_correlated_surface(nx, ny, dx, corr_len, corr_len, height_rms,
                                        seed=None if seed is None else seed + i)
        h /= dx
        h += mean_cells
        if device:
            from .device import LayeredMaterial
            yield LayeredMaterial((nz, ny, nx), dx, h[None], [epsilon_r, 1.0], [conductivity, 0.0],
                                  f'rough_surf_{i}', dict(meta), dtype)
            continue
        below = z <= h[np.newaxis]
        yield MaterialModel(np.where(below, epsilon_r, 1.0).astype(dtype),
                            np.where(below, conductivity, 0.0).astype(dtype), dx,
                            f'rough_surf_{i}', dict(meta))
