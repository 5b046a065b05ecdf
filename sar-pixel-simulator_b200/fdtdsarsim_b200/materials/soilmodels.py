"""Soil material generators (materials/soilmodels.py).

Each generator yields MaterialModel's of the material block: soil up to a
Gaussian-correlated rough surface (or two correlated surfaces for two
layers), vacuum above, with permittivity and conductivity from the
Hallikainen model at the simulation frequency (conductivity
|eps''| eps0 2 pi f, scipy's eps0). The cells are filled with vectorised
comparisons of each cell's z index against the surface heights rounded to
whole cells; a model has the dtype of the simulation.
"""
from typing import Sequence

import numpy as np
from scipy.constants import epsilon_0

from ..parameters import ParameterCollection
from .dielectricmodels import HallikainenSoilModel, hallikainen_soil_model
from .materialmodel import MaterialModel
from .roughsurface import gaussian_correlated_surface, two_layer_gaussian_correlated_surface

__all__ = ['one_layer_gaussian', 'two_layer_gaussian', 'gradient_gaussian']


def _soil(eps_cplx, freq):
    """(eps_r, sigma) of a complex permittivity at ``freq``."""
    return np.real(eps_cplx), np.abs(np.imag(eps_cplx)) * epsilon_0 * 2.0 * np.pi * freq


def _geometry(params: ParameterCollection, depth: float):
    g = params.geom_params
    nz, dx = g.size_z_material, g.cell_size
    if depth > nz * dx:
        raise ValueError('Requested mean soil depth is greater than the max height of the '
                         'simulator space.')
    return g.size_x, g.size_y, nz, dx, params.processing_params.datatype, \
        params.inc_beam_params.frequency


def _z(nz):
    return np.arange(nz)[:, None, None]


def one_layer_gaussian(params: ParameterCollection, moistures: Sequence[float], sand_frac: float,
                       clay_frac: float, height_rms: float, corr_len: float, mean_depth: float,
                       count: int, seed: int, grooved: bool = False, rabus_compat: bool = False,
                       device: bool = False):
    """One soil layer under a rough surface of mean depth ``mean_depth`` [m]
    (materials/soilmodels.py:16-90): ``count`` surfaces (seeds seed + i),
    each with every moisture in ``moistures``; ``grooved`` repeats the
    surface's first row along y. ``device`` (this package's addition)
    yields LayeredMaterial recipes that the device fills."""
    nx, ny, nz, dx, dtype, freq = _geometry(params, mean_depth)
    mean_cells = mean_depth / dx
    model = HallikainenSoilModel()
    for i in range(count):
        h = gaussian_correlated_surface(nx, ny, dx, corr_len, corr_len, height_rms, seed=seed + i,
                                        rabus_compat=rabus_compat)
        if grooved:
            h = np.repeat(h[0, :][np.newaxis, :], ny, axis=0)
        h /= dx
        h += mean_cells
        h = np.rint(h).astype(np.int32)
        below = _z(nz) <= h[np.newaxis]
        for mv in moistures:
            eps_r, sigma = _soil(model.get_epsilon(mv, sand_frac, clay_frac, freq), freq)
            meta = {'moisture': mv, 'sand_frac': sand_frac, 'clay_frac': clay_frac,
                    'epsilon_r': eps_r, 'conductivity': sigma, 'height_rms': height_rms,
                    'mean_depth': mean_depth, 'mean_depth_cells': mean_cells, 'corr_len': corr_len}
            if device:
                from .device import LayeredMaterial
                yield LayeredMaterial((nz, ny, nx), dx, h[None].astype(np.float64), [eps_r, 1.0],
                                      [sigma, 0.0], f'mv_{mv:.2f}_num_{i}', meta, dtype)
                continue
            eps = np.where(below, eps_r, 1.0).astype(dtype)
            sig = np.where(below, sigma, 0.0).astype(dtype)
            yield MaterialModel(eps, sig, dx, f'mv_{mv:.2f}_num_{i}', meta)


def _two_surfaces(params, nx, ny, dx, corr_len, height_rms, inter_layer_corr, mean_total_depth,
                  top_layer_height, seed, grooved, rabus_compat):
    """Bottom-layer top [0] and soil top [1] in whole cells."""
    h = two_layer_gaussian_correlated_surface(nx, ny, dx, corr_len, corr_len, height_rms,
                                              inter_layer_corr, seed, rabus_compat=rabus_compat)
    if grooved:
        h = np.repeat(h[:, 0, :][:, np.newaxis, :], ny, axis=1)
    h /= dx
    h += mean_total_depth / dx
    h[0] -= top_layer_height / dx
    return np.rint(h).astype(np.int32)


def _check_layers(mean_total_depth, top_layer_height, dx):
    if top_layer_height / dx > mean_total_depth / dx:
        raise ValueError('Top layer of soil is thicker than entire soil model')


def two_layer_gaussian(params: ParameterCollection, top_moisture: float,
                       bottom_moistures: Sequence[float], sand_frac: float, clay_frac: float,
                       height_rms: float, corr_len: float, inter_layer_corr: float,
                       mean_total_depth: float, top_layer_height: float, count: int, seed: int,
                       grooved: bool = False, rabus_compat: bool = False, device: bool = False):
    """Two soil layers of different moisture under two correlated rough
    surfaces (materials/soilmodels.py:93-195); ``device`` (this package's
    addition) yields LayeredMaterial recipes that the device fills."""
    nx, ny, nz, dx, dtype, freq = _geometry(params, mean_total_depth)
    _check_layers(mean_total_depth, top_layer_height, dx)
    model = HallikainenSoilModel()
    eps_top, sig_top = _soil(model.get_epsilon(top_moisture, sand_frac, clay_frac, freq), freq)
    for i in range(count):
        h = _two_surfaces(params, nx, ny, dx, corr_len, height_rms, inter_layer_corr,
                          mean_total_depth, top_layer_height, seed + i, grooved, rabus_compat)
        bottom = _z(nz) <= h[0][np.newaxis]
        top = ~bottom & (_z(nz) <= h[1][np.newaxis])
        for mv in bottom_moistures:
            eps_bot, sig_bot = _soil(model.get_epsilon(mv, sand_frac, clay_frac, freq), freq)
            eps_r = np.asarray([eps_bot, eps_top])
            sigma = np.asarray([sig_bot, sig_top])
            meta = {'top_moisture': top_moisture, 'bottom_moisture': mv, 'sand_frac': sand_frac,
                    'clay_frac': clay_frac, 'epsilon_r': eps_r, 'conductivity': sigma,
                    'height_rms': height_rms, 'mean_total_depth': mean_total_depth,
                    'total_depth_cells': mean_total_depth / dx,
                    'top_layer_height': top_layer_height, 'top_layer_cells': top_layer_height / dx,
                    'inter_layer_corr': inter_layer_corr, 'corr_len': corr_len}
            if device:
                from .device import LayeredMaterial
                yield LayeredMaterial((nz, ny, nx), dx, h.astype(np.float64), [eps_bot, eps_top, 1.0],
                                      [sig_bot, sig_top, 0.0], f'mv_{mv:.2f}_num_{i}', meta, dtype)
                continue
            eps = np.where(bottom, eps_bot, np.where(top, eps_top, 1.0)).astype(dtype)
            sig = np.where(bottom, sig_bot, np.where(top, sig_top, 0.0)).astype(dtype)
            yield MaterialModel(eps, sig, dx, f'mv_{mv:.2f}_num_{i}', meta)


def gradient_gaussian(params: ParameterCollection, top_moisture: float,
                      bottom_moistures: Sequence[float], sand_frac: float, clay_frac: float,
                      height_rms: float, corr_len: float, inter_layer_corr: float,
                      mean_total_depth: float, top_layer_height: float, count: int, seed: int,
                      grooved: bool = False, rabus_compat: bool = False):
    """Two layers as two_layer_gaussian, the top layer's moisture varying
    linearly from the bottom moisture at the lower surface to
    ``top_moisture`` at the upper one (materials/soilmodels.py:198-298)."""
    nx, ny, nz, dx, dtype, freq = _geometry(params, mean_total_depth)
    _check_layers(mean_total_depth, top_layer_height, dx)
    z = _z(nz)
    for i in range(count):
        h = _two_surfaces(params, nx, ny, dx, corr_len, height_rms, inter_layer_corr,
                          mean_total_depth, top_layer_height, seed + i, grooved, rabus_compat)
        h0, h1 = h[0][np.newaxis], h[1][np.newaxis]
        bottom = z <= h0
        top = ~bottom & (z <= h1)
        for mv in bottom_moistures:
            eps_bot, sig_bot = _soil(hallikainen_soil_model(mv, sand_frac, clay_frac, freq), freq)
            eps = np.ones((nz, ny, nx), dtype=dtype)
            sig = np.zeros((nz, ny, nx), dtype=dtype)
            eps[bottom] = eps_bot
            sig[bottom] = sig_bot
            zz, hh0, hh1 = np.broadcast_arrays(z, h0, h1)
            zt, t0, t1 = zz[top], hh0[top], hh1[top]
            sm = ((mv * (t1 - zt)) + (top_moisture * (zt - t0))) / (t1 - t0)
            # the model per distinct moisture (few: one per height pair and plane)
            vals, inv = np.unique(sm, return_inverse=True)
            e_r = np.empty(vals.size)
            s_r = np.empty(vals.size)
            for k, v in enumerate(vals):
                e_r[k], s_r[k] = _soil(hallikainen_soil_model(v, sand_frac, clay_frac, freq), freq)
            eps[top] = e_r[inv]
            sig[top] = s_r[inv]
            meta = {'top_moisture': top_moisture, 'bottom_moisture': mv, 'sand_frac': sand_frac,
                    'clay_frac': clay_frac, 'height_rms': height_rms,
                    'mean_total_depth': mean_total_depth,
                    'total_depth_cells': mean_total_depth / dx,
                    'top_layer_height': top_layer_height, 'top_layer_cells': top_layer_height / dx,
                    'inter_layer_corr': inter_layer_corr, 'corr_len': corr_len}
            yield MaterialModel(eps, sig, dx, f'mv_{mv:.2f}_num_{i}', meta)
