"""Rough surfaces with a Gaussian autocorrelation (materials/roughsurface.py).

A surface is white noise filtered by the Gaussian kernel
exp(-(x^2 / lx^2 + y^2 / ly^2)) sampled on 6 correlation lengths, then
shifted to zero mean and scaled to the requested rms height. The noise
comes from ``numpy.random.default_rng(seed)`` in the order the reference
draws it, so a seed gives the reference's surface. With ``rabus_compat``
the correlation lengths are divided by sqrt(2) (the convention of Rabus,
Wehn and Nolan, "The Importance of Soil Moisture and Soil Structure for
InSAR Phase and Backscatter, as Determined by FDTD Modeling").
"""
import logging

import numpy as np
import scipy.signal

logger = logging.getLogger(__name__)

__all__ = ['gaussian_correlated_surface', 'gaussian_correlated_surface_fast',
           'two_layer_gaussian_correlated_surface', 'correlate_layers']


def _kernel_samples(corr_len, dx):
    """Sample positions of the kernel along one axis: 6 correlation lengths
    (rounded to whole cells), centred as arange(-(n // 2) - (n % 2), n // 2)."""
    n = int(6.0 * round(corr_len / dx))
    return np.arange(-n // 2, n // 2) * dx, n


def _gaussian_kernel(corr_x, corr_y, dx):
    kx, nx_k = _kernel_samples(corr_x, dx)
    ky, ny_k = _kernel_samples(corr_y, dx)
    xx, yy = np.meshgrid(kx, ky)
    return np.exp(-(xx ** 2 / corr_x ** 2 + yy ** 2 / corr_y ** 2)), nx_k, ny_k


def _zero_mean_rms(h, height_rms):
    out = h - np.mean(h)
    out /= np.std(out)
    out *= height_rms
    return out


def gaussian_correlated_surface(nx, ny, dx, corr_len_x, corr_len_y, height_rms, seed=None,
                                rabus_compat=False, debug_plots=False):
    """(ny, nx) surface heights [m] (materials/roughsurface.py:12-69): normal
    noise of (ny + ky - 1, nx + kx - 1) samples filtered by FFT convolution
    in 'valid' mode."""
    if debug_plots:
        logger.info('debug plots are not drawn by this package')
    if rabus_compat:
        corr_len_x /= np.sqrt(2.0)
        corr_len_y /= np.sqrt(2.0)
    kernel, kx, ky = _gaussian_kernel(corr_len_x, corr_len_y, dx)
    rng = np.random.default_rng(seed=seed)
    noise = rng.normal(0, 1, size=(ny + ky - 1, nx + kx - 1))
    return _zero_mean_rms(scipy.signal.fftconvolve(noise, kernel, mode='valid'), height_rms)


def gaussian_correlated_surface_fast(nx, ny, dx, corr_len_x, corr_len_y, height_rms, rand_gen,
                                     rabus_compat=False):
    """(ny, nx) float32 surface heights from the generator ``rand_gen``
    (materials/roughsurface.py:72-130): float32 noise of the surface's own
    size, filtered by the separable kernel as causal 1-D convolutions along
    x and then y (the first nx / ny samples of each full convolution)."""
    if rabus_compat:
        corr_len_x /= np.sqrt(2.0)
        corr_len_y /= np.sqrt(2.0)
    cx, cy, rms = np.float32(corr_len_x), np.float32(corr_len_y), np.float32(height_rms)
    xs, _ = _kernel_samples(cx, dx)
    ys, _ = _kernel_samples(cy, dx)
    kx = np.exp(-(xs.astype(np.float32) ** 2 / cx ** 2))
    ky = np.exp(-(ys.astype(np.float32) ** 2 / cy ** 2))
    h = rand_gen.standard_normal(size=(ny, nx), dtype=np.float32)
    for y in range(ny):
        h[y, :] = np.convolve(h[y, :], kx)[:nx]
    for x in range(nx):
        h[:, x] = np.convolve(h[:, x], ky)[:ny]
    h = h - np.float32(np.mean(h))
    h /= np.float32(np.std(h))
    h *= rms
    return h


def correlate_layers(white_noise, cholesky):
    """Noise (ny, nx, layers) mixed across layers by a lower-triangular
    factor of the layers' covariance: out[y, x] = cholesky @ noise[y, x]."""
    return np.einsum('ij,yxj->yxi', cholesky, white_noise)


def two_layer_gaussian_correlated_surface(nx, ny, dx, corr_len_x, corr_len_y, height_rms,
                                          inter_layer_corr, seed=None, rabus_compat=False,
                                          debug_plots=False):
    """(2, ny, nx) heights [m] of two surfaces whose noise is correlated with
    coefficient ``inter_layer_corr`` (capped at 1 - 1e-5), each filtered by
    direct 2-D convolution in 'valid' mode (materials/roughsurface.py:
    133-213)."""
    if debug_plots:
        logger.info('debug plots are not drawn by this package')
    if rabus_compat:
        corr_len_x /= np.sqrt(2.0)
        corr_len_y /= np.sqrt(2.0)
    if inter_layer_corr >= 1.0:
        inter_layer_corr = 1.0 - 1e-5
    kernel, kx, ky = _gaussian_kernel(corr_len_x, corr_len_y, dx)
    rng = np.random.default_rng(seed=seed)
    noise = rng.normal(0, 1, size=(ny + ky - 1, nx + kx - 1, 2))
    chol = np.linalg.cholesky(np.array([[1.0, inter_layer_corr], [inter_layer_corr, 1.0]]))
    layers = np.transpose(correlate_layers(noise, chol), [2, 0, 1])
    out = np.zeros((2, ny, nx))
    for k in range(2):
        out[k] = _zero_mean_rms(scipy.signal.convolve2d(layers[k], kernel, mode='valid'), height_rms)
    return out
