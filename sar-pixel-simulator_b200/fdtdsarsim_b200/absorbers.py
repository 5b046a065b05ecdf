"""CPML coefficient profiles (Taflove ch. 7.9), as 1-D arrays.

The reference builds eight 1-D profiles and then tiles them into 24 full
3-D arrays, one per face and coefficient (absorbers.py:35-189). The device
kernels index the 1-D profiles directly, so only these are computed here.
They must be bit-identical to the reference's, so each expression keeps the
reference's numpy evaluation: every intermediate in the simulation dtype
(Python scalars are weak under NumPy 2 promotion), the same powers, and the
hard-coded eta0/eps0 of absorbers.py:50-51.
"""
import numpy as np

from .parameters import ParameterCollection

PROFILE_ORDER = ('be_d', 'bh_d', 'ce_d', 'ch_d', 'be_u', 'bh_u', 'ce_u', 'ch_u')


def cpml_profiles(params: ParameterCollection) -> dict:
    """Return the 1-D CPML coefficient profiles of length size_pml.

    Keys: be_d, bh_d, ce_d, ch_d (down, left and front faces) and
    be_u, bh_u, ce_u, ch_u (up, right and back faces).
    """
    g = params.geom_params
    dtype = np.dtype(params.processing_params.datatype)
    dx, dt, npml = g.cell_size, g.timestep, g.size_pml
    eta0 = 376.730313668
    eps0 = 8.8541878128E-12
    feps = np.finfo(dtype).eps
    kappa_max, alpha_max = 1, 0.2
    m_kappa = m_sigma = 3
    m_alpha = 1
    sigma_max = 0.8 * (m_sigma + 1) / (eta0 * dx)  # Taflove eq. 7.66

    inc = np.arange(npml, dtype=dtype)
    dec = npml - 1 - inc
    span = npml - 1

    def prof(base, m):
        return ((base / span) ** m).astype(dtype)

    # down / left / front (increasing depth towards index 0)
    alpha_e_l = alpha_max * prof(inc, m_alpha)
    alpha_h_l = alpha_max * prof(inc + 0.5, m_alpha)
    sigma_e_l = sigma_max * prof(dec, m_sigma)
    sigma_h_l = sigma_max * prof(dec - 0.5, m_sigma)
    kappa_e_l = 1 + (kappa_max - 1) * prof(dec, m_kappa)
    kappa_h_l = 1 + (kappa_max - 1) * prof(dec + 0.5, m_kappa)
    # up / right / back
    alpha_e_u = alpha_max * prof(dec, m_alpha)
    alpha_h_u = alpha_max * prof(dec - 0.5, m_alpha)
    alpha_h_u[alpha_h_u < 0.0] = 0.0
    sigma_e_u = sigma_max * prof(inc, m_sigma)
    sigma_h_u = sigma_max * prof(inc + 0.5, m_sigma)
    kappa_e_u = 1 + (kappa_max - 1) * prof(inc, m_kappa)
    kappa_h_u = 1 + (kappa_max - 1) * prof(inc + 0.5, m_kappa)

    def b_coef(sigma, kappa, alpha):     # Taflove eq. 7.102
        return np.exp(-(sigma / kappa + alpha) * dt / eps0)

    def c_coef(sigma, kappa, alpha):     # Taflove eq. 7.99
        return (sigma + feps) * (np.exp(-(sigma / kappa + alpha) * dt / eps0) - 1) \
            / (sigma * kappa + (kappa ** 2 * alpha) + feps)

    out = {
        'be_d': b_coef(sigma_e_l, kappa_e_l, alpha_e_l),
        'bh_d': b_coef(sigma_h_l, kappa_h_l, alpha_h_l),
        'ce_d': c_coef(sigma_e_l, kappa_e_l, alpha_e_l),
        'ch_d': c_coef(sigma_h_l, kappa_h_l, alpha_h_l),
        'be_u': b_coef(sigma_e_u, kappa_e_u, alpha_e_u),
        'bh_u': b_coef(sigma_h_u, kappa_h_u, alpha_h_u),
        'ce_u': c_coef(sigma_e_u, kappa_e_u, alpha_e_u),
        'ch_u': c_coef(sigma_h_u, kappa_h_u, alpha_h_u),
    }
    for k, v in out.items():
        if v.dtype != dtype:
            raise TypeError(f'CPML profile {k} came out {v.dtype}, expected {dtype}')
    return out


def packed_profiles(params: ParameterCollection) -> np.ndarray:
    """The eight profiles packed in fdtd_set_absorbers order."""
    p = cpml_profiles(params)
    return np.ascontiguousarray(np.concatenate([p[k] for k in PROFILE_ORDER]))


class Absorbers:
    """Holds the CPML profiles of one geometry (absorbers.py:13-33)."""

    def __init__(self, params: ParameterCollection):
        self.profiles = cpml_profiles(params)
        for k, v in self.profiles.items():
            setattr(self, k, v)
