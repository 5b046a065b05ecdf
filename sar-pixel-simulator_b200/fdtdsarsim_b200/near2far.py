"""Near-to-far transform on the device (fdtdsarsim/near2far.py:11-156)."""
from typing import Mapping

import numpy as np

from . import _native


class FarFieldTransform:
    """Far-field E/H at (r, theta, phi) from the top phasor plane.

    ``__call__`` has the reference's signature and output: a dict of
    E_theta, E_phi, H_theta, H_phi, each (nphi, ntheta) complex128 squeezed.
    The integration runs on the GPU (near2far.cu); the reference's choice of
    Simpson's rule is kept.
    """

    def __init__(self, device=0):
        self.device = device

    def __call__(self, phasors: Mapping, nx: int, ny: int, nz: int, dx: float, r: float,
                 thetas: np.ndarray, phis: np.ndarray, freq: float):
        thetas = np.asarray(thetas)
        phis = np.asarray(phis)
        if not (thetas.ndim == 1 and phis.ndim == 1):
            raise RuntimeError('Theta and phi arguments must be 1D arrays')
        ff = _native.near2far(np.asarray(phasors['ex_ph_u']), np.asarray(phasors['ey_ph_u']),
                              np.asarray(phasors['hx_ph_u']), np.asarray(phasors['hy_ph_u']),
                              int(nx), int(ny), int(nz), float(dx), float(r), thetas, phis,
                              float(freq), self.device)
        return {k: np.squeeze(v) for k, v in ff.items()}
