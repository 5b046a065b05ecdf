"""Gradient of the backscatter power with respect to per-cell eps_r and sigma.

The reference computes no gradient; this module differentiates its
backscatter observable. The objective is the scattered power in one far-field
direction, P_h = 1/2 Re(-E_phi conj(H_theta)) for HH and
P_v = 1/2 Re(E_theta conj(H_phi)) for VV (processresults.py:260-271), at the
backscatter direction theta = -theta_inc, phi = 0
(release_examples/cuda_example/gather.py:39-53), with the far field from the
near-to-far transform of the upper phasor plane (near2far.py:28-156).

E and H in one direction are linear in the four upper-plane phasors, so the
objective's derivative with respect to the real and imaginary part of every
phasor cell is exact and cheap on the host. The library then runs the
forward solve keeping a checkpoint every k steps and sweeps the transposed
step backwards, recomputing each segment from its checkpoint
(fdtd_grad_forward / fdtd_grad_backward), which yields dJ/dCa and dJ/dCb per
cell; the closed form of compute_material_arrays (materials/materials.py:
23-68) maps them to eps_r and sigma.

``BackscatterPower`` wraps this as a ``torch.autograd.Function``.
"""
from typing import Mapping, Optional

import numpy as np

from . import _native
from .absorbers import packed_profiles
from .materials import MaterialModel, compute_material_arrays
from .parameters import ParameterCollection

ETA0 = 376.730313668
C0 = 299792458
EPS0_MAT = 8.8541878128e-12   # the permittivity constant of the material code
RADIUS = 2.0e3                # far-field radius of process_results


def _simpson(n, dx):
    if n % 2 != 1 or n < 3:
        raise ValueError('odd sample count >= 3 required')
    w = np.ones(n)
    w[1:-1:2] = 4.0
    w[2:-1:2] = 2.0
    return w * dx / 3.0


def far_field_coefficients(nx_ph, ny_ph, nz_ph, dx, r, theta_deg, phi_deg, freq, pol='HH'):
    """(a, b, sign): complex planes (4, ny_ph, nx_ph) over (ex, ey, hx, hy)
    of the upper phasor plane with u = sum a p and v = sum b p the two
    far-field components of the power, P = sign * 1/2 Re(u conj(v)).
    HH: u = E_phi, v = H_theta, sign -1; VV: u = E_theta, v = H_phi, sign +1
    (the transform of near2far.py:28-156 in one direction: J = (-Hy, Hx),
    M = (Ey, -Ex), Simpson weights, plane height ((nz_ph - 1) // 2) dx)."""
    k = 2.0 * np.pi * freq / C0
    t_, p_ = np.deg2rad(theta_deg), np.deg2rad(phi_deg)
    x_loc = np.arange(-(nx_ph - 1) // 2, ((nx_ph - 1) // 2) + 1) * dx
    y_loc = np.arange(-(ny_ph - 1) // 2, ((ny_ph - 1) // 2) + 1) * dx
    z_val = ((nz_ph - 1) // 2) * dx
    xx, yy = np.meshgrid(x_loc, y_loc)
    e = np.exp(1j * k * (xx * np.sin(t_) * np.cos(p_) + yy * np.sin(t_) * np.sin(p_)
                         + z_val * np.cos(t_)))
    w = np.outer(_simpson(ny_ph, dx), _simpson(nx_ph, dx)) * e
    ct, cp, sp = np.cos(t_), np.cos(p_), np.sin(p_)
    ffw = 1j * k * np.exp(-1j * k * r) / (4.0 * np.pi * r)
    z0 = np.zeros_like(w)
    # potentials as planes over (ex, ey, hx, hy)
    nt = np.stack([z0, z0, w * ct * sp, -w * ct * cp])      # Jx ct cp + Jy ct sp
    np_ = np.stack([z0, z0, w * cp, w * sp])                # -Jx sp + Jy cp
    lt = np.stack([-w * ct * sp, w * ct * cp, z0, z0])      # Mx ct cp + My ct sp
    lp = np.stack([-w * cp, -w * sp, z0, z0])               # -Mx sp + My cp
    if pol.upper() == 'HH':
        return ffw * (lt - ETA0 * np_), ffw * (np_ - lt / ETA0), -1.0
    if pol.upper() == 'VV':
        return ffw * (-lp - ETA0 * nt), ffw * (-nt - lp / ETA0), 1.0
    raise ValueError('Invalid polarization')


def power_and_phasor_grad(p, a, b, sign):
    """P and (dP/dRe p, dP/dIm p) for p stacked (4, ny_ph, nx_ph)."""
    u = np.sum(a * p)
    v = np.sum(b * p)
    J = sign * 0.5 * float(np.real(u * np.conj(v)))
    g_re = sign * 0.5 * np.real(a * np.conj(v) + b * np.conj(u))
    g_im = sign * 0.5 * (np.imag(np.conj(a) * v) + np.imag(np.conj(b) * u))
    return J, g_re, g_im


def ca_cb_partials(eps_r, sigma, dt, dx):
    """dCa/deps_r, dCa/dsigma, dCb/deps_r, dCb/dsigma of
    Ca = (1 - x) / (1 + x), Cb = (dt / (eps_r eps0 dx)) / (1 + x),
    x = sigma dt / (2 eps_r eps0) (materials/materials.py:45-63)."""
    eps_r = np.asarray(eps_r, dtype=np.float64)
    sigma = np.asarray(sigma, dtype=np.float64)
    perm = eps_r * EPS0_MAT
    x = sigma * dt / (2.0 * perm)
    dx_de = -x / eps_r
    dx_ds = dt / (2.0 * perm)
    dca_dx = -2.0 / (1.0 + x) ** 2
    cb0 = dt / (perm * dx)
    dcb_de = -cb0 / eps_r / (1.0 + x) - cb0 / (1.0 + x) ** 2 * dx_de
    dcb_ds = -cb0 / (1.0 + x) ** 2 * dx_ds
    return dca_dx * dx_de, dca_dx * dx_ds, dcb_de, dcb_ds


class BackscatterGradient:
    """Backscatter power of one geometry and its gradient with respect to
    eps_r and sigma of the material block (size_z_material, ny, nx).

    ``incident`` holds the incident planes 'ex', 'ey', 'hx', 'hy'
    (size_t_inc, ny, nx) of the geometry. ``checkpoint_every`` is the
    forward checkpoint period k.
    """

    def __init__(self, params: ParameterCollection, incident: Mapping[str, np.ndarray],
                 checkpoint_every: int = 64, device: int = 0, theta_deg: Optional[float] = None,
                 phi_deg: float = 0.0, pol: Optional[str] = None, radius: float = RADIUS,
                 kernel: Optional[int] = None):
        from .gpu.main_sim import native_geometry
        self.params = params
        g = params.geom_params
        self.every = int(checkpoint_every)
        from . import tuning
        geom = native_geometry(params)
        self.sim = _native.NativeSim(geom, device)
        self.sim.set_absorbers(packed_profiles(params))
        tuning.apply(self.sim, tuning.choose(geom, kernel=kernel, device=device))
        self.sim.set_incident(incident['ex'], incident['ey'], incident['hx'], incident['hy'])
        theta = -params.inc_beam_params.theta_angle if theta_deg is None else theta_deg
        pol = params.inc_beam_params.polarization if pol is None else pol
        m = g.size_pml
        self.nx_ph, self.ny_ph, self.nz_ph = g.size_x - 2 * m, g.size_y - 2 * m, g.size_z - 2 * m
        self.a, self.b, self.sign = far_field_coefficients(
            self.nx_ph, self.ny_ph, self.nz_ph, g.cell_size, radius, theta, phi_deg,
            params.inc_beam_params.frequency, pol)

    def _set_materials(self, eps_r, sigma):
        g = self.params.geom_params
        dt = self.params.processing_params.datatype
        model = MaterialModel(np.asarray(eps_r, dtype=dt), np.asarray(sigma, dtype=dt),
                              g.cell_size)
        ca, cb = compute_material_arrays(self.params, model)
        self.sim.set_materials(ca, cb)

    def _upper_phasors(self):
        return np.stack([self.sim.get_phasor(k).astype(np.complex128) for k in (4, 5, 6, 7)])

    def value(self, eps_r, sigma):
        """Forward solve only: the backscatter power."""
        self._set_materials(eps_r, sigma)
        self.sim.reset()
        self.sim.run(self.params.geom_params.size_t)
        self.sim.synchronize()
        return power_and_phasor_grad(self._upper_phasors(), self.a, self.b, self.sign)[0]

    def value_and_grad(self, eps_r, sigma):
        """(P, dP/deps_r, dP/dsigma), the gradients with the material block's
        shape, in float64."""
        g = self.params.geom_params
        self._set_materials(eps_r, sigma)
        self.sim.grad_forward(self.every)
        J, g_re, g_im = power_and_phasor_grad(self._upper_phasors(), self.a, self.b, self.sign)
        nzm = g.size_z_material
        gca, gcb = self.sim.grad_backward(g_re, g_im, nzm)
        dca_de, dca_ds, dcb_de, dcb_ds = ca_cb_partials(eps_r, sigma, g.timestep, g.cell_size)
        return J, gca * dca_de + gcb * dcb_de, gca * dca_ds + gcb * dcb_ds

    def close(self):
        self.sim.close()


def _torch_function():
    import torch

    class BackscatterPower(torch.autograd.Function):
        """P = BackscatterPower.apply(eps_r, sigma, runner): the backscatter
        power of a BackscatterGradient runner as a differentiable function of
        the eps_r and sigma tensors (material block shape)."""

        @staticmethod
        def forward(ctx, eps_r, sigma, runner):
            J, ge, gs = runner.value_and_grad(eps_r.detach().cpu().numpy(),
                                              sigma.detach().cpu().numpy())
            ctx.save_for_backward(torch.from_numpy(ge).to(eps_r.device, eps_r.dtype),
                                  torch.from_numpy(gs).to(sigma.device, sigma.dtype))
            return torch.tensor(J, dtype=torch.float64, device=eps_r.device)

        @staticmethod
        def backward(ctx, grad_out):
            ge, gs = ctx.saved_tensors
            return grad_out.to(ge.dtype) * ge, grad_out.to(gs.dtype) * gs, None

    return BackscatterPower


_FN = None


def backscatter_power(eps_r, sigma, runner: BackscatterGradient):
    """Differentiable backscatter power (torch tensors in, scalar tensor out)."""
    global _FN
    if _FN is None:
        _FN = _torch_function()
    return _FN.apply(eps_r, sigma, runner)
