"""Host side of the gradient: the far-field coefficient planes reproduce the
near-to-far transform, and the phasor derivative of the power is exact."""
import numpy as np
import pytest

import fdtd_oracle as O
from fdtdsarsim_b200.adjoint import (ca_cb_partials, far_field_coefficients,
                                     power_and_phasor_grad)
from fdtdsarsim_b200.materials import MaterialModel, compute_material_arrays
from helpers import make_params


@pytest.mark.parametrize('pol', ['HH', 'VV'])
def test_coefficients_reproduce_near2far(pol):
    rng = np.random.default_rng(3)
    nx_ph, ny_ph, nz_ph, dx, f = 21, 17, 13, 0.0012, 5.4e9
    p = rng.standard_normal((4, ny_ph, nx_ph)) + 1j * rng.standard_normal((4, ny_ph, nx_ph))
    a, b, sign = far_field_coefficients(nx_ph, ny_ph, nz_ph, dx, 2000.0, -20.0, 0.0, f, pol)
    ff = O.near2far(p[0], p[1], p[2], p[3], nx_ph, ny_ph, nz_ph, dx, 2000.0, [-20.0], [0.0], f)
    u, v = np.sum(a * p), np.sum(b * p)
    if pol == 'HH':
        assert np.allclose(u, ff['E_phi'], rtol=1e-12) and np.allclose(v, ff['H_theta'], rtol=1e-12)
        ref = O.farfield_power(ff['E_theta'], ff['E_phi'], ff['H_theta'], ff['H_phi'])[0]
    else:
        assert np.allclose(u, ff['E_theta'], rtol=1e-12) and np.allclose(v, ff['H_phi'], rtol=1e-12)
        ref = O.farfield_power(ff['E_theta'], ff['E_phi'], ff['H_theta'], ff['H_phi'])[1]
    J = power_and_phasor_grad(p, a, b, sign)[0]
    assert np.isclose(J, ref, rtol=1e-12)


def test_phasor_gradient_is_exact():
    rng = np.random.default_rng(4)
    p = rng.standard_normal((4, 7, 9)) + 1j * rng.standard_normal((4, 7, 9))
    a, b, sign = far_field_coefficients(9, 7, 5, 0.001, 2000.0, -20.0, 0.0, 5.4e9, 'HH')
    J, g_re, g_im = power_and_phasor_grad(p, a, b, sign)
    for _ in range(6):
        k = tuple(rng.integers(0, s) for s in p.shape)
        for unit, g in ((1.0, g_re), (1j, g_im)):
            h = 1e-6
            q1, q2 = p.copy(), p.copy()
            q1[k] += unit * h
            q2[k] -= unit * h
            fd = (power_and_phasor_grad(q1, a, b, sign)[0] - power_and_phasor_grad(q2, a, b, sign)[0]) / (2 * h)
            assert abs(fd - g[k]) <= 1e-7 * abs(J) / h * 1e-3 + 1e-6 * abs(fd)


def test_material_partials_match_compute_material_arrays():
    pc = make_params(25, 23, 27, 14, 10, 5, dtype='float64')
    g = pc.geom_params
    rng = np.random.default_rng(5)
    shape = (g.size_z_material, g.size_y, g.size_x)
    eps = rng.uniform(2.0, 12.0, size=shape)
    sig = rng.uniform(0.0, 0.1, size=shape)
    dca_de, dca_ds, dcb_de, dcb_ds = ca_cb_partials(eps, sig, g.timestep, g.cell_size)
    for which, d_ca, d_cb in (('eps', dca_de, dcb_de), ('sig', dca_ds, dcb_ds)):
        h = 1e-6
        e1, e2, s1, s2 = eps.copy(), eps.copy(), sig.copy(), sig.copy()
        if which == 'eps':
            e1 += h * eps
            e2 -= h * eps
            step = 2 * h * eps
        else:
            s1 += h * np.maximum(sig, 1e-3)
            s2 -= h * np.maximum(sig, 1e-3)
            step = 2 * h * np.maximum(sig, 1e-3)
        ca1, cb1 = compute_material_arrays(pc, MaterialModel(e1, s1, g.cell_size))
        ca2, cb2 = compute_material_arrays(pc, MaterialModel(e2, s2, g.cell_size))
        nzm = g.size_z_material
        # central differences: relative truncation ~h^2, round-off ~1e-16 / h
        assert np.allclose((ca1 - ca2)[:nzm] / step, d_ca, rtol=1e-4, atol=1e-8 * np.abs(d_ca).max())
        assert np.allclose((cb1 - cb2)[:nzm] / step, d_cb, rtol=1e-4, atol=1e-8 * np.abs(d_cb).max())
