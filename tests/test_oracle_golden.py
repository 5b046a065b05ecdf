"""The oracle reproduces the reference's own outputs (fixtures generated by
running fdtdsarsim on its CPU path, tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import fdtd_oracle as O
from helpers import GOLDEN, bits_equal

PROFILE_KEYS = ['be_d', 'bh_d', 'ce_d', 'ch_d', 'be_u', 'bh_u', 'ce_u', 'ch_u']


def _oracle_from_fixture(g, dtype):
    ab = np.load(os.path.join(GOLDEN, 'absorbers.npz'))
    prof = {k: ab[f'{dtype}_0.021_{k}'] for k in PROFILE_KEYS}
    return O.OracleSim(int(g['nx']), int(g['ny']), int(g['nz']), 10, int(g['tfsf_z']),
                       float(g['dx']), float(g['dt']), float(g['freq']), dtype, prof)


@pytest.mark.parametrize('tag', ['f32', 'f32_tfsf_in_pml'])
def test_mainloop_f32_bit_exact(tag):
    g = np.load(os.path.join(GOLDEN, f'mainloop_{tag}.npz'))
    sim = _oracle_from_fixture(g, 'float32')
    inc = {c: g[f'inc_{c}'] for c in ('ex', 'ey', 'hx', 'hy')}
    sim.run(g['ca'], g['cb'], inc, int(g['nt']))
    for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
        assert bits_equal(getattr(sim, c), g[f'field_{c}']), c
    for name in O.PHASOR_NAMES:
        assert bits_equal(sim.ph[name], g[name]), name


def test_mainloop_f64_bit_exact():
    g = np.load(os.path.join(GOLDEN, 'mainloop_f64.npz'))
    sim = _oracle_from_fixture(g, 'float64')
    inc = {c: g[f'inc_{c}'] for c in ('ex', 'ey', 'hx', 'hy')}
    sim.run(g['ca'], g['cb'], inc, int(g['nt']))
    nz = int(g['nz'])
    for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
        f = getattr(sim, c)
        assert np.sum(f, dtype=np.float64) == g[f'field_{c}_sum'], c
        assert bits_equal(f[nz // 2], g[f'field_{c}_plane']), c
    for name in O.PHASOR_NAMES:
        assert bits_equal(sim.ph[name], g[name]), name


def test_near2far_matches_reference():
    g = np.load(os.path.join(GOLDEN, 'near2far.npz'))
    for prefix, phis in (('ff', g['phis']), ('ff35', np.asarray([35.0]))):
        ff = O.near2far(g['ex_ph_u'], g['ey_ph_u'], g['hx_ph_u'], g['hy_ph_u'], int(g['nx']),
                        int(g['ny']), int(g['nz']), float(g['dx']), float(g['r']), g['thetas'],
                        phis, float(g['freq']))
        for k in ('E_theta', 'E_phi', 'H_theta', 'H_phi'):
            ref = g[f'{prefix}_{k}']
            err = np.max(np.abs(ff[k] - ref)) / np.max(np.abs(ref))
            assert err < 1e-12, (prefix, k, err)


def test_simpson_weights_match_scipy():
    import scipy.integrate
    rng = np.random.default_rng(3)
    for n in (3, 5, 19, 741):
        y = rng.standard_normal(n)
        w = O.simpson_weights(n, 0.37)
        assert abs(w @ y - scipy.integrate.simpson(y, dx=0.37)) < 1e-12 * max(1.0, np.abs(y).sum())


def test_pipeline_fixture_backscatter_consistent():
    """The end-to-end fixture (run_experiment on the 31x39x39 flat-soil case)
    is self-consistent under the oracle's near2far."""
    g = np.load(os.path.join(GOLDEN, 'pipeline_cfg1.npz'))
    nx = int(g['param_size_x']) - 20
    ny = int(g['param_size_y']) - 20
    nz = int(g['param_size_z']) - 20
    thetas = np.linspace(-80.0, 80.0, num=161, endpoint=True)
    ff = O.near2far(g['ex_ph_u'], g['ey_ph_u'], g['hx_ph_u'], g['hy_ph_u'], nx, ny, nz,
                    float(g['param_cell_size']), 2.0e3, thetas, [float(g['param_phi_angle'])],
                    float(g['param_frequency']))
    for k, ref in (('E_theta', 'ff_e_theta'), ('E_phi', 'ff_e_phi')):
        err = np.max(np.abs(ff[k] - g[ref])) / np.max(np.abs(g[ref]))
        assert err < 1e-12, (k, err)
    ph, pv = O.farfield_power(ff['E_theta'], ff['E_phi'], ff['H_theta'], ff['H_phi'])
    assert np.allclose(ph, g['ff_out_pwr_far_h'], rtol=1e-10, atol=0)


def test_geom_cases_fixture_present():
    with open(os.path.join(GOLDEN, 'geom_cases.json')) as fh:
        cases = json.load(fh)
    assert len(cases) >= 8
