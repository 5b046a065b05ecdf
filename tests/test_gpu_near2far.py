"""Device near-to-far transform vs the oracle and the reference fixture."""
import os

import numpy as np
import pytest

import fdtd_oracle as O
from fdtdsarsim_b200 import _native
from fdtdsarsim_b200.near2far import FarFieldTransform
from helpers import GOLDEN

pytestmark = pytest.mark.gpu


def test_near2far_matches_reference_fixture():
    g = np.load(os.path.join(GOLDEN, 'near2far.npz'))
    for prefix, phis in (('ff', g['phis']), ('ff35', np.asarray([35.0]))):
        ff = FarFieldTransform()(g, int(g['nx']), int(g['ny']), int(g['nz']), float(g['dx']),
                                 float(g['r']), g['thetas'], phis, float(g['freq']))
        for k in ('E_theta', 'E_phi', 'H_theta', 'H_phi'):
            ref = g[f'{prefix}_{k}']
            err = np.max(np.abs(ff[k] - ref)) / np.max(np.abs(ref))
            assert err < 1e-10, (prefix, k, err)


def test_near2far_large_plane_vs_oracle():
    rng = np.random.default_rng(4)
    ny, nx = 181, 221
    planes = [(rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx))).astype(np.complex64)
              for _ in range(4)]
    thetas = np.linspace(-80.0, 80.0, 41)
    phis = np.asarray([0.0, 90.0])
    dx = 0.00116
    got = _native.near2far(*planes, nx, ny, 61, dx, 2.0e3, thetas, phis, 5.4e9)
    ref = O.near2far(*planes, nx, ny, 61, dx, 2.0e3, thetas, phis, 5.4e9)
    for k in ('E_theta', 'E_phi', 'H_theta', 'H_phi'):
        err = np.max(np.abs(got[k] - ref[k])) / np.max(np.abs(ref[k]))
        assert err < 1e-9, (k, err)


def test_pipeline_fixture_far_field_on_device():
    g = np.load(os.path.join(GOLDEN, 'pipeline_cfg1.npz'))
    nx = int(g['param_size_x']) - 20
    ny = int(g['param_size_y']) - 20
    nz = int(g['param_size_z']) - 20
    thetas = np.linspace(-80.0, 80.0, num=161, endpoint=True)
    ff = FarFieldTransform()(g, nx, ny, nz, float(g['param_cell_size']), 2.0e3, thetas,
                             np.asarray([float(g['param_phi_angle'])]), float(g['param_frequency']))
    for k, ref in (('E_theta', 'ff_e_theta'), ('E_phi', 'ff_e_phi'), ('H_theta', 'ff_h_theta'),
                   ('H_phi', 'ff_h_phi')):
        err = np.max(np.abs(ff[k] - g[ref])) / np.max(np.abs(g[ref]))
        assert err < 1e-10, (k, err)
