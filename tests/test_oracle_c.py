"""The C oracle (oracle/fdtd_oracle.c, POSIX threads) steps bit-identically to the
numpy oracle, and through it to the reference's own outputs."""
import os

import numpy as np
import pytest

import fdtd_oracle_c as OC
from helpers import GOLDEN, make_params, oracle_for, random_problem
from fdtdsarsim_b200.absorbers import cpml_profiles

pytestmark = pytest.mark.skipif(not OC.available(), reason='C oracle not built (make -C oracle)')


def _c_oracle(pc, nthreads):
    g = pc.geom_params
    return OC.COracleSim(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size,
                         g.timestep, pc.inc_beam_params.frequency, pc.processing_params.datatype,
                         cpml_profiles(pc), nthreads=nthreads)


def _same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


@pytest.mark.parametrize('case,nthreads', [((27, 25, 23, 14, 30, 20, 'float32'), 1),
                                           ((41, 37, 29, 16, 25, 25, 'float32'), 4),
                                           ((27, 25, 23, 20, 20, 12, 'float32'), 3),
                                           ((33, 23, 25, 12, 20, 10, 'float64'), 2)])
def test_c_oracle_matches_numpy_oracle(case, nthreads):
    nx, ny, nz, tfsf, nt, ntp, dtype = case
    pc = make_params(nx, ny, nz, tfsf, nt, ntp, dtype=dtype)
    _, _, ca, cb, inc = random_problem(pc, 77)
    a = oracle_for(pc)
    b = _c_oracle(pc, nthreads)
    a.run(ca, cb, inc, nt)
    b.run(ca, cb, inc, nt)
    for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
        assert _same(getattr(a, c), getattr(b, c)), c
    for name in a.ph:
        assert _same(a.ph[name], b.ph[name]), name
    for name in a.psi:
        assert _same(a.psi[name], b.psi[name]), name


def test_c_oracle_reproduces_reference_fixture():
    g = np.load(os.path.join(GOLDEN, 'mainloop_f32.npz'))
    ab = np.load(os.path.join(GOLDEN, 'absorbers.npz'))
    pc = make_params(int(g['nx']), int(g['ny']), int(g['nz']), int(g['tfsf_z']), int(g['nt']),
                     int(g['ntp']))
    gp = pc.geom_params
    prof = {k: ab[f'float32_0.021_{k}'] for k in ('be_d', 'bh_d', 'ce_d', 'ch_d', 'be_u', 'bh_u',
                                                   'ce_u', 'ch_u')}
    sim = OC.COracleSim(gp.size_x, gp.size_y, gp.size_z, gp.size_pml, gp.tfsf_z, gp.cell_size,
                        gp.timestep, pc.inc_beam_params.frequency, 'float32', prof, nthreads=4)
    inc = {c: g['inc_' + c] for c in ('ex', 'ey', 'hx', 'hy')}
    sim.run(g['ca'], g['cb'], inc, int(g['nt']))
    for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
        assert _same(getattr(sim, c), g[f'field_{c}']), c
    for name in sim.ph:
        assert _same(sim.ph[name], g[name]), name


def test_float32_against_float64_on_the_2x2_configuration():
    """The accuracy statement's first row (oracle/fp64_error.py): a full
    31x39x39 solve (720 steps) in float32 and in float64 -- the precisions
    the device reproduces bit for bit -- agree on the backscatter power to
    well inside the 1e-4 bar."""
    import fp64_error
    r = fp64_error.run('plain_2x2')
    assert r['grid'] == [31, 39, 39] and r['size_t'] == 720
    assert r['backscatter_power_rel_err'] < 1e-5
    assert r['backscatter_phasor_rel_err'] < 1e-5
    assert r['upper_plane_max_rel_err'] < 1e-4
