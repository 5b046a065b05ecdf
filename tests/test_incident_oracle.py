"""The incident-beam oracle against fixtures made by the reference itself
(tests/golden/incident_*.npz, from IncidentBeam.create_pulse /
create_inc_excitation and IncidentSimCpu, incidentbeam.py:174-298 and
cpu/incident_sim.py:67-171)."""
import os

import numpy as np
import pytest

import incident_oracle as IO
from helpers import GOLDEN, bits_equal, make_params
from fdtdsarsim_b200.absorbers import cpml_profiles

CASES = ('hh_f32', 'vv_f64')


def load(tag):
    return np.load(os.path.join(GOLDEN, f'incident_{tag}.npz'))


def fixture_params(g):
    """Parameters of the fixture's geometry for the host helpers."""
    dtype = str(g['dtype'])
    pc = make_params(int(g['nx']), int(g['ny']), int(g['nz_inc']), int(g['nz_inc']) // 2,
                     int(g['size_t_inc']), int(g['size_t_inc']), dtype=dtype, cell_wl=0.05)
    pc.geom_params.cell_size = float(g['dx'])
    pc.geom_params.timestep = float(g['dt'])
    return pc


@pytest.mark.parametrize('tag', CASES)
def test_pulse_matches_reference(tag):
    g = load(tag)
    tv, pulse, pfft, pfreq = IO.create_pulse(float(g['dt']), int(g['size_t_inc']),
                                             int(g['size_t_pulse']), float(g['duration']),
                                             float(g['freq']))
    assert bits_equal(tv, g['time_vals'])
    assert np.max(np.abs(pulse - g['pulse'])) <= 1e-15
    assert np.max(np.abs(pfft - g['pulse_fft'])) <= 1e-12 * np.max(np.abs(g['pulse_fft']))
    assert bits_equal(pfreq, g['pulse_freqs'])


@pytest.mark.parametrize('tag', CASES)
def test_excitation_matches_reference(tag):
    """The excitation to tolerance: the reference evaluates exp/hypot in
    numba, the oracle in numpy, and float32 cases round the stages to
    complex64 as the reference does."""
    g = load(tag)
    dtype = str(g['dtype'])
    radius = IO.gauss_radius(float(g['illumination_width']), float(g['freq']))
    ex, ey = IO.create_inc_excitation(int(g['nx']), int(g['ny']), float(g['dx']), g['pulse_fft'],
                                      g['pulse_freqs'], float(g['theta']), float(g['phi']),
                                      str(g['pol']), radius, dtype)
    steps = g['exc_steps']
    tol = 2e-6 if dtype == 'float32' else 1e-12
    for got, ref in ((ex.imag[steps], g['exc_ex_imag_at']), (ey.imag[steps], g['exc_ey_imag_at']),
                     (ex.real[steps], g['exc_ex_real_at'])):
        assert np.max(np.abs(got - ref)) <= tol * 10.0
    assert abs(max(np.abs(ex).max(), np.abs(ey).max()) - float(g['exc_absmax'])) <= tol * 10.0


def run_oracle(g, exc_ex, exc_ey):
    pc = fixture_params(g)
    o = IO.IncidentOracle(int(g['nx']), int(g['ny']), int(g['nz_inc']), int(g['npml']),
                          float(g['dx']), float(g['dt']), float(g['freq']), str(g['dtype']),
                          cpml_profiles(pc))
    rec = o.run_incident(exc_ex, exc_ey, int(g['size_t_inc']))
    return o, rec


def test_incident_run_bit_exact_from_reference_excitation():
    """Given the reference's own excitation, the recorded planes and the
    incident phasors equal the reference's bit for bit."""
    g = load('hh_f32')
    o, rec = run_oracle(g, g['exc_ex_imag'], g['exc_ey_imag'])
    steps = g['rec_steps']
    for c in ('ex', 'ey', 'hx', 'hy'):
        assert bits_equal(rec[c][steps], g[f'inc_{c}_at']), c
        assert np.array_equal(np.sum(rec[c], axis=(1, 2), dtype=np.float64), g[f'inc_{c}_stepsum']), c
        assert bits_equal(o.inc_ph[c], g[f'{c}_inc_phasor']), c


def test_incident_run_float64_from_oracle_excitation():
    """float64 end to end (excitation and run) against the reference."""
    g = load('vv_f64')
    radius = IO.gauss_radius(float(g['illumination_width']), float(g['freq']))
    ex, ey = IO.create_inc_excitation(int(g['nx']), int(g['ny']), float(g['dx']), g['pulse_fft'],
                                      g['pulse_freqs'], float(g['theta']), float(g['phi']),
                                      str(g['pol']), radius, 'float64')
    npulse = int(g['size_t_pulse'])
    o, rec = run_oracle(g, ex.imag[:npulse].copy(), ey.imag[:npulse].copy())
    steps = g['rec_steps']
    for c in ('ex', 'ey', 'hx', 'hy'):
        ref = g[f'inc_{c}_at']
        assert np.max(np.abs(rec[c][steps] - ref)) <= 1e-11 * np.max(np.abs(ref)), c
        ph = g[f'{c}_inc_phasor']
        assert np.max(np.abs(o.inc_ph[c] - ph)) <= 1e-11 * np.max(np.abs(ph)), c


def test_incident_height():
    g = load('hh_f32')
    assert IO.incident_height(float(g['dx']), float(g['freq'])) == int(g['nz_inc'])
