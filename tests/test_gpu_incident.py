"""Incident-beam generation on the device against the reference's own beam
(tests/golden/incident_*.npz and pipeline_cfg1.npz, made by
tests/golden/make_golden.py from IncidentBeam / IncidentSimCpu,
incidentbeam.py:41-298 and cpu/incident_sim.py:22-171)."""
import json
import os

import numpy as np
import pytest

import incident_oracle as IO
from helpers import GOLDEN, bits_equal, make_params, native_for, random_problem
from fdtdsarsim_b200 import _native
from fdtdsarsim_b200.absorbers import packed_profiles
from fdtdsarsim_b200.gpu.main_sim import native_geometry

pytestmark = pytest.mark.gpu


def load(tag):
    return np.load(os.path.join(GOLDEN, f'incident_{tag}.npz'))


def native_incident(g):
    """NativeIncident of a fixture's geometry."""
    dtype = str(g['dtype'])
    nz = int(g['nz_inc'])
    pc = make_params(int(g['nx']), int(g['ny']), nz, nz // 2, int(g['size_t_inc']), 0,
                     dtype=dtype, cell_wl=0.05)
    pc.geom_params.cell_size = float(g['dx'])
    pc.geom_params.timestep = float(g['dt'])
    pc.inc_beam_params.frequency = float(g['freq'])
    geom = native_geometry(pc)
    inc = _native.NativeIncident(geom, int(g['size_t_pulse']), 0)
    inc.set_absorbers(packed_profiles(pc))
    return inc


def make_exc(inc, g):
    k = (2 * np.pi * g['pulse_freqs']) / 299792458
    radius = IO.gauss_radius(float(g['illumination_width']), float(g['freq']))
    return inc.make_excitation(k, g['pulse_fft'], float(g['theta']), float(g['phi']), str(g['pol']),
                               radius)


@pytest.mark.parametrize('tag', ['hh_f32', 'vv_f64'])
def test_excitation_matches_reference(tag):
    """The device excitation (float64 throughout, cuFFT) against the
    reference's (complex64 stages for float32): within the float32 rounding
    of the reference's stages, 2e-6 of the peak of 10; float64 1e-11."""
    g = load(tag)
    inc = native_incident(g)
    try:
        make_exc(inc, g)
        ex, ey = inc.get_excitation()
    finally:
        inc.close()
    tol = (2e-6 if str(g['dtype']) == 'float32' else 1e-11) * 10.0
    s = g['exc_steps']
    assert np.max(np.abs(ex[s] - g['exc_ex_imag_at'])) <= tol
    assert np.max(np.abs(ey[s] - g['exc_ey_imag_at'])) <= tol
    if 'exc_ex_imag' in g.files:
        assert np.max(np.abs(ex - g['exc_ex_imag'])) <= tol
        assert np.max(np.abs(ey - g['exc_ey_imag'])) <= tol


@pytest.mark.parametrize('kernel', [_native.FDTD_KERNEL_SPLIT, _native.FDTD_KERNEL_FUSED],
                         ids=['split', 'fused'])
def test_run_bit_exact_from_reference_excitation(kernel):
    """From the reference's excitation, the recorded planes and incident
    phasors equal the reference's bit for bit (float32), on the split step
    and on the fused step (whose source plane is written after each step)."""
    g = load('hh_f32')
    inc = native_incident(g)
    inc.set_option(_native.OPT_KERNEL, kernel)
    try:
        inc.set_excitation(g['exc_ex_imag'], g['exc_ey_imag'])
        inc.run()
        planes, ph = inc.get_planes(), inc.get_phasors()
    finally:
        inc.close()
    s = g['rec_steps']
    for c in ('ex', 'ey', 'hx', 'hy'):
        assert bits_equal(planes[c][s], g[f'inc_{c}_at']), c
        assert np.array_equal(np.sum(planes[c], axis=(1, 2), dtype=np.float64), g[f'inc_{c}_stepsum']), c
        assert bits_equal(ph[f'{c}_inc_phasor'], g[f'{c}_inc_phasor']), c


@pytest.mark.parametrize('tag', ['hh_f32', 'vv_f64'])
def test_device_beam_end_to_end(tag):
    """Excitation and run on the device against the reference's beam:
    relative to each plane set's peak, 2e-5 (float32) / 1e-10 (float64)."""
    g = load(tag)
    inc = native_incident(g)
    try:
        make_exc(inc, g)
        inc.run()
        planes, ph = inc.get_planes(), inc.get_phasors()
    finally:
        inc.close()
    tol = 2e-5 if str(g['dtype']) == 'float32' else 1e-10
    s = g['rec_steps']
    for c in ('ex', 'ey', 'hx', 'hy'):
        ref = g[f'inc_{c}_at']
        assert np.max(np.abs(planes[c][s] - ref)) <= tol * np.max(np.abs(ref)), c
        p = g[f'{c}_inc_phasor']
        assert np.max(np.abs(ph[f'{c}_inc_phasor'] - p)) <= tol * np.max(np.abs(p)), c


def test_set_incident_from_equals_host_upload():
    """A main simulation fed device to device by an incident run steps
    exactly as one fed the same planes from host memory."""
    pc = make_params(41, 37, 33, 16, 40, 30)
    _, _, ca, cb, _ = random_problem(pc, 5)
    g = pc.geom_params
    ipc = make_params(g.size_x, g.size_y, 60, 30, 36, 0, cell_wl=0.021)
    geom = native_geometry(ipc)
    inc = _native.NativeIncident(geom, 20, 0)
    inc.set_absorbers(packed_profiles(ipc))
    rng = np.random.default_rng(2)
    exc = [rng.standard_normal((20, g.size_y, g.size_x)).astype(np.float32) for _ in range(2)]
    inc.set_excitation(*exc)
    inc.run()
    planes = inc.get_planes()
    a, b = native_for(pc), native_for(pc)
    try:
        for s in (a, b):
            s.set_materials(ca, cb)
        a.set_incident_from(inc)
        b.set_incident(*[planes[c][:g.size_t_inc] for c in ('ex', 'ey', 'hx', 'hy')])
        for s in (a, b):
            s.run(g.size_t)
            s.synchronize()
        for c in ('ex', 'hy'):
            assert bits_equal(a.get_field(c), b.get_field(c)), c
        assert np.abs(a.get_field('ey')).max() > 0
    finally:
        a.close()
        b.close()
        inc.close()


def test_invalid_polarization_and_order():
    g = load('hh_f32')
    inc = native_incident(g)
    try:
        with pytest.raises(_native.FdtdError) as ei:
            inc.run()
        assert ei.value.code == _native.FDTD_ERR_STATE
        k = (2 * np.pi * g['pulse_freqs']) / 299792458
        rc = _native.lib.fdtd_incident_make_excitation(
            inc.h, _native.ptr(np.ascontiguousarray(k)), _native.ptr(np.ascontiguousarray(g['pulse_fft'])),
            int(k.size), 20.0, 0.0, 9, 0.01, None)
        assert rc == _native.FDTD_ERR_INVALID
        assert 'polarization' in _native.last_error()
    finally:
        inc.close()


def test_run_experiment_cfg1_with_device_beam(tmp_path):
    """run_experiment end to end on the 31x39x39 flat-soil configuration,
    incident beam made on the device, against the reference's own
    run_experiment: incident planes within 2e-5 of their peak, the phasor
    planes within 1e-4, and the backscatter power within 1e-4."""
    import fdtdsarsim_b200 as fdtd
    from fdtdsarsim_b200 import resultsio
    from fdtdsarsim_b200.parameters import inc_filename, results_filename
    ref = np.load(os.path.join(GOLDEN, 'pipeline_cfg1.npz'))
    user = json.loads(str(ref['params_json']))
    user.update({'processing_type': 'gpu', 'project_dir': str(tmp_path), 'gpu_num': 0})
    path = tmp_path / 'params.json'
    path.write_text(json.dumps(user))
    pc = fdtd.load_from_json(str(path))
    mats = fdtd.materials.flat_surface(pc, 6.0, 0.01, name='flat')
    fdtd.run_experiment(pc, mats)
    with resultsio.File(inc_filename(pc), 'r') as f:
        for c in ('ex', 'ey', 'hx', 'hy'):
            d = np.asarray(f[c])
            for t in (150, 300):
                r = ref[f'inc_{c}_t{t}']
                assert np.max(np.abs(d[t] - r)) <= 2e-5 * np.max(np.abs(r)), (c, t)
    with resultsio.File(results_filename(pc, 'flat'), 'r') as f:
        for name in _native.PHASOR_NAMES:
            got = np.asarray(f['phasors'][name])
            r = ref[name]
            assert np.max(np.abs(got - r)) <= 1e-4 * np.max(np.abs(r)), name
        pw = np.asarray(f['farfield']['out_pwr_far_h'])
        r = ref['ff_out_pwr_far_h']
        assert np.max(np.abs(pw - r)) <= 1e-4 * np.max(np.abs(r))


def test_run_experiment_hands_the_beam_over_on_the_device(tmp_path):
    """The beam IncidentBeam.setup makes is copied device to device into
    the main simulation (nothing is left held afterwards); a later
    experiment that reads the written incident file gets bit-identical
    phasors."""
    import fdtdsarsim_b200 as fdtd
    from fdtdsarsim_b200 import incident, resultsio
    from fdtdsarsim_b200.parameters import results_filename
    ref = np.load(os.path.join(GOLDEN, 'pipeline_cfg1.npz'))
    user = json.loads(str(ref['params_json']))
    user.update({'processing_type': 'gpu', 'project_dir': str(tmp_path), 'gpu_num': 0})
    path = tmp_path / 'params.json'
    path.write_text(json.dumps(user))
    pc = fdtd.load_from_json(str(path))
    fdtd.run_experiment(pc, fdtd.materials.flat_surface(pc, 6.0, 0.01, name='first'))
    assert not incident._RESIDENT
    fdtd.run_experiment(pc, fdtd.materials.flat_surface(pc, 6.0, 0.01, name='second'))
    out = []
    for name in ('first', 'second'):
        with resultsio.File(results_filename(pc, name), 'r') as f:
            out.append({k: np.asarray(f['phasors'][k]) for k in _native.PHASOR_NAMES})
    for k in _native.PHASOR_NAMES:
        assert bits_equal(out[0][k], out[1][k]), k


def test_run_eps_sigma_equals_run_with_host_coefficients(tmp_path):
    """MainSimGpu.run_eps_sigma (Ca/Cb computed on the device, the path
    run_experiment takes) writes the same result file as run() given the
    host's compute_material_arrays (materials/materials.py:23-68), bit for
    bit, on a rough two-material block; a block of the wrong shape is
    rejected before anything runs."""
    import fdtdsarsim_b200 as fdtd
    from fdtdsarsim_b200 import resultsio
    from fdtdsarsim_b200.gpu.main_sim import MainSimGpu
    from fdtdsarsim_b200.materials import compute_material_arrays
    from fdtdsarsim_b200.parameters import results_filename
    ref = np.load(os.path.join(GOLDEN, 'pipeline_cfg1.npz'))
    user = json.loads(str(ref['params_json']))
    user.update({'processing_type': 'gpu', 'project_dir': str(tmp_path), 'gpu_num': 0})
    path = tmp_path / 'params.json'
    path.write_text(json.dumps(user))
    pc = fdtd.load_from_json(str(path))
    g = pc.geom_params
    model = next(fdtd.materials.rough_dielectric(pc, 7.5, 0.03, 0.3 * g.cell_size * 4,
                                                 0.5 * g.size_z_material * g.cell_size,
                                                 4 * g.cell_size, 1, seed=11))
    fdtd.IncidentBeam(pc).setup()
    sim = MainSimGpu(pc)
    try:
        ca, cb = compute_material_arrays(pc, model)
        sim.run(ca, cb, 'host', model.metadata)
        sim.run_eps_sigma(model.relative_permittivity, model.conductivity, 'device',
                          model.metadata)
        with pytest.raises(ValueError):
            sim.run_eps_sigma(model.relative_permittivity[1:], model.conductivity[1:], 'bad', {})
        with pytest.raises(RuntimeError):
            sim.run_eps_sigma(model.relative_permittivity, model.conductivity[1:], 'bad', {})
    finally:
        sim.close()
    out = []
    for name in ('host', 'device'):
        with resultsio.File(results_filename(pc, name), 'r') as f:
            out.append({k: np.asarray(f['phasors'][k]) for k in _native.PHASOR_NAMES})
    for k in _native.PHASOR_NAMES:
        assert bits_equal(out[0][k], out[1][k]), k
    assert np.max(np.abs(out[0]['ex_ph_u'])) > 0
