"""Host logic of the package (geometry, CPML profiles, material
coefficients, file layout) against the reference's own outputs."""
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, bits_equal, make_params
from fdtdsarsim_b200 import parameters as P
from fdtdsarsim_b200.absorbers import cpml_profiles, packed_profiles, PROFILE_ORDER
from fdtdsarsim_b200.materials import MaterialModel, compute_material_arrays
from fdtdsarsim_b200 import resultsio


def test_set_geom_params_matches_reference():
    with open(os.path.join(GOLDEN, 'geom_cases.json')) as fh:
        cases = json.load(fh)
    for case in cases:
        sx, sy, sz, dur, cs, unit, mf, incd, freq = case['args']
        pc = P.ParameterCollection()
        pc.inc_beam_params.frequency = freq
        pc.inc_beam_params.duration = incd
        pc.material_params.material_fraction = mf
        P.set_geom_params(pc, sx, sy, sz, dur, cs, unit)
        for k, v in case['geom'].items():
            assert getattr(pc.geom_params, k) == v, (case['args'], k)


def test_set_geom_params_bad_unit():
    pc = P.ParameterCollection()
    pc.inc_beam_params.frequency = 5.4e9
    with pytest.raises(ValueError):
        P.set_geom_params(pc, 1.0, 1.0, 0.5, 10.0, 0.05, 'furlong')


def test_round_to_odd():
    assert P.round_to_odd(39.0) == 39
    assert P.round_to_odd(30.0) == 31
    assert P.round_to_odd(30.9) == 31
    with pytest.raises(ValueError):
        P.round_to_odd(-1.0)


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
@pytest.mark.parametrize('cell_wl', [0.021, 0.05])
def test_cpml_profiles_bit_exact(dtype, cell_wl):
    ab = np.load(os.path.join(GOLDEN, 'absorbers.npz'))
    pc = make_params(25, 23, 27, 14, 10, 5, dtype=dtype, cell_wl=cell_wl)
    tag = f'{dtype}_{cell_wl}'
    assert pc.geom_params.cell_size == float(ab[f'{tag}_dx'])
    prof = cpml_profiles(pc)
    for k in PROFILE_ORDER:
        assert bits_equal(prof[k], ab[f'{tag}_{k}']), k
    packed = packed_profiles(pc)
    assert packed.shape == (80,) and packed.dtype == np.dtype(dtype)


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_material_arrays_bit_exact(dtype):
    m = np.load(os.path.join(GOLDEN, 'materials.npz'))
    pc = make_params(25, 23, int(m[f'{dtype}_nz']), 14, 10, 5, dtype=dtype)
    pc.geom_params.size_z_material = m[f'{dtype}_eps'].shape[0]
    ca, cb = compute_material_arrays(pc, MaterialModel(m[f'{dtype}_eps'], m[f'{dtype}_sigma'], 1.0))
    assert bits_equal(ca, m[f'{dtype}_ca'])
    assert bits_equal(cb, m[f'{dtype}_cb'])


def test_material_shape_mismatch():
    pc = make_params(25, 23, 27, 14, 10, 5)
    with pytest.raises(RuntimeError):
        compute_material_arrays(pc, MaterialModel(np.ones((3, 23, 25), 'float32'),
                                                  np.ones((4, 23, 25), 'float32'), 1.0))


def test_load_from_json(tmp_path):
    d = {
        'processing_type': 'gpu', 'gpu_num': 0, 'threads_per_proc': 6,
        'datatype': 'float32', 'project_dir': str(tmp_path), 'frequency_hz': 5.4e9,
        'polarization': 'HH', 'theta_angle_deg': 20.0, 'phi_angle_deg': 0.0,
        'incident_duration': 8.0, 'illumination_width': 8.0, 'generate_new': False,
        'size_x': 14.0, 'size_y': 14.0, 'size_z_material': 4.0, 'simulation_duration': 16.0,
        'cell_size': 0.025, 'unit': 'wavelength', 'material_fraction': 0.7,
        'disp_inc_results': False, 'disp_inc_sim_movie': False, 'disp_debug': False,
        'disp_main_sim_movie': False, 'disp_materials': False,
    }
    p = tmp_path / 'params.json'
    p.write_text(json.dumps(d))
    pc = P.load_from_json(str(p))
    with open(os.path.join(GOLDEN, 'geom_cases.json')) as fh:
        ref = [c for c in json.load(fh) if c['args'][:3] == [14.0, 14.0, 4.0]][0]['geom']
    for k, v in ref.items():
        if k != 'simulation_duration':  # set by load_from_json, not set_geom_params
            assert getattr(pc.geom_params, k) == v, k
    assert pc.geom_params.simulation_duration == 16.0
    assert P.inc_filename(pc).endswith(
        f'incident/inc_nx{ref["size_x"]}_ny{ref["size_y"]}_nt{ref["size_t_inc"]}_theta20_phi0_HH.hdf5')
    assert P.results_filename(pc, 'm1').endswith('results/m1.hdf5')
    del d['size_x']
    p.write_text(json.dumps(d))
    pc2 = P.load_from_json(str(p))
    assert pc2.geom_params.size_x == 0 and pc2.geom_params.simulation_duration == 16.0


def test_resultsio_roundtrip(tmp_path):
    fname = str(tmp_path / 'r.hdf5')
    with resultsio.File(fname, 'w') as f:
        g = f.create_group('phasors')
        g.attrs['nx_phasor'] = 5
        g.create_dataset('ex_ph_u', data=np.arange(6, dtype=np.complex64).reshape(2, 3))
        f.create_group('parameters').attrs['polarization'] = 'HH'
        f.create_group('material_metadata')
    assert resultsio.exists(fname)
    with resultsio.File(fname, 'r+') as f:
        assert f['phasors'].attrs['nx_phasor'] == 5
        assert str(f['parameters'].attrs['polarization']) == 'HH'
        assert 'material_metadata' in f
        np.testing.assert_array_equal(f['phasors/ex_ph_u'][:],
                                      np.arange(6, dtype=np.complex64).reshape(2, 3))
        f.create_group('farfield').create_dataset('e_phi', data=np.ones(3))
    with resultsio.File(fname, 'r') as f:
        assert f['farfield']['e_phi'].shape == (3,)


def test_incident_file_roundtrip_and_checks(tmp_path):
    """An incident file written in the reference's layout passes
    IncidentBeam's shape, dtype and metadata checks (incidentbeam.py:
    74-165), and each kind of mismatch is rejected with the reference's
    ValueError."""
    import copy
    from fdtdsarsim_b200 import resultsio
    from fdtdsarsim_b200.incidentbeam import IncidentBeam, write_incident_file
    from fdtdsarsim_b200.parameters import inc_filename
    from helpers import make_params
    pc = make_params(25, 23, 27, 14, 10, 6)
    pc.processing_params.project_dir = str(tmp_path)
    g = pc.geom_params
    planes = [np.full((g.size_t_inc, g.size_y, g.size_x), k, np.float32) for k in range(4)]
    ph = {f'{c}_inc_phasor': np.zeros((g.size_y - 20, g.size_x - 20), np.complex64)
          for c in ('ex', 'ey', 'hx', 'hy')}
    write_incident_file(pc, *planes, ph)
    beam = IncidentBeam(pc)
    assert beam.inc_beam_exists()
    beam.load_existing()
    other = copy.deepcopy(pc)
    other.inc_beam_params.duration = pc.inc_beam_params.duration + 1.0
    with resultsio.File(inc_filename(pc), 'r') as f:
        with pytest.raises(ValueError, match='duration'):
            IncidentBeam(other).check_metadata(f.attrs)
    with pytest.raises(ValueError, match='wrong shape'):
        beam.check_array_sizes(np.zeros((1, 2, 3), np.float32))
    with pytest.raises(ValueError, match='incorrect datatype'):
        beam.check_array_sizes(np.zeros((g.size_t_inc, g.size_y, g.size_x), np.float64))


def test_tuning_cache_choose_and_apply(tmp_path, monkeypatch):
    """tuning.choose takes an explicit choice, else a cached measurement,
    else the default; tuning.apply sets the matching library options."""
    import json
    from fdtdsarsim_b200 import _native, tuning
    from fdtdsarsim_b200.gpu.main_sim import native_geometry
    from helpers import make_params
    monkeypatch.setenv('FDTDSARSIM_B200_TUNING', str(tmp_path / 'tune.json'))
    geom = native_geometry(make_params(41, 37, 29, 16, 12, 10))
    assert tuning.choose(geom, device=0)['kernel'] == _native.FDTD_KERNEL_FUSED
    key = tuning._key(geom, tuning._device_name(0))
    (tmp_path / 'tune.json').write_text(json.dumps({key: {'kernel': 1, 'tile_y': 7, 'zchunk': 26,
                                                          'slab': 1, 'shell': 1}}))
    c = tuning.choose(geom, device=0)
    assert (c['tile_y'], c['zchunk'], c['slab'], c['shell']) == (7, 26, 1, _native.SHELL_SPLIT)
    assert tuning.choose(geom, kernel=_native.FDTD_KERNEL_SPLIT)['kernel'] == _native.FDTD_KERNEL_SPLIT

    class Fake:
        def __init__(self):
            self.opts = {}

        def set_option(self, k, v):
            self.opts[k] = v
    f = Fake()
    tuning.apply(f, c)
    assert f.opts == {_native.OPT_KERNEL: 1, _native.OPT_TILE_X: 32, _native.OPT_TILE_Y: 7,
                      _native.OPT_ZCHUNK: 26, _native.OPT_FUSED_SLAB: 1,
                      _native.OPT_SHELL: _native.SHELL_SPLIT}
    # the default choice sweeps the shell with the split passes
    assert tuning.choose(geom, kernel=_native.FDTD_KERNEL_FUSED)['shell'] == _native.SHELL_SPLIT


def test_incident_pulse_matches_reference():
    """The package's create_pulse (host) against the reference's pulse and
    spectrum (incidentbeam.py:174-199, fixture incident_hh_f32.npz)."""
    from fdtdsarsim_b200.incident import create_pulse, taper_radius
    from helpers import make_params
    g = np.load(os.path.join(GOLDEN, 'incident_hh_f32.npz'))
    pc = make_params(int(g['nx']), int(g['ny']), 60, 30, int(g['size_t_inc']), int(g['size_t_inc']))
    pc.geom_params.timestep = float(g['dt'])
    pc.geom_params.size_t_pulse = int(g['size_t_pulse'])
    pc.inc_beam_params.duration = float(g['duration'])
    pc.inc_beam_params.frequency = float(g['freq'])
    pc.inc_beam_params.illumination_width = float(g['illumination_width'])
    tv, pulse, pfft, pfreq = create_pulse(pc)
    assert np.array_equal(tv, g['time_vals']) and np.array_equal(pfreq, g['pulse_freqs'])
    assert np.max(np.abs(pulse - g['pulse'])) <= 1e-15
    assert np.max(np.abs(pfft - g['pulse_fft'])) <= 1e-12 * np.max(np.abs(g['pulse_fft']))
    assert taper_radius(pc) > 0


def test_process_results_host_stages_match_reference(tmp_path):
    """The host stages of process_results on a result file in the
    reference's layout (written through resultsio): far-field power
    (processresults.py:66-76), near-field Poynting power through every face
    (:83-93,128-257) and the scattering coefficient (:97-119) equal the
    reference's own values for the 31x39x39 flat-soil run bit for bit
    (fixture pipeline_cfg1.npz; the far field itself is the device
    transform's, tested on the GPU, so it is taken from the fixture)."""
    from fdtdsarsim_b200.processresults import (THETAS, backscatter, farfield_power,
                                                process_results)
    g = np.load(os.path.join(GOLDEN, 'pipeline_cfg1.npz'))
    for pol, (e, h) in (('h', ('e_phi', 'h_theta')), ('v', ('e_theta', 'h_phi'))):
        ph_h, ph_v = farfield_power(g['ff_e_theta'], g['ff_e_phi'], g['ff_h_theta'], g['ff_h_phi'])
        np.testing.assert_array_equal(ph_h if pol == 'h' else ph_v, g[f'ff_out_pwr_far_{pol}'])
    fname = str(tmp_path / 'flat.hdf5')
    planes = [k for k in g.files if '_ph_' in k or k.endswith('_inc_phasor')]
    assert len(planes) == 28
    with resultsio.File(fname, 'w') as f:
        pg = f.create_group('phasors')
        ny, nx = g['ex_ph_u'].shape
        pg.attrs['nx_phasor'], pg.attrs['ny_phasor'] = nx, ny
        pg.attrs['nz_phasor'] = g['ey_ph_l'].shape[0]
        for k in planes:
            pg.create_dataset(k, data=g[k])
        par = f.create_group('parameters')
        for k in g.files:
            if k.startswith('param_'):
                v = g[k][()]
                par.attrs[k[6:]] = str(v) if isinstance(v, np.str_) else v
        f.create_group('material_metadata')
        ff = f.create_group('farfield')
        for k in ('e_theta', 'e_phi', 'h_theta', 'h_phi', 'out_pwr_far_h', 'out_pwr_far_v'):
            ff.create_dataset(k, data=g[f'ff_{k}'])
        ff.attrs['theta_angles'] = THETAS
        ff.attrs['farfields_computed'] = True
    process_results(fname)
    with resultsio.File(fname, 'r') as f:
        nf = f['near_field_power'].attrs
        for k in g.files:
            if k.startswith('nfp_'):
                assert nf[k[4:]] == g[k][()], k
        for pol in ('h', 'v'):
            np.testing.assert_array_equal(f['scattering_coefficient'][f'scattering_coeff_{pol}'][()],
                                          g[f'scattering_coeff_{pol}'])
    theta = float(g['param_theta_angle'])
    key = 'ff_e_phi' if str(g['param_polarization']).upper() == 'HH' else 'ff_e_theta'
    idx = int(np.where(THETAS == -theta)[0][0])
    assert backscatter(fname) == complex(g[key][idx])
