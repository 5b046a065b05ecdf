"""Generate the golden fixtures in this folder by running the reference
package ``fdtdsarsim`` (wyatt-sfu/sar-pixel-simulator) on its CPU path.

The reference is imported from its checkout (``--reference PATH`` or the
``FDTDSARSIM_REFERENCE`` environment variable) with the in-memory
``h5py``/``matplotlib`` stand-ins of ``_refshims.py``; nothing of it is
copied. Run once, in a container that has the reference checked out:

    python tests/golden/make_golden.py --reference PATH [geom abs mat main n2f pipe inc matgen]

Outputs (all small, committed):
  geom_cases.json      set_geom_params results (parameters.py:242-305)
  absorbers.npz        1-D CPML b/c profiles (absorbers.py:35-189)
  materials.npz        compute_material_arrays (materials/materials.py:23-68)
  mainloop_*.npz       MainSimCpu.run fields + 24 phasor planes
                       (cpu/main_sim.py:39-195) on seeded random inputs
  near2far.npz         FarFieldTransform (near2far.py:28-112)
  pipeline_cfg1.npz    run_experiment end to end (experiment.py:41-97),
                       incident beam generation included
  material_gen.npz     the material generators (materials/roughsurface.py,
                       dielectricmodels.py, bubbles.py, soilmodels.py,
                       materials.py:112-164) on small seeded cases
  incident_*.npz       IncidentBeam.create_pulse / create_inc_excitation
                       (incidentbeam.py:174-298) and IncidentSimCpu
                       (cpu/incident_sim.py:22-171) on small geometries
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout (fdtdsarsim), from --reference PATH or the
# FDTDSARSIM_REFERENCE environment variable
REF = None
for _k, _a in enumerate(sys.argv[1:]):
    if _a.startswith('--reference='):
        REF = _a.split('=', 1)[1]
    elif _a == '--reference' and _k + 2 < len(sys.argv):
        REF = sys.argv[_k + 2]
REF = REF or os.environ.get('FDTDSARSIM_REFERENCE')
if not REF or not os.path.isdir(os.path.join(REF, 'fdtdsarsim')):
    sys.exit('make_golden.py: pass --reference PATH (or set FDTDSARSIM_REFERENCE) to the '
             'fdtdsarsim checkout')

sys.path.insert(0, HERE)
import _refshims  # noqa: E402

_refshims.install()
sys.path.insert(0, REF)

import scipy.constants  # noqa: E402
import fdtdsarsim as fdtd  # noqa: E402
from fdtdsarsim.absorbers import Absorbers  # noqa: E402
from fdtdsarsim.cpu.main_sim import MainSimCpu  # noqa: E402
from fdtdsarsim.materials.materials import compute_material_arrays  # noqa: E402
from fdtdsarsim.materials.materialmodel import MaterialModel  # noqa: E402
from fdtdsarsim.near2far import FarFieldTransform  # noqa: E402
from fdtdsarsim.parameters import (ParameterCollection, inc_filename,  # noqa: E402
                                   set_geom_params)

FREQ = 5.4e9
LAM = scipy.constants.c / FREQ

GEOM_FIELDS = ['cell_size', 'simulation_duration', 'timestep', 'size_t',
               'size_t_inc', 'size_t_pulse', 'size_x', 'size_y', 'size_z',
               'size_pml', 'size_z_material', 'tfsf_z', 'courant']

# (size_x, size_y, size_z_material, sim_duration, cell_size, unit,
#  material_fraction, incident_duration, frequency)
GEOM_CASES = [
    (2.0, 2.0, 0.5, 18.0, 0.05, 'wavelength', 0.7, 10.0, FREQ),
    (2.0, 2.0, 0.5, 18.0, 0.05, 'wavelength', 0.3, 10.0, FREQ),
    (8.0, 8.0, 1.5, 18.0, 0.021, 'wavelength', 0.7, 10.0, FREQ),
    (16.0, 16.0, 3.0, 18.0, 0.021, 'wavelength', 0.7, 10.0, FREQ),
    (4.0, 4.0, 1.0, 18.0, 0.03, 'wavelength', 0.7, 10.0, FREQ),
    (4.0, 4.0, 1.0, 18.0, 0.03, 'wavelength', 0.6, 10.0, FREQ),
    (2.0, 8.0, 0.5, 18.0, 0.03, 'wavelength', 0.4, 10.0, FREQ),
    (14.0, 14.0, 4.0, 16.0, 0.025, 'wavelength', 0.7, 8.0, FREQ),
    (0.3, 0.25, 0.08, 12.0, 0.004, 'metre', 0.5, 6.0, 1.2e9),
    (1.0, 1.0, 0.3, 3.0, 0.05, 'wavelength', 0.7, 10.0, FREQ),
]


def make_params(dtype='float32', project_dir='', threads=2):
    pc = ParameterCollection()
    pc.processing_params.processing_type = 'cpu'
    pc.processing_params.threads_per_proc = threads
    pc.processing_params.datatype = dtype
    pc.processing_params.project_dir = project_dir
    pc.inc_beam_params.frequency = FREQ
    pc.inc_beam_params.polarization = 'HH'
    pc.inc_beam_params.theta_angle = 20.0
    pc.inc_beam_params.phi_angle = 0.0
    pc.inc_beam_params.duration = 10.0
    pc.inc_beam_params.illumination_width = 2.0
    return pc


def gen_geom():
    out = []
    for case in GEOM_CASES:
        sx, sy, sz, dur, cs, unit, mf, incd, freq = case
        pc = make_params()
        pc.inc_beam_params.frequency = freq
        pc.inc_beam_params.duration = incd
        pc.material_params.material_fraction = mf
        set_geom_params(pc, sx, sy, sz, dur, cs, unit)
        g = {f: getattr(pc.geom_params, f) for f in GEOM_FIELDS}
        out.append({'args': list(case), 'geom': g})
    with open(os.path.join(HERE, 'geom_cases.json'), 'w') as f:
        json.dump(out, f, indent=1)


def raw_geom(pc, nx, ny, nz, tfsf_z, nt, ntp, cell_wl=0.021):
    g = pc.geom_params
    g.courant = 0.5
    g.size_pml = 10
    g.cell_size = LAM * cell_wl
    g.timestep = g.cell_size * g.courant / scipy.constants.c
    g.size_x, g.size_y, g.size_z = nx, ny, nz
    g.size_z_material = tfsf_z - 2
    g.tfsf_z = tfsf_z
    g.size_t = nt
    g.size_t_inc = ntp
    g.size_t_pulse = ntp // 2
    g.simulation_duration = 18.0


ABS_KEYS = ['be_d', 'bh_d', 'ce_d', 'ch_d', 'be_u', 'bh_u', 'ce_u', 'ch_u']


def gen_absorbers():
    out = {}
    for dtype in ('float32', 'float64'):
        for cell_wl in (0.021, 0.05):
            pc = make_params(dtype)
            raw_geom(pc, 25, 23, 27, 14, 10, 5, cell_wl)
            ab = Absorbers(pc)
            tag = f'{dtype}_{cell_wl}'
            out[f'{tag}_dx'] = pc.geom_params.cell_size
            out[f'{tag}_dt'] = pc.geom_params.timestep
            for k in ABS_KEYS:
                out[f'{tag}_{k}'] = np.ascontiguousarray(getattr(ab, k)[:, 0, 0])
            # the x- and y-face tiles must be the same 1-D profiles
            assert np.array_equal(ab.be_l[0, 0, :], ab.be_d[:, 0, 0])
            assert np.array_equal(ab.ch_b[0, :, 0], ab.ch_u[:, 0, 0])
    np.savez_compressed(os.path.join(HERE, 'absorbers.npz'), **out)


def random_model(rng, nz_mat, ny, nx, dtype):
    eps = rng.uniform(1.0, 20.0, size=(nz_mat, ny, nx)).astype(dtype)
    sig = rng.uniform(0.0, 0.3, size=(nz_mat, ny, nx)).astype(dtype)
    return eps, sig


def gen_materials():
    out = {}
    rng = np.random.default_rng(1234)
    for dtype in ('float32', 'float64'):
        pc = make_params(dtype)
        raw_geom(pc, 25, 23, 27, 14, 10, 5)
        eps, sig = random_model(rng, pc.geom_params.size_z_material, 23, 25,
                                dtype)
        ca, cb = compute_material_arrays(pc, MaterialModel(eps, sig, 1.0))
        out[f'{dtype}_eps'] = eps
        out[f'{dtype}_sigma'] = sig
        out[f'{dtype}_ca'] = ca
        out[f'{dtype}_cb'] = cb
        out[f'{dtype}_dx'] = pc.geom_params.cell_size
        out[f'{dtype}_dt'] = pc.geom_params.timestep
        out[f'{dtype}_nz'] = pc.geom_params.size_z
    np.savez_compressed(os.path.join(HERE, 'materials.npz'), **out)


PHASOR_NAMES = [
    'ex_ph_d', 'ey_ph_d', 'hx_ph_d', 'hy_ph_d',
    'ex_ph_u', 'ey_ph_u', 'hx_ph_u', 'hy_ph_u',
    'ey_ph_l', 'ez_ph_l', 'hy_ph_l', 'hz_ph_l',
    'ey_ph_r', 'ez_ph_r', 'hy_ph_r', 'hz_ph_r',
    'ex_ph_f', 'ez_ph_f', 'hx_ph_f', 'hz_ph_f',
    'ex_ph_b', 'ez_ph_b', 'hx_ph_b', 'hz_ph_b',
]


def gen_mainloop(tag, dtype, nx, ny, nz, tfsf_z, nt, ntp, seed, full_fields):
    """One MainSimCpu.run on seeded random materials and incident planes."""
    rng = np.random.default_rng(seed)
    with tempfile.TemporaryDirectory() as proj:
        pc = make_params(dtype, proj, threads=3)
        raw_geom(pc, nx, ny, nz, tfsf_z, nt, ntp)
        nz_mat = max(1, min(nz - 1, tfsf_z - 2))
        pc.geom_params.size_z_material = nz_mat
        eps, sig = random_model(rng, nz_mat, ny, nx, dtype)
        ca, cb = compute_material_arrays(pc, MaterialModel(eps, sig, 1.0))
        inc = {}
        for comp, scale in (('ex', 1.0), ('ey', 1.0),
                            ('hx', 1 / 376.73), ('hy', 1 / 376.73)):
            inc[comp] = (scale * rng.standard_normal((ntp, ny, nx))).astype(dtype)
        import h5py
        with h5py.File(inc_filename(pc), 'w') as f:
            for comp in ('ex', 'ey', 'hx', 'hy'):
                f.create_dataset(comp, data=inc[comp])
            g = f.create_group('phasors')
            for comp in ('ex', 'ey', 'hx', 'hy'):
                g.create_dataset(f'{comp}_inc_phasor',
                                 data=np.zeros((ny - 20, nx - 20), 'complex64'))
        sim = MainSimCpu(pc, mpi=True)
        sim.run(ca, cb, 'case', {'seed': seed})
        out = {'nx': nx, 'ny': ny, 'nz': nz, 'tfsf_z': tfsf_z, 'nt': nt,
               'ntp': ntp, 'dx': pc.geom_params.cell_size,
               'dt': pc.geom_params.timestep, 'freq': FREQ, 'seed': seed,
               'ca': ca, 'cb': cb}
        for comp in ('ex', 'ey', 'hx', 'hy'):
            out[f'inc_{comp}'] = inc[comp]
        for comp in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
            fld = getattr(sim, comp)
            if full_fields:
                out[f'field_{comp}'] = fld
            else:
                out[f'field_{comp}_sum'] = np.sum(fld, dtype=np.float64)
                out[f'field_{comp}_abssum'] = np.sum(np.abs(fld), dtype=np.float64)
                out[f'field_{comp}_plane'] = fld[nz // 2]
        for name in PHASOR_NAMES:
            out[name] = getattr(sim, name)
    np.savez_compressed(os.path.join(HERE, f'mainloop_{tag}.npz'), **out)


def gen_near2far():
    rng = np.random.default_rng(77)
    ny_ph, nx_ph, nz_ph = 29, 31, 15
    ph = {}
    for name in ('ex_ph_u', 'ey_ph_u', 'hx_ph_u', 'hy_ph_u'):
        scale = 1.0 if name[0] == 'e' else 1 / 376.73
        ph[name] = (scale * (rng.standard_normal((ny_ph, nx_ph))
                             + 1j * rng.standard_normal((ny_ph, nx_ph)))
                    ).astype('complex64')
    dx = 0.021 * LAM
    thetas = np.linspace(-80.0, 80.0, num=161, endpoint=True)
    phis = np.asarray([0.0])
    ff = FarFieldTransform()(ph, nx_ph, ny_ph, nz_ph, dx, 2.0e3, thetas,
                             phis, FREQ)
    out = dict(ph)
    out.update({'nx': nx_ph, 'ny': ny_ph, 'nz': nz_ph, 'dx': dx, 'r': 2.0e3,
                'freq': FREQ, 'thetas': thetas, 'phis': phis})
    for k, v in ff.items():
        out[f'ff_{k}'] = v
    # a second azimuth exercises the sin(phi) terms
    ff2 = FarFieldTransform()(ph, nx_ph, ny_ph, nz_ph, dx, 2.0e3, thetas,
                              np.asarray([35.0]), FREQ)
    for k, v in ff2.items():
        out[f'ff35_{k}'] = v
    np.savez_compressed(os.path.join(HERE, 'near2far.npz'), **out)


def gen_pipeline_cfg1():
    """run_experiment on the smallest valid variant of the 2x2 wavelength,
    flat-soil configuration (material_fraction 0.3 -> 31x39x39)."""
    import h5py
    from fdtdsarsim.materials.materials import flat_surface
    with tempfile.TemporaryDirectory() as proj:
        params_json = {
            'processing_type': 'cpu', 'threads_per_proc': 8,
            'datatype': 'float32', 'project_dir': proj,
            'frequency_hz': FREQ, 'polarization': 'HH',
            'theta_angle_deg': 20.0, 'phi_angle_deg': 0.0,
            'incident_duration': 10.0, 'illumination_width': 2.0,
            'generate_new': False,
            'size_x': 2.0, 'size_y': 2.0, 'size_z_material': 0.5,
            'simulation_duration': 18.0, 'cell_size': 0.05,
            'unit': 'wavelength', 'material_fraction': 0.3,
            'disp_inc_results': False, 'disp_inc_sim_movie': False,
            'disp_debug': False, 'disp_main_sim_movie': False,
            'disp_materials': False,
        }
        jpath = os.path.join(proj, 'params.json')
        with open(jpath, 'w') as f:
            json.dump(params_json, f)
        pc = fdtd.load_from_json(jpath)
        mats = flat_surface(pc, 6.0, 0.01, name='flat')
        fdtd.run_experiment(pc, mats)
        out = {'params_json': json.dumps(params_json)}
        with h5py.File(inc_filename(pc), 'r') as f:
            for comp in ('ex', 'ey', 'hx', 'hy'):
                d = f[comp][:]
                out[f'inc_{comp}_sum'] = np.sum(d, dtype=np.float64)
                out[f'inc_{comp}_abssum'] = np.sum(np.abs(d), dtype=np.float64)
                out[f'inc_{comp}_t150'] = d[150]
                out[f'inc_{comp}_t300'] = d[300]
            for comp in ('ex', 'ey', 'hx', 'hy'):
                out[f'{comp}_inc_phasor'] = f['phasors'][f'{comp}_inc_phasor'][:]
        res = os.path.join(proj, 'results', 'flat.hdf5')
        with h5py.File(res, 'r') as f:
            for name in PHASOR_NAMES:
                out[name] = f['phasors'][name][:]
            for k in ('e_theta', 'e_phi', 'h_theta', 'h_phi',
                      'out_pwr_far_h', 'out_pwr_far_v'):
                out[f'ff_{k}'] = f['farfield'][k][:]
            for k, v in f['near_field_power'].attrs.items():
                out[f'nfp_{k}'] = v
            for k in ('scattering_coeff_h', 'scattering_coeff_v'):
                out[k] = f['scattering_coefficient'][k][:]
            for k, v in f['parameters'].attrs.items():
                out[f'param_{k}'] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, 'pipeline_cfg1.npz'), **out)


# (tag, dtype, pol, theta, phi, size_x, size_y, duration, store_full_excitation)
INCIDENT_CASES = [
    ('hh_f32', 'float32', 'HH', 20.0, 0.0, 1.5, 1.5, 2.0, True),
    ('vv_f64', 'float64', 'VV', 35.0, 30.0, 1.3, 1.6, 2.0, False),
]


def gen_incident(tag, dtype, pol, theta, phi, sx, sy, duration, full):
    """The incident beam of a small geometry: the temporal pulse, the
    excitation fed into the incident simulation, and the planes and phasors
    that simulation records."""
    from fdtdsarsim.cpu.incident_sim import IncidentSimCpu
    from fdtdsarsim.incidentbeam import IncidentBeam
    import h5py
    with tempfile.TemporaryDirectory() as proj:
        pc = make_params(dtype, proj, threads=3)
        pc.inc_beam_params.polarization = pol
        pc.inc_beam_params.theta_angle = theta
        pc.inc_beam_params.phi_angle = phi
        pc.inc_beam_params.duration = duration
        pc.inc_beam_params.illumination_width = 0.8 * sx
        pc.material_params.material_fraction = 0.5
        set_geom_params(pc, sx, sy, 0.5, 18.0, 0.05, 'wavelength')
        g = pc.geom_params
        beam = IncidentBeam(pc)
        beam.create_pulse()
        pulse_ex, pulse_ey = beam.create_inc_excitation()
        sim = IncidentSimCpu(pc)
        sim.run(pulse_ex, pulse_ey)
        ntp, npulse = g.size_t_inc, g.size_t_pulse
        out = {'dtype': dtype, 'pol': pol, 'theta': theta, 'phi': phi,
               'freq': pc.inc_beam_params.frequency, 'duration': duration,
               'illumination_width': pc.inc_beam_params.illumination_width,
               'nx': g.size_x, 'ny': g.size_y, 'nz_inc': sim.params.geom_params.size_z,
               'npml': g.size_pml, 'dx': g.cell_size, 'dt': g.timestep,
               'size_t_inc': ntp, 'size_t_pulse': npulse,
               'time_vals': beam.time_vals, 'pulse': beam.pulse,
               'pulse_fft': beam.pulse_fft, 'pulse_freqs': beam.pulse_freqs}
        exi, eyi = np.imag(pulse_ex), np.imag(pulse_ey)
        if full:
            out['exc_ex_imag'] = exi[:npulse]
            out['exc_ey_imag'] = eyi[:npulse]
        steps = np.arange(0, npulse, 7)
        out['exc_steps'] = steps
        out['exc_ex_imag_at'] = exi[steps]
        out['exc_ey_imag_at'] = eyi[steps]
        out['exc_ex_real_at'] = np.real(pulse_ex)[steps]
        out['exc_absmax'] = max(np.abs(pulse_ex).max(), np.abs(pulse_ey).max())
        with h5py.File(inc_filename(pc), 'r') as f:
            rec = np.arange(0, ntp, 6)
            out['rec_steps'] = rec
            for comp in ('ex', 'ey', 'hx', 'hy'):
                d = f[comp][:]
                out[f'inc_{comp}_at'] = d[rec]
                out[f'inc_{comp}_stepsum'] = np.sum(d, axis=(1, 2), dtype=np.float64)
                out[f'{comp}_inc_phasor'] = f['phasors'][f'{comp}_inc_phasor'][:]
    np.savez_compressed(os.path.join(HERE, f'incident_{tag}.npz'), **out)


def gen_material_generators():
    """Seeded runs of the reference's material generators. rough_dielectric
    draws unseeded surfaces; it is run with gaussian_correlated_surface
    wrapped to seeds 300 + i (the port takes those seeds as an argument)."""
    import fdtdsarsim.materials.materials as rm
    from fdtdsarsim.materials import bubbles, dielectricmodels as dm, roughsurface as rs, soilmodels as sm
    out = {}
    dx = 0.003
    out['gcs'] = rs.gaussian_correlated_surface(41, 37, dx, 0.010, 0.015, 0.002, seed=11)
    out['gcs_rabus'] = rs.gaussian_correlated_surface(41, 37, dx, 0.010, 0.015, 0.002, seed=11,
                                                      rabus_compat=True)
    out['gcs_fast'] = rs.gaussian_correlated_surface_fast(41, 37, dx, 0.010, 0.015, 0.002,
                                                          np.random.default_rng(12))
    out['two_layer'] = rs.two_layer_gaussian_correlated_surface(41, 37, dx, 0.010, 0.012, 0.002,
                                                                0.6, seed=13)
    out['two_layer_full'] = rs.two_layer_gaussian_correlated_surface(41, 37, dx, 0.010, 0.012,
                                                                     0.002, 1.0, seed=14)
    cases = np.array([(mv, sand, clay, f) for mv in (0.05, 0.2, 0.41)
                      for sand, clay in ((0.3, 0.2), (0.6, 0.1))
                      for f in (1.4e9, 5.4e9, 9.7e9, 18e9)])
    out['hall_cases'] = cases
    model = dm.HallikainenSoilModel()
    out['hall_class'] = np.array([model.get_epsilon(*c) for c in cases])
    out['hall_func'] = np.array([dm.hallikainen_soil_model(*c) for c in cases])
    pc = make_params('float32')
    raw_geom(pc, 23, 21, 30, 20, 10, 5)
    g = pc.geom_params
    g.size_z_material = 12
    g.cell_size = dx
    orig = rm.gaussian_correlated_surface
    seeds = iter(range(300, 400))
    rm.gaussian_correlated_surface = lambda *a, **k: orig(*a, seed=next(seeds), **k)
    try:
        for i, m in enumerate(rm.rough_dielectric(pc, 7.0, 0.03, 0.004, 0.02, 0.01, 2)):
            out[f'rough_{i}_eps'] = m.relative_permittivity
            out[f'rough_{i}_sig'] = m.conductivity
    finally:
        rm.gaussian_correlated_surface = orig
    for tag, gen in (
            ('one', sm.one_layer_gaussian(pc, [0.1, 0.3], 0.4, 0.2, 0.004, 0.01, 0.02, 2, 21)),
            ('one_groove', sm.one_layer_gaussian(pc, [0.2], 0.4, 0.2, 0.004, 0.01, 0.02, 1, 22,
                                                 grooved=True, rabus_compat=True)),
            ('two', sm.two_layer_gaussian(pc, 0.15, [0.3, 0.35], 0.5, 0.1, 0.003, 0.01, 0.7,
                                          0.025, 0.01, 1, 23)),
            ('grad', sm.gradient_gaussian(pc, 0.1, [0.35], 0.5, 0.1, 0.003, 0.01, 0.7,
                                          0.025, 0.01, 1, 24)),
            ('grad_groove', sm.gradient_gaussian(pc, 0.1, [0.3], 0.5, 0.1, 0.003, 0.01, 0.7,
                                                 0.025, 0.01, 1, 25, grooved=True))):
        for i, m in enumerate(gen):
            out[f'{tag}_{i}_eps'] = m.relative_permittivity
            out[f'{tag}_{i}_sig'] = m.conductivity
            out[f'{tag}_{i}_name'] = m.name
    # bubbles in a one-layer model with a flat surface at 9 cells
    surf = np.full((21, 23), 9.0)
    for tag, fn, args in (('bub', bubbles.add_bubbles, (0.15, 0.0065, 3.2, 0.0, 31)),
                          ('bub_rand', bubbles.add_bubbles_randsize, (0.15, 0.004, 0.008, 3.2, 0.0, 32))):
        m = next(sm.one_layer_gaussian(pc, [0.2], 0.4, 0.2, 0.0, 0.01, 0.03, 1, 26))
        eps = np.where(np.arange(12)[:, None, None] <= 9, m.relative_permittivity[0, 0, 0], 1.0)
        sig = np.where(np.arange(12)[:, None, None] <= 9, m.conductivity[0, 0, 0], 0.0)
        m.relative_permittivity = np.broadcast_to(eps, (12, 21, 23)).astype(np.float32).copy()
        m.conductivity = np.broadcast_to(sig, (12, 21, 23)).astype(np.float32).copy()
        m.metadata = {}
        out[f'{tag}_in_eps'] = m.relative_permittivity.copy()
        out[f'{tag}_in_sig'] = m.conductivity.copy()
        r = fn(m, surf, *args)
        out[f'{tag}_eps'] = r.relative_permittivity
        out[f'{tag}_sig'] = r.conductivity
    out['bub_surf'] = surf
    np.savez_compressed(os.path.join(HERE, 'material_gen.npz'), **out)


if __name__ == '__main__':
    args = [a for k, a in enumerate(sys.argv[1:])
            if not a.startswith('--reference') and not (k > 0 and sys.argv[k] == '--reference')]
    which = args or ['geom', 'abs', 'mat', 'main', 'n2f', 'pipe', 'inc', 'matgen']
    if 'geom' in which:
        gen_geom()
    if 'abs' in which:
        gen_absorbers()
    if 'mat' in which:
        gen_materials()
    if 'main' in which:
        gen_mainloop('f32', 'float32', 25, 23, 27, 14, 60, 40, 11, True)
        gen_mainloop('f32_tfsf_in_pml', 'float32', 27, 25, 23, 20, 45, 30,
                     12, True)
        gen_mainloop('f64', 'float64', 25, 23, 27, 14, 40, 20, 13, False)
    if 'n2f' in which:
        gen_near2far()
    if 'pipe' in which:
        gen_pipeline_cfg1()
    if 'inc' in which:
        for case in INCIDENT_CASES:
            gen_incident(*case)
    if 'matgen' in which:
        gen_material_generators()
