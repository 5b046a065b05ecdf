"""Post-processing of result files (fdtdsarsim/processresults.py:15-271).

The far-field transform runs on the device; near-field Poynting power and
the scattering coefficient are small host reductions kept in numpy/scipy
with the reference's integration rule.
"""
import glob
import os.path
from typing import Mapping

import numpy as np
import scipy.integrate

from . import resultsio
from .near2far import FarFieldTransform

RADIUS = 2.0e3
THETAS = np.linspace(-80.0, 80.0, num=161, endpoint=True)


def process_all_results(project_dir: str, debug_plots=False):
    """Process every result file of a project (processresults.py:15-22)."""
    for fname in sorted(glob.glob(os.path.join(project_dir, 'results', '*.hdf5'))):
        process_results(fname, debug_plots)


def farfield_power(e_theta, e_phi, h_theta, h_phi):
    """(horizontal, vertical) scattered power (processresults.py:260-271)."""
    out_h = 0.5 * np.real(-e_phi * np.conj(h_theta))
    out_v = 0.5 * np.real(e_theta * np.conj(h_phi))
    return out_h, out_v


def _poynting(E, H, normal):
    return np.dot(np.real(0.5 * np.cross(E, np.conj(H))), np.asarray(normal))


def _int2(f, dx):
    return scipy.integrate.simpson(scipy.integrate.simpson(f, dx=dx, axis=1), dx=dx, axis=0)


def near_field_power(phasors: Mapping, dx: float, size_z_material: int):
    """Poynting power through the internal faces (processresults.py:128-257)."""
    p = {k: np.asarray(phasors[k]) for k in phasors.keys()}
    z = np.zeros_like
    power = {}
    E = np.stack([p['ex_inc_phasor'], p['ey_inc_phasor'], z(p['ey_inc_phasor'])], axis=-1)
    H = np.stack([p['hx_inc_phasor'], p['hy_inc_phasor'], z(p['hy_inc_phasor'])], axis=-1)
    power['incident'] = _int2(_poynting(E, H, [0.0, 0.0, -1.0]), dx)
    sides = {
        'left': (lambda s: (z(p['ey_ph_' + s]), p['ey_ph_' + s], p['ez_ph_' + s]),
                 lambda s: (z(p['hy_ph_' + s]), p['hy_ph_' + s], p['hz_ph_' + s]),
                 'l', [-1.0, 0.0, 0.0]),
        'right': (lambda s: (z(p['ey_ph_' + s]), p['ey_ph_' + s], p['ez_ph_' + s]),
                  lambda s: (z(p['hy_ph_' + s]), p['hy_ph_' + s], p['hz_ph_' + s]),
                  'r', [1.0, 0.0, 0.0]),
        'front': (lambda s: (p['ex_ph_' + s], z(p['ex_ph_' + s]), p['ez_ph_' + s]),
                  lambda s: (p['hx_ph_' + s], z(p['hx_ph_' + s]), p['hz_ph_' + s]),
                  'f', [0.0, -1.0, 0.0]),
        'back': (lambda s: (p['ex_ph_' + s], z(p['ex_ph_' + s]), p['ez_ph_' + s]),
                 lambda s: (p['hx_ph_' + s], z(p['hx_ph_' + s]), p['hz_ph_' + s]),
                 'b', [0.0, 1.0, 0.0]),
    }
    for name, (ef, hf, s, nrm) in sides.items():
        flux = _poynting(np.stack(ef(s), axis=-1), np.stack(hf(s), axis=-1), nrm)
        power[f'{name}_bottom'] = _int2(flux[0:size_z_material, :], dx)
        power[f'{name}_top'] = _int2(flux[size_z_material:-1, :], dx)
    for name, s, nrm in (('down', 'd', [0.0, 0.0, -1.0]), ('up', 'u', [0.0, 0.0, 1.0])):
        E = np.stack([p['ex_ph_' + s], p['ey_ph_' + s], z(p['ex_ph_' + s])], axis=-1)
        H = np.stack([p['hx_ph_' + s], p['hy_ph_' + s], z(p['hx_ph_' + s])], axis=-1)
        power[name] = _int2(_poynting(E, H, nrm), dx)
    power['top_total'] = power['up'] + power['left_top'] + power['right_top'] \
        + power['front_top'] + power['back_top']
    power['bottom_total'] = power['down'] + power['left_bottom'] + power['right_bottom'] \
        + power['front_bottom'] + power['back_bottom']
    return power


def simpson_weights(n, dx):
    """The weights scipy.integrate.simpson applies to n samples spaced dx:
    the integral of each unit vector (so even n gets scipy's own end
    correction)."""
    return scipy.integrate.simpson(np.eye(n), dx=dx, axis=1)


_NF_KEYS = ('incident', 'left_bottom', 'left_top', 'right_bottom', 'right_top', 'front_bottom',
            'front_top', 'back_bottom', 'back_top', 'down', 'up')


def near_field_power_device(native, inc_phasors: Mapping, dx: float, size_z_material: int):
    """near_field_power from a simulation's phasors on the device
    (fdtd_near_field_power: the flux formed in float64, summed with the
    Simpson weights scipy applies); same keys as near_field_power. native:
    the simulation's NativeSim, after its run."""
    nx, ny, nz = native.nx_ph, native.ny_ph, native.nz_ph
    szm = int(size_z_material)
    w = np.concatenate([simpson_weights(ny, dx), simpson_weights(nx, dx), simpson_weights(szm, dx),
                        simpson_weights(nz - 1 - szm, dx)])
    vals = native.near_field_power(inc_phasors, szm, w)
    power = dict(zip(_NF_KEYS, (float(v) for v in vals)))
    power['top_total'] = power['up'] + power['left_top'] + power['right_top'] \
        + power['front_top'] + power['back_top']
    power['bottom_total'] = power['down'] + power['left_bottom'] + power['right_bottom'] \
        + power['front_bottom'] + power['back_bottom']
    return power


def scattering_coefficient(out_pwr_far, incident_power, nx_phasor, ny_phasor, dx):
    """Far-field power normalised by the incident power through the
    illuminated area, times 4 pi r^2 (processresults.py:103-119)."""
    pwr = np.asarray(out_pwr_far) / incident_power
    return pwr * 4.0 * np.pi * (RADIUS ** 2) / (nx_phasor * ny_phasor * dx * dx)


def process_results(filename: str, debug_plots=False, device=0):
    """Far field, near-field power and scattering coefficient of one result
    file, written back into it (processresults.py:25-125)."""
    with resultsio.File(filename, 'r+') as results:
        pg = results['parameters']
        ph = results['phasors']
        dx = pg.attrs['cell_size']
        size_z_material = pg.attrs['size_z_material']
        nx_ph, ny_ph, nz_ph = ph.attrs['nx_phasor'], ph.attrs['ny_phasor'], ph.attrs['nz_phasor']
        ff_grp = results['farfield'] if 'farfield' in results else results.create_group('farfield')
        if 'farfields_computed' not in ff_grp.attrs:
            phis = np.asarray([pg.attrs['phi_angle']])
            freq = pg.attrs['frequency']
            ff = FarFieldTransform(device)(ph, nx_ph, ny_ph, nz_ph, dx, RADIUS, THETAS, phis, freq)
            for src, dst in (('E_theta', 'e_theta'), ('E_phi', 'e_phi'),
                             ('H_theta', 'h_theta'), ('H_phi', 'h_phi')):
                ff_grp.create_dataset(dst, data=ff[src])
            ff_grp.attrs['theta_angles'] = THETAS
            ff_grp.attrs['phi_angles'] = phis
            ff_grp.attrs['radius'] = RADIUS
            ph_h, ph_v = farfield_power(ff['E_theta'], ff['E_phi'], ff['H_theta'], ff['H_phi'])
            ff_grp.create_dataset('out_pwr_far_h', data=ph_h)
            ff_grp.create_dataset('out_pwr_far_v', data=ph_v)
            ff_grp.attrs['farfields_computed'] = True
        nf_grp = results['near_field_power'] if 'near_field_power' in results \
            else results.create_group('near_field_power')
        if 'powers_computed' not in nf_grp.attrs:
            for k, v in near_field_power(ph, dx, size_z_material).items():
                nf_grp.attrs[k] = v
            nf_grp.attrs['powers_computed'] = True
        sc_grp = results['scattering_coefficient'] if 'scattering_coefficient' in results \
            else results.create_group('scattering_coefficient')
        if 'scattering_computed' not in sc_grp.attrs:
            inp = nf_grp.attrs['incident']
            for pol in ('h', 'v'):
                sc_grp.create_dataset(f'scattering_coeff_{pol}', data=scattering_coefficient(
                    ff_grp[f'out_pwr_far_{pol}'][()], inp, nx_ph, ny_ph, dx))
            sc_grp.attrs['scattering_computed'] = True


def backscatter(filename: str):
    """Backscatter phasor: far field at theta = -theta_inc, E_phi for HH and
    E_theta for VV (release_examples/cuda_example/gather.py:39-53)."""
    with resultsio.File(filename, 'r') as f:
        inc = f['parameters'].attrs['theta_angle']
        pol = str(f['parameters'].attrs['polarization'])
        angles = np.asarray(f['farfield'].attrs['theta_angles'])
        idx = int(np.squeeze(np.where(angles == -inc)))
        key = 'e_phi' if pol.upper() == 'HH' else 'e_theta'
        return complex(np.asarray(f['farfield'][key][()])[idx])
