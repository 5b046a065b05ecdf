"""MainSimGpu: the drop-in for the reference's GPU simulator class
(fdtdsarsim/gpu/main_sim.py:42-825), backed by libfdtd_b200.

Same constructor and ``run`` signature and the same behaviour around them:
``run`` casts Ca/Cb to the simulation dtype, skips the model when its
result file exists, otherwise zeroes the state, runs ``size_t`` steps and
writes ``results/<name>.hdf5`` with the reference's layout. The incident
beam is uploaded to device memory once per simulator and stays resident
across models (the reference re-reads a slice from HDF5 every step).
"""
import dataclasses
import logging
import time

import numpy as np
import scipy.constants

from .. import _native, resultsio
from ..absorbers import packed_profiles
from ..parameters import ParameterCollection, inc_filename, results_filename

logger = logging.getLogger(__name__)

PHASOR_NAMES = _native.PHASOR_NAMES


def native_geometry(params: ParameterCollection) -> _native.Geometry:
    """fdtd_geometry of a parameter set, with the update scalars rounded to
    the simulation dtype as the reference rounds them (cpu/main_sim.py:
    116-130: np_type(dt / (mu0 * dx)), np_type(dt / mu0),
    np_type(dt / (e0 * dx)) with scipy.constants eps0/mu0)."""
    g = params.geom_params
    dtype = params.processing_params.datatype
    if dtype == 'float32':
        np_type = np.float32
    elif dtype == 'float64':
        np_type = np.float64
    else:
        raise ValueError('Invalid dtype specifier')
    dt, dx = g.timestep, g.cell_size
    mu0, e0 = scipy.constants.mu_0, scipy.constants.epsilon_0
    return _native.Geometry(
        nx=g.size_x, ny=g.size_y, nz=g.size_z, npml=g.size_pml, tfsf_z=g.tfsf_z,
        nt=g.size_t, nt_inc=g.size_t_inc, dtype=_native.dtype_code(dtype),
        cell_size=dx, timestep=dt, frequency=params.inc_beam_params.frequency,
        db=float(np_type(dt / (mu0 * dx))), dtm0=float(np_type(dt / mu0)),
        dte0dx=float(np_type(dt / (e0 * dx))))


def _device_of(params):
    gpu = params.processing_params.gpu_num
    if isinstance(gpu, (list, tuple)):
        gpu = gpu[0] if gpu else 0
    return int(gpu)


class MainSimGpu:
    """Runs one material model per ``run`` call on one B200."""

    # With True, save_results also writes the near-field power computed on
    # the device from the resident phasors (fdtd_near_field_power; float64
    # flux, equal to the reference's host evaluation to rounding), and
    # process_results keeps it; with False (the default) process_results
    # evaluates it on the host from the file, bit for bit as the reference.
    device_postprocess = False

    def __init__(self, params: ParameterCollection, mpi=False, kernel=None, tile=None):
        self.params = params
        self.mpi = mpi
        self.gpu_num = _device_of(params)
        self.dtype = np.dtype(params.processing_params.datatype)
        if self.dtype not in (np.float32, np.float64):
            raise ValueError('Invalid dtype specifier')
        self.geom = native_geometry(params)
        self.native = _native.NativeSim(self.geom, self.gpu_num)
        self.native.set_absorbers(packed_profiles(params))
        self._configure(kernel, tile)
        self._incident_loaded = None
        g = params.geom_params
        self.nx_ph = g.size_x - 2 * g.size_pml
        self.ny_ph = g.size_y - 2 * g.size_pml
        self.nz_ph = g.size_z - 2 * g.size_pml

    def _configure(self, kernel, tile):
        from .. import tuning
        choice = tuning.choose(self.geom, kernel=kernel, tile=tile, device=self.gpu_num)
        tuning.apply(self.native, choice)
        self.kernel_choice = choice

    # -- incident beam ----------------------------------------------------
    def load_incident(self, ex, ey, hx, hy, inc_phasors=None):
        """Upload an incident beam (four (size_t_inc, ny, nx) arrays) that
        stays on the device for every following ``run``."""
        self.native.set_incident(ex, ey, hx, hy)
        self._incident_loaded = 'arrays'
        self._inc_phasors = inc_phasors

    def use_incident_run(self, run, phasors) -> bool:
        """Take the planes of an incident run still on the device (the
        IncidentSimGpu that IncidentBeam.setup made) device to device; False,
        with nothing changed, when its grid, element type or device does not
        fit this simulation. The caller keeps and closes the run."""
        g = run.native.geom
        if (g.nx, g.ny, g.dtype) != (self.geom.nx, self.geom.ny, self.geom.dtype) or \
                g.nt < self.geom.nt_inc:
            return False
        try:
            self.native.set_incident_from(run.native)   # checks the device too
        except _native.FdtdError:
            return False   # another device: the caller reads the file
        self._inc_phasors = {k: np.asarray(v) for k, v in phasors.items()}
        self._incident_loaded = inc_filename(self.params)
        return True

    def _ensure_incident(self):
        if self._incident_loaded is not None:
            return
        fname = inc_filename(self.params)
        from ..incident import take_resident
        held = take_resident(fname)
        if held is not None:
            # the beam IncidentBeam.setup just made in this process: copy its
            # planes device to device instead of reading the file back
            run, phasors = held
            try:
                if self.use_incident_run(run, phasors):
                    return
            finally:
                run.close()
        self._load_incident_file(fname)

    def _load_incident_file(self, fname):
        from ..incident import wait_written
        wait_written(fname)                 # a file this process is still writing
        with resultsio.File(fname, 'r') as f:
            comps = [np.asarray(f[c][:], dtype=self.dtype) for c in ('ex', 'ey', 'hx', 'hy')]
            self._inc_phasors = {f'{c}_inc_phasor': np.asarray(f['phasors'][f'{c}_inc_phasor'][:])
                                 for c in ('ex', 'ey', 'hx', 'hy')}
        self.native.set_incident(*comps)
        self._incident_loaded = fname

    # -- time stepping ----------------------------------------------------
    def reset(self):
        self.native.reset()

    def step(self, nsteps):
        self.native.run(nsteps)

    def simulate(self, Ca, Cb):
        """Zero the state, upload Ca/Cb and run all ``size_t`` steps."""
        self.native.reset()
        self.native.set_materials(Ca, Cb)
        self._ensure_incident()
        self.native.run(self.params.geom_params.size_t)
        self.native.synchronize()

    def simulate_eps_sigma(self, eps_r, sigma):
        """As simulate, with Ca/Cb computed on the device from the material
        block's relative permittivity and conductivity (vacuum above it),
        bit-identical to compute_material_arrays."""
        self.native.reset()
        self.native.set_materials_eps_sigma(eps_r, sigma)
        self._ensure_incident()
        self.native.run(self.params.geom_params.size_t)
        self.native.synchronize()

    def simulate_layered(self, recipe):
        """As simulate, with the material block made on the device from a
        LayeredMaterial recipe (fdtd_fill_layers, fdtd_paint_spheres) and
        Ca/Cb computed from it."""
        self.native.reset()
        recipe.stage(self.native)
        self.native.set_materials_staged()
        self._ensure_incident()
        self.native.run(self.params.geom_params.size_t)
        self.native.synchronize()

    def run_layered(self, recipe):
        """run() for a material model given as a LayeredMaterial recipe
        (materials/device.py): the device fills the block, so it is never
        made on the host nor uploaded; the result file is the one
        run_eps_sigma writes for recipe.to_model()."""
        g = self.params.geom_params
        want = (g.size_z_material, g.size_y, g.size_x)
        if tuple(recipe.shape) != want:
            raise ValueError(f'material block is {tuple(recipe.shape)}, expected {want}')
        self.Ca = self.Cb = None
        self._run_and_save(lambda: self.simulate_layered(recipe), recipe.name, recipe.metadata)

    def run(self, Ca: np.ndarray, Cb: np.ndarray, material_name: str, material_meta: dict):
        """Simulate one material model and save its phasors
        (gpu/main_sim.py:74-115)."""
        self.Ca = np.asarray(Ca, dtype=self.dtype)
        self.Cb = np.asarray(Cb, dtype=self.dtype)
        self._run_and_save(lambda: self.simulate(self.Ca, self.Cb), material_name, material_meta)

    def run_eps_sigma(self, eps_r: np.ndarray, sigma: np.ndarray, material_name: str,
                      material_meta: dict):
        """run() for a material block given as (size_z_material, ny, nx)
        relative permittivity and conductivity: the update coefficients are
        computed on the device instead of by compute_material_arrays on the
        host (same values bit for bit, a fraction of the host's time and
        0.7x the upload)."""
        if np.shape(eps_r) != np.shape(sigma):
            raise RuntimeError('Permittivity and conductivity arrays have different shapes')
        g = self.params.geom_params
        want = (g.size_z_material, g.size_y, g.size_x)
        if tuple(np.shape(eps_r)) != want:
            raise ValueError(f'material block is {tuple(np.shape(eps_r))}, expected {want}')
        self.Ca = self.Cb = None
        self._run_and_save(lambda: self.simulate_eps_sigma(eps_r, sigma), material_name,
                           material_meta)

    def _run_and_save(self, simulate, material_name, material_meta):
        logger.info('Starting a GPU FDTD simulation of %s on GPU %s', material_name, self.gpu_num)
        t0 = time.monotonic()
        out_name = results_filename(self.params, material_name)
        if not resultsio.exists(out_name):
            simulate()
            self.save_results(material_name, material_meta)
        else:
            logger.info('%s already exists, skipping', out_name)
        logger.info('Simulation of %s on GPU %s is complete (%.3fs)', material_name,
                    self.gpu_num, time.monotonic() - t0)

    def phasors(self):
        return self.native.get_phasors()

    def fields(self):
        return self.native.get_fields()

    def save_results(self, material_name, material_meta):
        """Write phasors, parameters and metadata (gpu/main_sim.py:387-449)."""
        out_filename = results_filename(self.params, material_name)
        if resultsio.exists(out_filename):
            raise RuntimeError('Overwriting a previous simulation. This is probably bad!')
        ph = self.native.get_phasors()
        if self._incident_loaded is None:
            self._ensure_incident()
        with resultsio.File(out_filename, 'w') as out:
            pg = out.create_group('phasors')
            parg = out.create_group('parameters')
            mg = out.create_group('material_metadata')
            pg.attrs['nx_phasor'] = self.nx_ph
            pg.attrs['ny_phasor'] = self.ny_ph
            pg.attrs['nz_phasor'] = self.nz_ph
            for name in PHASOR_NAMES:
                pg.create_dataset(name, data=ph[name])
            inc_ph = self._inc_phasors or {}
            for c in ('ex', 'ey', 'hx', 'hy'):
                key = f'{c}_inc_phasor'
                val = inc_ph.get(key)
                if val is None:
                    val = np.zeros((self.ny_ph, self.nx_ph), ph['ex_ph_u'].dtype)
                pg.create_dataset(key, data=val)
            for grp in dataclasses.fields(self.params):
                obj = getattr(self.params, grp.name)
                for f in dataclasses.fields(obj):
                    parg.attrs[f.name] = getattr(obj, f.name)
            if material_meta is not None:
                for k, v in material_meta.items():
                    mg.attrs[k] = v
            if self.device_postprocess:
                from ..processresults import near_field_power_device
                g = self.params.geom_params
                inc = {k: pg[k][()] for k in ('ex_inc_phasor', 'ey_inc_phasor', 'hx_inc_phasor',
                                              'hy_inc_phasor')}
                nf = out.create_group('near_field_power')
                for k, v in near_field_power_device(self.native, inc, g.cell_size,
                                                    g.size_z_material).items():
                    nf.attrs[k] = v
                nf.attrs['powers_computed'] = True

    def close(self):
        self.native.close()
