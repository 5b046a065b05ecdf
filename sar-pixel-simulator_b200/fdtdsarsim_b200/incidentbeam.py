"""Incident beam files (fdtdsarsim/incidentbeam.py:25-172)."""
import logging
import os

import numpy as np

from . import resultsio
from .parameters import ParameterCollection, inc_filename

logger = logging.getLogger(__name__)

_META_CHECKS = (
    ('datatype', 'processing_params', 'datatype'),
    ('frequency', 'inc_beam_params', 'frequency'),
    ('polarization', 'inc_beam_params', 'polarization'),
    ('theta_angle', 'inc_beam_params', 'theta_angle'),
    ('phi_angle', 'inc_beam_params', 'phi_angle'),
    ('duration', 'inc_beam_params', 'duration'),
    ('illumination_width', 'inc_beam_params', 'illumination_width'),
    ('cell_size', 'geom_params', 'cell_size'),
    ('timestep', 'geom_params', 'timestep'),
    ('size_t_inc', 'geom_params', 'size_t_inc'),
    ('size_t_pulse', 'geom_params', 'size_t_pulse'),
    ('size_x', 'geom_params', 'size_x'),
    ('size_y', 'geom_params', 'size_y'),
    ('size_pml', 'geom_params', 'size_pml'),
    ('courant', 'geom_params', 'courant'),
)


class IncidentBeam:
    """Creates or validates the incident beam file of a geometry."""

    def __init__(self, params: ParameterCollection):
        self.params = params
        self.inc_beam_params = params.inc_beam_params
        self.geom_params = params.geom_params
        self.processing_params = params.processing_params

    def inc_beam_exists(self):
        from .incident import wait_written
        fname = inc_filename(self.params)
        wait_written(fname)                 # a file this process is still writing
        return resultsio.exists(fname)

    def setup(self):
        """Load the geometry's incident file, or make the beam on the device
        and write it first (incidentbeam.py:41-71)."""
        if not self.inc_beam_params.generate_new and self.inc_beam_exists():
            logger.info('Loading existing incident beam files')
            self.load_existing()
            return
        logger.info('Generating new incident beam on the device')
        from .incident import keep_resident, make_incident_beam, store_incident_beam
        planes, phasors, sim = make_incident_beam(self.params)
        # the planes stay on the device for the main simulation of this
        # geometry (MainSimGpu takes them without reading the file back);
        # the file is written, then checked, on a thread meanwhile
        keep_resident(inc_filename(self.params), sim, phasors)
        store_incident_beam(self.params, planes, phasors, background=True)

    def create_pulse(self):
        """The temporal pulse and its spectrum (incidentbeam.py:174-204):
        sets time_vals, pulse, pulse_fft and pulse_freqs."""
        from .incident import create_pulse
        self.time_vals, self.pulse, self.pulse_fft, self.pulse_freqs = create_pulse(self.params)

    def create_inc_excitation(self):
        """The excitation of the incident simulation, computed on the device
        (incidentbeam.py:206-298). Returns the part of the reference's
        complex (size_t_inc, ny, nx) arrays that the simulation injects: the
        imaginary parts of the first size_t_pulse samples
        (cpu/incident_sim.py:108-110,141-144), as (Ex, Ey) real arrays of the
        simulation dtype. Call create_pulse() first."""
        from .incident import IncidentSimGpu
        from .gpu.main_sim import _device_of
        sim = IncidentSimGpu(self.params, _device_of(self.params))
        try:
            sim.make_excitation(self.pulse_fft, self.pulse_freqs)
            return sim.native.get_excitation()
        finally:
            sim.close()

    def load_existing(self):
        from .incident import wait_written
        wait_written(inc_filename(self.params))
        self.check_file()

    def check_file(self):
        """Shape, dtype and metadata checks of the incident file
        (incidentbeam.py:74-165)."""
        with resultsio.File(inc_filename(self.params), 'r') as f:
            self.check_array_sizes(f['ex'], f['ey'], f['hx'], f['hy'])
            self.check_metadata(f.attrs)

    def check_array_sizes(self, *fields):
        """Shape and dtype checks of incidentbeam.py:82-103."""
        g = self.geom_params
        want = (g.size_t_inc, g.size_y, g.size_x)
        for fld in fields:
            if tuple(fld.shape) != want:
                raise ValueError(f'A component of the incident beam has the wrong shape. '
                                 f'Got {tuple(fld.shape)}, expected {want}.')
            if np.dtype(fld.dtype) != np.dtype(self.processing_params.datatype):
                raise ValueError('Incident beam has incorrect datatype. Please delete the '
                                 'incident beam file and re-run the simulation.')

    def check_metadata(self, meta):
        """Metadata consistency checks of incidentbeam.py:105-165."""
        for key, group, field in _META_CHECKS:
            val = getattr(getattr(self.params, group), field)
            got = meta[key]
            if isinstance(got, bytes):
                got = got.decode()
            if isinstance(val, str):
                same = str(got) == val
            else:
                same = got == val
            if not same:
                raise ValueError(f'Incident beam metadata inconsistency ({key})')
        if not bool(meta['incident_complete']):
            raise ValueError('Incident beam simulation was not completed')


def write_incident_file(params: ParameterCollection, ex, ey, hx, hy, inc_phasors):
    """Write an incident beam file with the reference's datasets and
    metadata (cpu/incident_sim.py:94-98,166-224)."""
    fname = inc_filename(params)
    if os.path.exists(fname):
        os.remove(fname)
    proc, inc, g = params.processing_params, params.inc_beam_params, params.geom_params
    with resultsio.File(fname, 'w') as f:
        for name, arr in (('ex', ex), ('ey', ey), ('hx', hx), ('hy', hy)):
            f.create_dataset(name, data=np.asarray(arr, dtype=proc.datatype))
        pg = f.create_group('phasors')
        for c in ('ex', 'ey', 'hx', 'hy'):
            pg.create_dataset(f'{c}_inc_phasor', data=inc_phasors[f'{c}_inc_phasor'])
        a = f.attrs
        a['datatype'] = proc.datatype
        a['frequency'] = inc.frequency
        a['polarization'] = inc.polarization
        a['theta_angle'] = inc.theta_angle
        a['phi_angle'] = inc.phi_angle
        a['duration'] = inc.duration
        a['illumination_width'] = inc.illumination_width
        a['cell_size'] = g.cell_size
        a['timestep'] = g.timestep
        a['size_t_inc'] = g.size_t_inc
        a['size_t_pulse'] = g.size_t_pulse
        a['size_x'] = g.size_x
        a['size_y'] = g.size_y
        a['size_pml'] = g.size_pml
        a['courant'] = g.courant
        a['incident_complete'] = True
    return fname
