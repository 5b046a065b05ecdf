"""Simulation parameters: the same dataclasses, JSON keys and derived
geometry as the reference's ``fdtdsarsim.parameters`` (parameters.py:16-356).

The derived quantities (grid sizes, time step, step counts, TFSF plane) must
come out identical to the reference's, so ``set_geom_params`` keeps its
arithmetic: Python float floor-division for the sizes, ``round_to_odd`` on
those quotients, ``scipy.constants.c`` for the wavelength and time step.
Field names and their order also fix the ``/parameters`` attributes written
into every result file.
"""
import dataclasses
import json
import logging
import os.path
from dataclasses import dataclass
from typing import List, Union

import numpy as np
import scipy.constants

__all__ = ['ProcessingParams', 'IncBeamParams', 'GeomParams', 'MaterialParams',
           'DisplayParams', 'ParameterCollection', 'load_from_json', 'set_geom_params',
           'inc_filename', 'results_filename', 'inc_file_dir', 'results_file_dir',
           'round_to_odd']

logger = logging.getLogger(__name__)


def round_to_odd(value):
    """Truncate towards zero and bump even results to the next odd integer
    (utils/rounding.py:4-15)."""
    if value < 0:
        raise ValueError('Only use this with positive values for now')
    out = np.fix(value).item()
    if np.remainder(out, 2).item() == 0:
        out += 1
    return int(out)


def _describe(obj):
    if not dataclasses.is_dataclass(obj):
        raise ValueError('Can only print a dataclass')
    text = f'{type(obj).__name__}:\n'
    for f in dataclasses.fields(obj):
        text += f'   {f.name}: {getattr(obj, f.name)}\n'
    return text


@dataclass
class ProcessingParams:
    """Where and how a simulation runs (parameters.py:16-27)."""
    processing_type: str = 'cpu'
    gpu_num: Union[int, List[int]] = 0
    threads_per_proc: int = 1
    datatype: str = 'float32'
    project_dir: str = ''

    def __str__(self):
        return _describe(self)


@dataclass
class IncBeamParams:
    """Incident beam definition (parameters.py:30-55)."""
    frequency: float = 0
    polarization: str = 0
    theta_angle: float = 0
    phi_angle: float = 0
    duration: float = 0
    illumination_width: float = 0
    generate_new: bool = False

    def __str__(self):
        return _describe(self)


@dataclass
class GeomParams:
    """Grid geometry and time stepping (parameters.py:58-94)."""
    cell_size: float = 0
    simulation_duration: float = 0
    timestep: float = 0
    size_t: int = 0
    size_t_inc: int = 0
    size_t_pulse: int = 0
    size_x: int = 0
    size_y: int = 0
    size_z: int = 0
    size_pml: int = 0
    size_z_material: int = 0
    tfsf_z: int = 0
    courant: float = 0

    def __str__(self):
        return _describe(self)


@dataclass
class MaterialParams:
    """Material-volume controls (parameters.py:97-111)."""
    material_fraction: float = 0.7

    def __str__(self):
        return _describe(self)


@dataclass
class DisplayParams:
    """Display switches (parameters.py:114-130). This package is headless:
    the flags are kept for file compatibility and never open a window."""
    display_limit: float = 0.0
    display_step: int = 10
    inc_results: bool = False
    inc_sim_movie: bool = False
    debug_plots: bool = False
    main_sim_movie: bool = False
    material_plot: bool = False

    def __str__(self):
        return _describe(self)


@dataclass
class ParameterCollection:
    """All parameters of one experiment (parameters.py:133-156)."""
    processing_params: ProcessingParams = dataclasses.field(default_factory=ProcessingParams)
    inc_beam_params: IncBeamParams = dataclasses.field(default_factory=IncBeamParams)
    geom_params: GeomParams = dataclasses.field(default_factory=GeomParams)
    material_params: MaterialParams = dataclasses.field(default_factory=MaterialParams)
    display_params: DisplayParams = dataclasses.field(default_factory=DisplayParams)

    def __str__(self):
        return ''.join(f'{getattr(self, f.name)}\n' for f in dataclasses.fields(self))


_GEOM_KEYS = ('size_x', 'size_y', 'size_z_material', 'simulation_duration', 'cell_size', 'unit')


def load_from_json(filename: str) -> ParameterCollection:
    """Read a params.json with the reference's keys (parameters.py:159-239).
    Geometry is derived immediately when all six geometry keys are present,
    otherwise later from the first material model."""
    logger.info('Loading parameters from the file %s', filename)
    with open(filename, 'r') as fh:
        user = json.loads(fh.read())
    pc = ParameterCollection()
    proc, inc = pc.processing_params, pc.inc_beam_params
    proc.processing_type = user['processing_type']
    proc.gpu_num = user.get('gpu_num', 0)
    proc.threads_per_proc = user['threads_per_proc']
    proc.datatype = user['datatype']
    proc.project_dir = user['project_dir']
    inc.frequency = user['frequency_hz']
    inc.polarization = user['polarization']
    inc.theta_angle = user['theta_angle_deg']
    inc.phi_angle = user['phi_angle_deg']
    inc.duration = user['incident_duration']
    inc.illumination_width = user['illumination_width']
    inc.generate_new = user['generate_new']
    pc.material_params.material_fraction = user['material_fraction']
    disp = pc.display_params
    disp.display_limit = 0.5
    disp.display_step = 10
    disp.inc_results = user['disp_inc_results']
    disp.inc_sim_movie = user['disp_inc_sim_movie']
    disp.debug_plots = user['disp_debug']
    disp.main_sim_movie = user['disp_main_sim_movie']
    disp.material_plot = user['disp_materials']
    pc.geom_params.simulation_duration = user['simulation_duration']
    if all(k in user for k in _GEOM_KEYS):
        set_geom_params(pc, user['size_x'], user['size_y'], user['size_z_material'],
                        user['simulation_duration'], user['cell_size'], user['unit'])
    return pc


def set_geom_params(pc: ParameterCollection, size_x: float, size_y: float,
                    size_z_material: float, size_t: float, cell_size: float, unit: str):
    """Derive grid sizes and time stepping (parameters.py:242-305).

    ``unit`` is 'metre'/'meter' or 'wavelength'; sizes and cell_size are
    read in that unit. Courant number 0.5 and a 10-cell CPML are fixed.
    """
    g = pc.geom_params
    g.courant = 0.5
    g.size_pml = 10
    lam = scipy.constants.c / pc.inc_beam_params.frequency
    u = unit.lower()
    if u in ('metre', 'meter'):
        g.cell_size = cell_size
    elif u == 'wavelength':
        g.cell_size = lam * cell_size
    else:
        raise ValueError(f'Unknown value of unit: {unit}')
    g.size_x = round_to_odd(size_x // cell_size)
    g.size_y = round_to_odd(size_y // cell_size)
    g.size_z_material = int(size_z_material // cell_size)
    g.size_z = round_to_odd(g.size_z_material / pc.material_params.material_fraction)
    g.tfsf_z = g.size_z_material + int(0.3 * lam / g.cell_size)
    g.timestep = g.cell_size * g.courant / scipy.constants.c
    dt = g.timestep
    freq = pc.inc_beam_params.frequency
    g.size_t_pulse = round(1.2 * pc.inc_beam_params.duration * lam / (scipy.constants.c * dt))
    g.size_t_inc = round(1.2 * g.size_t_pulse)
    g.size_t = round(size_t / dt / freq)
    if g.size_t_inc > g.size_t:
        logger.warning('Reducing the number of timesteps in the incident beam')
        g.size_t_inc = g.size_t


def inc_file_dir(proc_params: ProcessingParams) -> str:
    d = os.path.join(proc_params.project_dir, 'incident')
    os.makedirs(d, exist_ok=True)
    return d


def results_file_dir(proc_params: ProcessingParams) -> str:
    d = os.path.join(proc_params.project_dir, 'results')
    os.makedirs(d, exist_ok=True)
    return d


def inc_filename(pc: ParameterCollection) -> str:
    """Incident beam file path (parameters.py:308-324)."""
    g, b = pc.geom_params, pc.inc_beam_params
    fname = (f'inc_nx{g.size_x}_ny{g.size_y}_nt{g.size_t_inc}'
             f'_theta{round(b.theta_angle)}_phi{round(b.phi_angle)}_{b.polarization}.hdf5')
    return os.path.join(inc_file_dir(pc.processing_params), fname)


def results_filename(pc: ParameterCollection, material_name: str) -> str:
    """Result file path (parameters.py:327-334)."""
    return os.path.join(results_file_dir(pc.processing_params), material_name + '.hdf5')
