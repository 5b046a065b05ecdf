"""Experiment entry points: the reference's functions (fdtdsarsim/experiment.py:
19-97) over the device simulator."""
import logging
import os
from typing import Iterable

from .incidentbeam import IncidentBeam
from .materials.materialmodel import MaterialModel
from .parameters import ParameterCollection, set_geom_params
from .processresults import process_all_results

logger = logging.getLogger(__name__)


def get_fdtd_simulator(params: ParameterCollection):
    """Simulator class for ``processing_type`` (experiment.py:19-38).

    'gpu' selects the B200 simulator and exports CUDA_DEVICE like the
    reference. This package has no CPU solver: 'cpu' is rejected with a
    clear error rather than silently running something else.
    """
    proc_type = params.processing_params.processing_type.lower()
    if proc_type == 'gpu':
        os.environ['CUDA_DEVICE'] = str(params.processing_params.gpu_num)
        from .gpu.main_sim import MainSimGpu
        return MainSimGpu
    if proc_type == 'cpu':
        raise ValueError("fdtdsarsim_b200 implements processing_type 'gpu' only; "
                         "use the reference package for 'cpu'")
    raise ValueError('Invalid processing type')


def run_experiment(params: ParameterCollection, materials: Iterable[MaterialModel]):
    """Simulate every material model with one shared incident beam, then
    post-process all results (experiment.py:41-97)."""
    g = params.geom_params
    geom_specified = not (g.size_x == 0 and g.size_y == 0 and g.size_z == 0)
    sim = None
    if geom_specified:
        sim = get_fdtd_simulator(params)(params)
        IncidentBeam(params).setup()
    for material in materials:
        if sim is None:
            nz_mat, ny, nx = material.conductivity.shape
            dx = material.cell_size
            set_geom_params(params, nx * dx, ny * dx, nz_mat * dx,
                            params.geom_params.simulation_duration, dx, 'metre')
            sim = get_fdtd_simulator(params)(params)
            IncidentBeam(params).setup()
        # Ca/Cb on the device: the values compute_material_arrays gives
        sim.run_eps_sigma(material.relative_permittivity, material.conductivity,
                          material.name, material.metadata)
    process_all_results(params.processing_params.project_dir,
                        params.display_params.debug_plots)
