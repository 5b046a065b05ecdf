"""Batched sweep over material models of uneven sizes: the batched form of
run_experiment (experiment.py:41-97).

The reference solves one model per MainSimGpu.run and one geometry per
experiment (experiment.py:61-84), so a sweep over models of different
extents is a loop of experiments, each with its own incident beam and its
own time loop per model. Here each model gets the geometry of its own
extent, the incident beam of each geometry is made once (IncidentBeam.setup:
on the device, or read from its file) and copied device to device into
every model that uses it, and up to ``batch_size`` models are advanced
together by one fdtd_batch -- by default each model's own step on its own
stream, side by side (FDTD_OPT_BATCH_STREAMS). Each model then writes the
reference's result file exactly as MainSimGpu.run does; models whose result
file exists are skipped; every result is post-processed at the end.
"""
import copy
import logging
from typing import Iterable

import numpy as np

from . import _native, resultsio
from .experiment import get_fdtd_simulator, prefetched
from .incident import take_resident, wait_written
from .incidentbeam import IncidentBeam
from .materials.materialmodel import MaterialModel
from .parameters import ParameterCollection, inc_filename, results_filename, set_geom_params
from .processresults import process_all_results

logger = logging.getLogger(__name__)

__all__ = ['model_params', 'run_experiment_batched']


def model_params(params: ParameterCollection, model: MaterialModel) -> ParameterCollection:
    """A copy of ``params`` with the geometry of ``model``'s extent, derived
    by set_geom_params in metres as run_experiment derives it from a model
    when the parameters name no geometry (experiment.py:66-80). The extent
    must be one set_geom_params makes (odd x and y sizes)."""
    nz_mat, ny, nx = np.shape(model.relative_permittivity)
    if np.shape(model.conductivity) != (nz_mat, ny, nx):
        raise RuntimeError('Permittivity and conductivity arrays have different shapes')
    dx = model.cell_size
    pc = copy.deepcopy(params)
    # half a cell above each extent: the floor division gives the extent itself
    set_geom_params(pc, (nx + 0.5) * dx, (ny + 0.5) * dx, (nz_mat + 0.5) * dx,
                    params.geom_params.simulation_duration, dx, 'metre')
    g = pc.geom_params
    if (g.size_z_material, g.size_y, g.size_x) != (nz_mat, ny, nx):
        raise ValueError(f'model {model.name}: extent {(nz_mat, ny, nx)} is not a grid that '
                         f'set_geom_params makes (x and y sizes must be odd)')
    return pc


def run_experiment_batched(params: ParameterCollection, materials: Iterable[MaterialModel],
                           batch_size: int = 64, streams: bool = True, prefetch: bool = True):
    """Simulate every model of ``materials`` (uneven extents allowed) in
    batches of ``batch_size``, write each result file, then post-process
    all results. ``streams`` selects the batch mode (True: each model's own
    step on its own stream; False: one launch per pass for all models).
    With ``prefetch`` the next batch's models are made on the host while
    the device runs the current batch."""
    if batch_size < 1:
        raise ValueError('batch_size must be at least 1')
    sim_class = get_fdtd_simulator(params)          # 'gpu' only, as run_experiment
    source = prefetched(materials, batch_size) if prefetch else iter(materials)
    pending = []
    for model in source:
        pending.append(model)
        if len(pending) == batch_size:
            _run_batch(sim_class, params, pending, streams)
            pending = []
    if pending:
        _run_batch(sim_class, params, pending, streams)
    process_all_results(params.processing_params.project_dir, params.display_params.debug_plots)
    wait_written()       # every incident file of this sweep is on disk


def _run_batch(sim_class, params, models, streams):
    members = []                                  # (model, params, simulator)
    taken = set()
    try:
        for model in models:
            pc = model_params(params, model)
            out = results_filename(pc, model.name)
            # a result file that exists, or that an earlier model of this
            # batch will write, is skipped as run_experiment skips it
            if resultsio.exists(out) or out in taken:
                logger.info('%s already exists, skipping', out)
                continue
            taken.add(out)
            members.append((model, pc, sim_class(pc)))
        if not members:
            return
        # materials, and each geometry's incident beam made or loaded once
        by_beam = {}
        for m in members:
            by_beam.setdefault(inc_filename(m[1]), []).append(m)
        for fname, group in by_beam.items():
            IncidentBeam(group[0][1]).setup()
            held = take_resident(fname)
            try:
                for model, pc, sim in group:
                    sim.native.reset()
                    sim.native.set_materials_eps_sigma(model.relative_permittivity,
                                                       model.conductivity)
                    if held is None or not sim.use_incident_run(*held):
                        sim._ensure_incident()
            finally:
                if held is not None:
                    held[0].close()
        # advance together; members of one batch share their step count
        by_steps = {}
        for m in members:
            by_steps.setdefault(m[1].geom_params.size_t, []).append(m)
        for nt, group in by_steps.items():
            logger.info('Batch of %d models, %d steps', len(group), nt)
            batch = _native.Batch([sim.native for _, _, sim in group], streams=streams)
            try:
                batch.run(nt)
                batch.synchronize()
            finally:
                batch.close()
        for model, pc, sim in members:
            sim.native.synchronize()
            sim.save_results(model.name, model.metadata)
    finally:
        for _, _, sim in members:
            sim.close()
