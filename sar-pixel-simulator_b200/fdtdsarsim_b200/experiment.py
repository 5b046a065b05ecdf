"""Experiment entry points: the reference's functions (fdtdsarsim/experiment.py:
19-97) over the device simulator."""
import logging
import os
import queue
import threading
from typing import Iterable, Iterator, TypeVar

from .incident import wait_written
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


T = TypeVar('T')


def prefetched(items: Iterable[T], depth: int = 1) -> Iterator[T]:
    """``items`` in order, produced by a background thread up to ``depth``
    ahead of the consumer, so that a host-side material generator makes the
    next model while the device solves the current one (the solve waits in
    the library with the GIL released). An exception of the producer is
    raised in the consumer where the item would have been; closing the
    iterator early stops the producer."""
    q: queue.Queue = queue.Queue(maxsize=max(1, depth))
    stop = threading.Event()
    end = object()

    def put(entry):
        while not stop.is_set():
            try:
                q.put(entry, timeout=0.1)
                return True
            except queue.Full:
                continue
        return False

    def produce():
        try:
            for item in items:
                if not put((True, item)):
                    return
            put((True, end))
        except BaseException as exc:  # handed to the consumer
            put((False, exc))

    worker = threading.Thread(target=produce, name='material-prefetch', daemon=True)
    worker.start()
    try:
        while True:
            try:
                ok, item = q.get(timeout=0.5)
            except queue.Empty:
                if not worker.is_alive() and q.empty():
                    raise RuntimeError('material prefetch thread ended without a result')
                continue
            if not ok:
                raise item
            if item is end:
                return
            yield item
    finally:
        stop.set()


def run_experiment(params: ParameterCollection, materials: Iterable[MaterialModel],
                   prefetch: int = 1):
    """Simulate every material model with one shared incident beam, then
    post-process all results (experiment.py:41-97). ``prefetch`` (this
    package's addition; 0 turns it off) is how many models the host makes
    ahead while the device runs."""
    g = params.geom_params
    geom_specified = not (g.size_x == 0 and g.size_y == 0 and g.size_z == 0)
    it = iter(materials)
    sim = None
    if geom_specified:
        sim = get_fdtd_simulator(params)(params)
        IncidentBeam(params).setup()
    else:
        # the first model sets the geometry before any other model is made
        first = next(it, None)
        if first is not None:
            nz_mat, ny, nx = _shape(first)
            dx = first.cell_size
            set_geom_params(params, nx * dx, ny * dx, nz_mat * dx,
                            params.geom_params.simulation_duration, dx, 'metre')
            sim = get_fdtd_simulator(params)(params)
            IncidentBeam(params).setup()
            _simulate(sim, first)
    if sim is not None:
        for material in (prefetched(it, prefetch) if prefetch > 0 else it):
            _simulate(sim, material)
    process_all_results(params.processing_params.project_dir,
                        params.display_params.debug_plots)
    wait_written()       # every incident file of this experiment is on disk


def _shape(material):
    from .materials.device import LayeredMaterial
    if isinstance(material, LayeredMaterial):
        return material.shape
    return material.conductivity.shape


def _simulate(sim, material: MaterialModel):
    from .materials.device import LayeredMaterial
    if isinstance(material, LayeredMaterial):
        # the block made on the device from its recipe
        sim.run_layered(material)
        return
    # Ca/Cb on the device: the values compute_material_arrays gives
    sim.run_eps_sigma(material.relative_permittivity, material.conductivity,
                      material.name, material.metadata)
