"""fdtdsarsim_b200: B200-native drop-in for the time-stepping path of
fdtdsarsim (wyatt-sfu/sar-pixel-simulator).

    import fdtdsarsim_b200 as fdtd
    params = fdtd.load_from_json('params.json')   # processing_type "gpu"
    fdtd.run_experiment(params, materials)

All compute runs in libfdtd_b200.so (hand-written sm_100a CUDA behind a
C-ABI). The host-only modules (parameters, material models and
generators, CPML profiles, synthetic inputs) import without the library;
the first use of anything that runs on the device (run_experiment,
get_fdtd_simulator, run_experiment_batched, IncidentBeam, near2far,
processresults, or the _native binding itself) loads it and fails with an
error when it is not built. There is no CPU fallback.
"""
import importlib

from .parameters import *  # noqa: F401,F403
from .parameters import __all__ as _param_all
from . import materials  # noqa: F401
from .materials import MaterialModel, compute_material_arrays

# name -> (module, attribute or None for the module itself); loaded on
# first access, each of them loads libfdtd_b200.so
_DEVICE = {
    'get_fdtd_simulator': ('.experiment', 'get_fdtd_simulator'),
    'run_experiment': ('.experiment', 'run_experiment'),
    'run_experiment_batched': ('.sweep', 'run_experiment_batched'),
    'IncidentBeam': ('.incidentbeam', 'IncidentBeam'),
    'near2far': ('.near2far', None),
    'processresults': ('.processresults', None),
}


def __getattr__(name):
    if name in _DEVICE:
        mod, attr = _DEVICE[name]
        importlib.import_module('._native', __name__)   # the library, or an error
        m = importlib.import_module(mod, __name__)
        value = m if attr is None else getattr(m, attr)
        globals()[name] = value
        return value
    raise AttributeError(f'module {__name__!r} has no attribute {name!r}')


__all__ = list(_param_all) + ['get_fdtd_simulator', 'run_experiment', 'run_experiment_batched',
                              'IncidentBeam', 'materials', 'near2far', 'processresults',
                              'MaterialModel', 'compute_material_arrays']
