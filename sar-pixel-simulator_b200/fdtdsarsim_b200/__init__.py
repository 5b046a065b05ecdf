"""fdtdsarsim_b200: B200-native drop-in for the time-stepping path of
fdtdsarsim (wyatt-sfu/sar-pixel-simulator).

    import fdtdsarsim_b200 as fdtd
    params = fdtd.load_from_json('params.json')   # processing_type "gpu"
    fdtd.run_experiment(params, materials)

All compute runs in libfdtd_b200.so (hand-written sm_100a CUDA behind a
C-ABI); importing the package fails when the library is not built.
"""
from .parameters import *  # noqa: F401,F403
from .parameters import __all__ as _param_all
from . import _native  # noqa: F401  (loads libfdtd_b200.so or fails)
from .experiment import get_fdtd_simulator, run_experiment
from .incidentbeam import IncidentBeam
from . import materials, near2far, processresults  # noqa: F401
from .materials import MaterialModel, compute_material_arrays
from .sweep import run_experiment_batched

__all__ = list(_param_all) + ['get_fdtd_simulator', 'run_experiment', 'run_experiment_batched',
                              'IncidentBeam', 'materials', 'near2far', 'processresults',
                              'MaterialModel', 'compute_material_arrays']
