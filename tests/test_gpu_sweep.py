"""run_experiment_batched on the device against run_experiment, model by
model: four material models of uneven extents (two sharing one geometry),
batched in both batch modes, give the same result files as a sequential
run_experiment of each model with its own geometry: all 24 phasor planes,
the incident phasors and the post-processed far field bit for bit."""
import os

import numpy as np
import pytest

from fdtdsarsim_b200 import _native, resultsio, sweep, synthetic
from fdtdsarsim_b200.experiment import run_experiment
from fdtdsarsim_b200.materials import MaterialModel
from fdtdsarsim_b200.parameters import results_filename

pytestmark = pytest.mark.gpu


def _base(project_dir):
    pc = synthetic.base_params('float32', pol='VV', mf=0.2, illum=1.0)
    pc.processing_params.project_dir = str(project_dir)
    pc.geom_params.simulation_duration = 1.5        # about 100 steps at 0.03 wavelength cells
    pc.inc_beam_params.duration = 0.5
    pc.geom_params.size_x = pc.geom_params.size_y = pc.geom_params.size_z = 0
    return pc


def _model(pc, shape, seed, name):
    rng = np.random.default_rng(seed)
    dx = 0.03 * 2.99792458e8 / pc.inc_beam_params.frequency
    return MaterialModel(rng.uniform(1.0, 9.0, shape).astype(np.float32),
                         rng.uniform(0.0, 0.05, shape).astype(np.float32), dx, name, {'seed': seed})


def _read(path):
    out = {}
    with resultsio.File(path, 'r') as f:
        for name in f['phasors'].keys():
            out['phasors/' + name] = np.asarray(f['phasors'][name][()])
        if 'farfield' in f:
            for name in f['farfield'].keys():
                out['farfield/' + name] = np.asarray(f['farfield'][name][()])
    return out


@pytest.mark.parametrize('streams', [True, False], ids=['streams', 'split'])
def test_batched_sweep_equals_sequential_experiments(tmp_path, streams):
    shapes = [(7, 25, 27), (9, 25, 27), (7, 29, 23), (9, 23, 31)]
    batched_dir, seq_dir = tmp_path / 'batched', tmp_path / 'sequential'
    pcb = _base(batched_dir)
    models = [_model(pcb, s, k + 1, f'm{k}') for k, s in enumerate(shapes)]
    sweep.run_experiment_batched(pcb, iter(models), batch_size=3, streams=streams)
    pcs = _base(seq_dir)
    for m in models:
        run_experiment(sweep.model_params(pcs, m), [m])
    checked = 0
    for m in models:
        a = _read(results_filename(sweep.model_params(pcb, m), m.name))
        b = _read(results_filename(sweep.model_params(pcs, m), m.name))
        assert set(a) == set(b) and len(a) >= 28, sorted(a)
        assert np.max(np.abs(a['phasors/ey_ph_u'])) > 0
        for k in a:
            assert a[k].dtype == b[k].dtype and np.array_equal(a[k], b[k]), (m.name, k)
            checked += 1
    assert checked >= 4 * 28
    print('result files written with', resultsio.BACKEND)
