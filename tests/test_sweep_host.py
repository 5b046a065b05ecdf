"""run_experiment_batched (fdtdsarsim_b200.sweep) on the CPU: the device
simulation, batch and incident run are replaced by stand-ins driven by the
numpy oracle, so the orchestration -- per-model geometry, one incident beam
per geometry shared device to device or read from its file, batches,
skip-if-exists, result files in the reference's layout -- is checked
against direct oracle runs of the same models, bit for bit."""
import os

import numpy as np
import pytest

import fdtd_oracle as O
from fdtdsarsim_b200 import _native, incident, resultsio, sweep, synthetic
from fdtdsarsim_b200.absorbers import cpml_profiles
from fdtdsarsim_b200.gpu.main_sim import MainSimGpu, native_geometry
from fdtdsarsim_b200.incidentbeam import write_incident_file
from fdtdsarsim_b200.materials import MaterialModel, compute_material_arrays
from fdtdsarsim_b200.parameters import inc_filename, results_filename


class OracleNative:
    """NativeSim's calls used by the sweep, computed by the oracle."""

    def __init__(self, pc):
        g = pc.geom_params
        self.pc, self.geom = pc, native_geometry(pc)
        self.orc = O.OracleSim(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size,
                               g.timestep, pc.inc_beam_params.frequency,
                               pc.processing_params.datatype, cpml_profiles(pc))
        self.inc = None
        self.closed = False

    def reset(self):
        self.orc.reset()

    def set_materials_eps_sigma(self, eps, sig):
        self.ca, self.cb = compute_material_arrays(
            self.pc, MaterialModel(np.asarray(eps), np.asarray(sig), self.pc.geom_params.cell_size))

    def set_incident(self, ex, ey, hx, hy):
        self.inc = {'ex': ex, 'ey': ey, 'hx': hx, 'hy': hy}

    def set_incident_from(self, other):
        n = self.geom.nt_inc
        self.inc = {c: other.planes[c][:n] for c in ('ex', 'ey', 'hx', 'hy')}

    def run(self, n):
        self.orc.run(self.ca, self.cb, self.inc, n)

    def synchronize(self):
        pass

    def get_phasors(self):
        return dict(self.orc.ph)

    def close(self):
        self.closed = True


class StandInSim(MainSimGpu):
    created = []

    def __init__(self, params, mpi=False):
        g = params.geom_params
        self.params, self.mpi, self.gpu_num = params, mpi, 0
        self.dtype = np.dtype(params.processing_params.datatype)
        self.geom = native_geometry(params)
        self.native = OracleNative(params)
        self._incident_loaded = None
        self._inc_phasors = None
        self.nx_ph, self.ny_ph, self.nz_ph = (g.size_x - 2 * g.size_pml, g.size_y - 2 * g.size_pml,
                                              g.size_z - 2 * g.size_pml)
        StandInSim.created.append(self)


class StandInBatch:
    made = []

    def __init__(self, sims, graph_chunk=None, streams=False):
        self.sims, self.streams = list(sims), streams
        StandInBatch.made.append((len(self.sims), streams))

    def run(self, n):
        for s in self.sims:
            s.run(n)

    def synchronize(self):
        pass

    def close(self):
        pass


class StandInRun:
    def __init__(self, pc, planes):
        self.native = OracleNative(pc)
        self.native.planes = planes
        self.closed = False

    def close(self):
        self.closed = True


class StandInBeam:
    """IncidentBeam.setup: an existing file is used as it is; otherwise a
    beam is made (a seeded plane wave here), written and held resident."""
    made = []

    def __init__(self, params):
        self.params = params

    def setup(self):
        fname = inc_filename(self.params)
        if os.path.exists(fname):
            return
        g = self.params.geom_params
        dtype = self.params.processing_params.datatype
        planes = synthetic.plane_wave_incident(self.params, g.size_t_inc, dtype)
        cd = np.complex64 if dtype == 'float32' else np.complex128
        rng = np.random.default_rng(g.size_x * 1000 + g.size_y)
        phasors = {f'{c}_inc_phasor': (rng.standard_normal((g.size_y - 20, g.size_x - 20))
                                       + 1j).astype(cd) for c in ('ex', 'ey', 'hx', 'hy')}
        write_incident_file(self.params, planes['ex'], planes['ey'], planes['hx'], planes['hy'],
                            phasors)
        incident.keep_resident(fname, StandInRun(self.params, planes), phasors)
        StandInBeam.made.append(fname)


@pytest.fixture
def stand_ins(monkeypatch):
    StandInSim.created, StandInBatch.made, StandInBeam.made = [], [], []
    processed = []
    monkeypatch.setattr(sweep, 'get_fdtd_simulator', lambda params: StandInSim)
    monkeypatch.setattr(sweep, 'IncidentBeam', StandInBeam)
    monkeypatch.setattr(_native, 'Batch', StandInBatch)
    monkeypatch.setattr(sweep, 'process_all_results', lambda d, p: processed.append(d))
    yield processed
    incident._RESIDENT.clear()


def base(tmp_path):
    pc = synthetic.base_params('float32', pol='VV', mf=0.2, illum=1.0)
    pc.processing_params.project_dir = str(tmp_path)
    pc.geom_params.simulation_duration = 1.5        # about 100 steps at 0.03 wavelength cells
    pc.inc_beam_params.duration = 0.5
    pc.geom_params.size_x = pc.geom_params.size_y = pc.geom_params.size_z = 0
    return pc


def model(pc, shape, seed, name):
    rng = np.random.default_rng(seed)
    dx = 0.03 * 2.99792458e8 / pc.inc_beam_params.frequency
    return MaterialModel(rng.uniform(1.0, 9.0, shape).astype(np.float32),
                         rng.uniform(0.0, 0.05, shape).astype(np.float32), dx, name,
                         {'seed': seed})


def oracle_phasors(pc, m):
    g = pc.geom_params
    ca, cb = compute_material_arrays(pc, m)
    with resultsio.File(inc_filename(pc), 'r') as f:
        inc = {c: np.asarray(f[c][()]) for c in ('ex', 'ey', 'hx', 'hy')}
    orc = O.OracleSim(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size,
                      g.timestep, pc.inc_beam_params.frequency, 'float32', cpml_profiles(pc))
    orc.run(ca, cb, inc, g.size_t)
    return orc.ph


def test_batched_sweep_writes_each_models_result(stand_ins, tmp_path):
    pc = base(tmp_path)
    models = [model(pc, (7, 25, 27), 1, 'a'), model(pc, (9, 25, 27), 2, 'b'),   # one beam
              model(pc, (7, 29, 23), 3, 'c'), model(pc, (9, 23, 31), 4, 'd')]
    sweep.run_experiment_batched(pc, iter(models), batch_size=3)
    assert StandInBatch.made == [(3, True), (1, True)]
    assert len(StandInBeam.made) == 3                  # one per distinct x-y geometry
    assert all(s.native.closed for s in StandInSim.created)
    assert not incident._RESIDENT
    assert stand_ins == [str(tmp_path)]
    for m in models:
        mp = sweep.model_params(pc, m)
        g = mp.geom_params
        want = oracle_phasors(mp, m)
        assert np.max(np.abs(want['ey_ph_u'])) > 0 and np.max(np.abs(want['ex_ph_d'])) > 0
        with resultsio.File(results_filename(mp, m.name), 'r') as f:
            for name in _native.PHASOR_NAMES:
                got = f['phasors'][name][()]
                assert got.dtype == np.complex64 and np.array_equal(got, want[name]), (m.name, name)
            assert f['parameters'].attrs['size_x'] == g.size_x
            assert f['parameters'].attrs['size_z'] == g.size_z
            assert f['phasors'].attrs['nz_phasor'] == g.size_z - 20
            assert f['material_metadata'].attrs['seed'] == m.metadata['seed']
            with resultsio.File(inc_filename(mp), 'r') as inc:
                np.testing.assert_array_equal(f['phasors']['ex_inc_phasor'][()],
                                              inc['phasors']['ex_inc_phasor'][()])


def test_batched_sweep_skips_existing_and_reads_beams_from_files(stand_ins, tmp_path):
    pc = base(tmp_path)
    first = model(pc, (7, 25, 27), 1, 'a')
    sweep.run_experiment_batched(pc, [first], batch_size=4, streams=False, prefetch=False)
    path = results_filename(sweep.model_params(pc, first), 'a')
    stamp = os.stat(path).st_mtime_ns
    StandInBeam.made.clear()
    later = model(pc, (9, 25, 27), 5, 'e')              # same beam, its file already written
    sweep.run_experiment_batched(pc, [first, later], batch_size=4)
    assert os.stat(path).st_mtime_ns == stamp           # skipped
    assert StandInBeam.made == []                       # the beam came from its file
    assert StandInBatch.made == [(1, False), (1, True)]
    mp = sweep.model_params(pc, later)
    want = oracle_phasors(mp, later)
    with resultsio.File(results_filename(mp, 'e'), 'r') as f:
        for name in _native.PHASOR_NAMES:
            assert np.array_equal(f['phasors'][name][()], want[name]), name


def test_model_params_rejects_extents_set_geom_params_cannot_make(tmp_path):
    pc = base(tmp_path)
    with pytest.raises(ValueError, match='odd'):
        sweep.model_params(pc, model(pc, (7, 24, 27), 1, 'even'))
    bad = model(pc, (7, 25, 27), 1, 'mismatch')
    bad.conductivity = bad.conductivity[1:]
    with pytest.raises(RuntimeError):
        sweep.model_params(pc, bad)
    with pytest.raises(ValueError):
        sweep.run_experiment_batched(pc, [], batch_size=0)
    pc.processing_params.processing_type = 'cpu'       # no CPU solver here, as run_experiment
    with pytest.raises(ValueError):
        sweep.run_experiment_batched(pc, [])


def test_a_repeated_name_is_skipped_as_run_experiment_skips_it(stand_ins, tmp_path):
    """Two models of one name in one batch: the first is simulated, the
    second skipped, as the sequential run_experiment skips a model whose
    result file an earlier model wrote (gpu/main_sim.py:100-110)."""
    pc = base(tmp_path)
    first, again = model(pc, (7, 25, 27), 1, 'same'), model(pc, (7, 25, 27), 9, 'same')
    sweep.run_experiment_batched(pc, [first, again], batch_size=4)
    assert StandInBatch.made == [(1, True)]
    mp = sweep.model_params(pc, first)
    want = oracle_phasors(mp, first)
    with resultsio.File(results_filename(mp, 'same'), 'r') as f:
        assert np.array_equal(f['phasors']['ey_ph_u'][()], want['ey_ph_u'])
        assert f['material_metadata'].attrs['seed'] == 1


@pytest.mark.parametrize('name', ['plain_2x2', 'adjoint_4x4', 'plain_8x8', 'plain_16x16'])
def test_model_params_gives_the_geometry_the_model_was_made_for(name):
    """A model made for a configuration's geometry gets exactly that
    geometry back (every field the result file stores in /parameters)."""
    import dataclasses
    pc = synthetic.config_params(name, 'float32')
    g = pc.geom_params
    shape = (g.size_z_material, g.size_y, g.size_x)
    m = MaterialModel(np.ones(shape, np.float32), np.zeros(shape, np.float32), g.cell_size, 'm')
    blank = synthetic.config_params(name, 'float32')
    blank.geom_params.size_x = blank.geom_params.size_y = blank.geom_params.size_z = 0
    got = sweep.model_params(blank, m).geom_params
    for f in dataclasses.fields(g):
        assert getattr(got, f.name) == getattr(g, f.name), f.name


def test_batched_sweep_with_no_models(stand_ins, tmp_path):
    pc = base(tmp_path)
    sweep.run_experiment_batched(pc, iter([]))
    assert StandInSim.created == [] and StandInBatch.made == [] and stand_ins == [str(tmp_path)]
