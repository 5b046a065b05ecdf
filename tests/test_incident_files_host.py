"""Incident files written beside the device work (fdtdsarsim_b200.incident):
IncidentBeam.setup keeps the beam it made on the device and writes its file
on a thread; readers in the process wait for that write, its errors reach
the caller, and run_experiment returns only when every incident file is on
disk. The device stage is replaced by seeded planes here."""
import os
import time

import numpy as np
import pytest

from fdtdsarsim_b200 import experiment, incident, incidentbeam, synthetic
from fdtdsarsim_b200.incidentbeam import IncidentBeam
from fdtdsarsim_b200.materials import MaterialModel
from fdtdsarsim_b200.parameters import inc_filename
from helpers import make_params


def params(tmp_path):
    pc = make_params(27, 25, 23, 14, 10, 6)
    pc.processing_params.project_dir = str(tmp_path)
    pc.inc_beam_params.duration = 1.0
    pc.inc_beam_params.illumination_width = 1.0
    return pc


def beam(pc):
    g = pc.geom_params
    planes = synthetic.plane_wave_incident(pc, g.size_t_inc, 'float32')
    phasors = {f'{c}_inc_phasor': np.full((g.size_y - 20, g.size_x - 20), 1 + 2j, np.complex64)
               for c in ('ex', 'ey', 'hx', 'hy')}
    return planes, phasors


class HeldRun:
    closed = False

    def close(self):
        self.closed = True


@pytest.fixture
def slow_writes(monkeypatch):
    real = incidentbeam.write_incident_file

    def slow(*a, **k):
        time.sleep(0.4)
        return real(*a, **k)

    monkeypatch.setattr(incidentbeam, 'write_incident_file', slow)
    yield
    incident.wait_written()
    incident._RESIDENT.clear()


def test_readers_wait_for_a_background_write(tmp_path, slow_writes):
    pc = params(tmp_path)
    planes, phasors = beam(pc)
    fname = inc_filename(pc)
    t0 = time.perf_counter()
    incident.store_incident_beam(pc, planes, phasors, background=True)
    assert time.perf_counter() - t0 < 0.3 and not os.path.exists(fname)
    assert IncidentBeam(pc).inc_beam_exists()           # waited for the write
    IncidentBeam(pc).load_existing()
    assert not incident._WRITES


def test_a_failed_background_write_reaches_the_caller(tmp_path, monkeypatch):
    pc = params(tmp_path)
    planes, phasors = beam(pc)

    def fail(*a, **k):
        raise OSError('disk full')

    monkeypatch.setattr(incidentbeam, 'write_incident_file', fail)
    incident.store_incident_beam(pc, planes, phasors, background=True)
    with pytest.raises(OSError, match='disk full'):
        incident.wait_written()
    assert not incident._WRITES


def test_setup_keeps_the_beam_and_writes_its_file_beside(tmp_path, slow_writes, monkeypatch):
    pc = params(tmp_path)
    run = HeldRun()
    planes, phasors = beam(pc)
    monkeypatch.setattr(incident, 'make_incident_beam', lambda p, device=None: (planes, phasors, run))
    t0 = time.perf_counter()
    IncidentBeam(pc).setup()
    assert time.perf_counter() - t0 < 0.3               # did not wait for the file
    held = incident.take_resident(inc_filename(pc))
    assert held is not None and held[0] is run
    incident.wait_written(inc_filename(pc))
    assert os.path.exists(inc_filename(pc))
    IncidentBeam(pc).check_file()


def test_run_experiment_returns_with_the_incident_file_on_disk(tmp_path, slow_writes, monkeypatch):
    pc = params(tmp_path)
    planes, phasors = beam(pc)
    monkeypatch.setattr(incident, 'make_incident_beam',
                        lambda p, device=None: (planes, phasors, HeldRun()))

    class Sim:
        def __init__(self, params):
            pass

        def run_eps_sigma(self, eps, sig, name, meta):
            pass

    monkeypatch.setattr(experiment, 'get_fdtd_simulator', lambda p: Sim)
    monkeypatch.setattr(experiment, 'process_all_results', lambda d, p: None)
    g = pc.geom_params
    shape = (g.size_z_material, g.size_y, g.size_x)
    experiment.run_experiment(pc, [MaterialModel(np.ones(shape, np.float32),
                                                 np.zeros(shape, np.float32), g.cell_size, 'm')])
    assert os.path.exists(inc_filename(pc)) and not incident._WRITES


def test_concurrent_waiters_all_block_and_all_see_the_error(tmp_path, monkeypatch):
    """Two threads wait for the same background write: both return only once
    it has ended, and both get its error."""
    import threading
    pc = params(tmp_path)
    planes, phasors = beam(pc)
    started = threading.Event()

    def slow_fail(*a, **k):
        started.set()
        time.sleep(0.4)
        raise OSError('disk full')

    monkeypatch.setattr(incidentbeam, 'write_incident_file', slow_fail)
    incident.store_incident_beam(pc, planes, phasors, background=True)
    assert started.wait(5)
    fname = inc_filename(pc)
    seen = {}

    def waiter(k):
        t0 = time.perf_counter()
        try:
            incident.wait_written(fname)
            seen[k] = ('ok', time.perf_counter() - t0)
        except OSError as e:
            seen[k] = (str(e), time.perf_counter() - t0)

    ts = [threading.Thread(target=waiter, args=(k,)) for k in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(10)
    assert [seen[k][0] for k in range(2)] == ['disk full', 'disk full'], seen
    assert all(seen[k][1] > 0.2 for k in range(2)), seen     # both waited for the write
    assert not incident._WRITES
