"""Failure detection on the host, with no device and nothing that could
fault one: error codes injected through a stand-in for the C-ABI library
reach the caller as FdtdError with their code and message; a missing,
corrupt or truncated incident file is reported, not half-read; a simulator
error in the middle of an experiment ends it and stops the model prefetch."""
import ctypes
import os
import threading
import time

import numpy as np
import pytest

from fdtdsarsim_b200 import _native, experiment, incident, synthetic
from fdtdsarsim_b200.incidentbeam import IncidentBeam, write_incident_file
from fdtdsarsim_b200.materials import MaterialModel
from fdtdsarsim_b200.parameters import inc_filename
from helpers import make_params


class FailingLibrary:
    """Every entry point returns 0, except those named in ``codes``; the
    error text of the last failure is served by fdtd_last_error."""

    def __init__(self, codes):
        self.codes = codes
        self.message = b''

    def __getattr__(self, name):
        def call(*args):
            if name == 'fdtd_last_error':
                buf, n = args
                ctypes.memmove(buf, self.message, min(len(self.message), n - 1))
                return len(self.message)
            code = self.codes.get(name, 0)
            if code:
                self.message = f'{name}: injected failure {code}'.encode()
            return code
        return call


GEOM = dict(nx=27, ny=25, nz=23, npml=10, tfsf_z=14, nt=10, nt_inc=5, dtype=0, cell_size=1e-3,
            timestep=1e-12, frequency=5.4e9, db=1.0, dtm0=1.0, dte0dx=1.0)


@pytest.mark.parametrize('code', [_native.FDTD_ERR_INVALID, _native.FDTD_ERR_CUDA,
                                  _native.FDTD_ERR_STATE, _native.FDTD_ERR_NONFINITE,
                                  _native.FDTD_ERR_NOMEM])
def test_injected_error_codes_reach_the_caller(monkeypatch, code):
    lib = FailingLibrary({'fdtd_run': code, 'fdtd_synchronize': code})
    monkeypatch.setattr(_native, 'lib', lib)
    sim = _native.NativeSim(_native.Geometry(**GEOM), 0)
    sim.reset()                                        # succeeds
    for call in (lambda: sim.run(3), sim.synchronize):
        with pytest.raises(_native.FdtdError) as ei:
            call()
        assert ei.value.code == code and 'injected failure' in str(ei.value)
    sim.h = None                                       # nothing was allocated


def test_a_failed_create_leaves_no_handle(monkeypatch):
    monkeypatch.setattr(_native, 'lib', FailingLibrary({'fdtd_create': _native.FDTD_ERR_NOMEM}))
    with pytest.raises(_native.FdtdError) as ei:
        _native.NativeSim(_native.Geometry(**GEOM), 0)
    assert ei.value.code == _native.FDTD_ERR_NOMEM


def _incident_params(tmp_path):
    pc = make_params(27, 25, 23, 14, 10, 6)
    pc.processing_params.project_dir = str(tmp_path)
    return pc


def _write_beam(pc):
    g = pc.geom_params
    planes = synthetic.plane_wave_incident(pc, g.size_t_inc, 'float32')
    ph = {f'{c}_inc_phasor': np.zeros((g.size_y - 20, g.size_x - 20), np.complex64)
          for c in ('ex', 'ey', 'hx', 'hy')}
    write_incident_file(pc, planes['ex'], planes['ey'], planes['hx'], planes['hy'], ph)


def test_missing_incident_file(tmp_path):
    pc = _incident_params(tmp_path)
    assert not IncidentBeam(pc).inc_beam_exists()
    with pytest.raises(FileNotFoundError):
        IncidentBeam(pc).load_existing()


def test_corrupt_incident_file(tmp_path):
    pc = _incident_params(tmp_path)
    with open(inc_filename(pc), 'wb') as fh:
        fh.write(os.urandom(4096))
    with pytest.raises(OSError, match='signature'):
        IncidentBeam(pc).load_existing()


def test_truncated_incident_file(tmp_path):
    """A file cut short (a copy that stopped early) fails its read instead
    of returning fewer planes."""
    from fdtdsarsim_b200 import resultsio
    pc = _incident_params(tmp_path)
    _write_beam(pc)
    fname = inc_filename(pc)
    with resultsio.File(fname, 'r') as f:
        cut = f['ex']._addr + f['ex'].nbytes // 2        # inside the first plane set
        with open(fname, 'r+b') as fh:                    # the file shrinks while open
            fh.truncate(cut)
        with pytest.raises(OSError, match='truncated'):
            np.asarray(f['ex'][:])
        with pytest.raises(OSError, match='truncated'):
            f['ex'][1]
    with pytest.raises(OSError, match='truncated'):     # its metadata is gone too
        IncidentBeam(pc).load_existing()


def test_simulator_error_ends_the_experiment_and_the_prefetch(monkeypatch, tmp_path):
    pc = _incident_params(tmp_path)
    g = pc.geom_params
    shape = (g.size_z_material, g.size_y, g.size_x)
    made = []

    def models():
        for k in range(100):
            made.append(k)
            yield MaterialModel(np.ones(shape, np.float32), np.zeros(shape, np.float32),
                                g.cell_size, f'm{k}')

    class Sim:
        def __init__(self, params):
            self.n = 0

        def run_eps_sigma(self, eps, sig, name, meta):
            self.n += 1
            if self.n == 2:
                raise _native.FdtdError(_native.FDTD_ERR_NONFINITE, 'fields became non-finite')

    class Beam:
        def __init__(self, params):
            pass

        def setup(self):
            pass

    monkeypatch.setattr(experiment, 'get_fdtd_simulator', lambda p: Sim)
    monkeypatch.setattr(experiment, 'IncidentBeam', Beam)
    monkeypatch.setattr(experiment, 'process_all_results', lambda d, p: None)
    with pytest.raises(_native.FdtdError) as ei:
        experiment.run_experiment(pc, models())
    assert ei.value.code == _native.FDTD_ERR_NONFINITE
    time.sleep(0.5)
    n = len(made)
    time.sleep(0.3)
    assert len(made) == n <= 5                          # the producer stopped
    assert not [t for t in threading.enumerate()
                if t.name == 'material-prefetch' and t.is_alive()]
    assert not incident._WRITES
