"""run_experiment's host side without a device: the one-ahead material
prefetch (order, errors, early stop, overlap with the solve) and the
experiment loop of experiment.py:41-97 over a stand-in simulator."""
import threading
import time

import numpy as np
import pytest

from fdtdsarsim_b200 import experiment
from fdtdsarsim_b200.materials import MaterialModel
from helpers import make_params


def test_prefetched_keeps_order_and_items():
    for depth in (1, 3):
        assert list(experiment.prefetched(range(50), depth)) == list(range(50))
    assert list(experiment.prefetched([], 1)) == []


def test_prefetched_raises_where_the_producer_failed():
    def gen():
        yield 0
        yield 1
        raise ValueError('bad model')

    got = []
    with pytest.raises(ValueError, match='bad model'):
        for x in experiment.prefetched(gen()):
            got.append(x)
    assert got == [0, 1]


def test_prefetched_stops_the_producer_when_closed_early():
    made = []

    def gen():
        for k in range(1000):
            made.append(k)
            yield k

    it = experiment.prefetched(gen(), depth=1)
    assert [next(it), next(it)] == [0, 1]
    it.close()
    time.sleep(0.5)
    n = len(made)
    time.sleep(0.3)
    assert len(made) == n <= 5
    assert not [t for t in threading.enumerate() if t.name == 'material-prefetch' and t.is_alive()]


def test_prefetched_overlaps_producer_and_consumer():
    def gen():
        for k in range(6):
            time.sleep(0.15)          # making a model
            yield k

    t0 = time.perf_counter()
    for _ in experiment.prefetched(gen()):
        time.sleep(0.15)              # solving it
    overlapped = time.perf_counter() - t0
    assert overlapped < 0.75 * (6 * 0.3), overlapped


class FakeSim:
    calls = []

    def __init__(self, params):
        self.params = params

    def run_eps_sigma(self, eps_r, sigma, name, meta):
        g = self.params.geom_params
        assert eps_r.shape[1:] == (g.size_y, g.size_x)
        time.sleep(0.05)
        FakeSim.calls.append((name, float(eps_r[0, 0, 0])))


class FakeBeam:
    def __init__(self, params):
        pass

    def setup(self):
        pass


@pytest.fixture
def fake_device(monkeypatch):
    FakeSim.calls = []
    done = []
    monkeypatch.setattr(experiment, 'get_fdtd_simulator', lambda params: FakeSim)
    monkeypatch.setattr(experiment, 'IncidentBeam', FakeBeam)
    monkeypatch.setattr(experiment, 'process_all_results', lambda d, p: done.append(d))
    return done


def models(pc, n, eps0=2.0):
    g = pc.geom_params
    shape = (g.size_z_material, g.size_y, g.size_x)
    for k in range(n):
        yield MaterialModel(np.full(shape, eps0 + k, np.float32), np.zeros(shape, np.float32),
                            g.cell_size, f'm{k}', {'k': k})


@pytest.mark.parametrize('prefetch', [0, 1, 2])
def test_run_experiment_runs_every_model_in_order(fake_device, prefetch):
    pc = make_params(27, 25, 23, 14, 10, 5)
    experiment.run_experiment(pc, models(pc, 5), prefetch=prefetch)
    assert FakeSim.calls == [(f'm{k}', 2.0 + k) for k in range(5)]
    assert fake_device == [pc.processing_params.project_dir]


def test_run_experiment_takes_the_geometry_from_the_first_model(fake_device):
    """With no geometry in the parameters the first model sets it
    (experiment.py:66-80) before the next one is made."""
    pc = make_params(27, 25, 23, 14, 10, 5)
    made = list(models(pc, 3))
    g = pc.geom_params
    want = (g.size_x, g.size_y, g.size_z)
    g.size_x = g.size_y = g.size_z = 0
    seen = []

    def gen():
        for m in made:
            seen.append(g.size_x)       # the geometry when this model is made
            yield m

    experiment.run_experiment(pc, gen())
    assert (g.size_x, g.size_y) == want[:2]
    assert seen == [0, want[0], want[0]]
    assert [c[0] for c in FakeSim.calls] == ['m0', 'm1', 'm2']


def test_run_experiment_propagates_a_generator_error(fake_device):
    pc = make_params(27, 25, 23, 14, 10, 5)

    def broken():
        yield from models(pc, 2)
        raise RuntimeError('generator failed')

    with pytest.raises(RuntimeError, match='generator failed'):
        experiment.run_experiment(pc, broken())
    assert [c[0] for c in FakeSim.calls] == ['m0', 'm1']


def test_run_experiment_with_no_models(fake_device):
    """No models: no simulator is made when the geometry comes from the
    models (experiment.py:61-84), and the project is still post-processed."""
    pc = make_params(27, 25, 23, 14, 10, 5)
    pc.geom_params.size_x = pc.geom_params.size_y = pc.geom_params.size_z = 0
    experiment.run_experiment(pc, iter([]))
    assert FakeSim.calls == [] and fake_device == [pc.processing_params.project_dir]
