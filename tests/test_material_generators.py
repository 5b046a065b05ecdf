"""The material generators against the reference's own output on seeded
cases (tests/golden/material_gen.npz, made by tests/golden/make_golden.py
from fdtdsarsim.materials: roughsurface.py, dielectricmodels.py,
bubbles.py, soilmodels.py, materials.py:112-164)."""
import os

import numpy as np
import pytest

from helpers import GOLDEN, make_params
from fdtdsarsim_b200.materials import (HallikainenSoilModel, MaterialModel, bubbles,
                                       gaussian_correlated_surface,
                                       gaussian_correlated_surface_fast, hallikainen_soil_model,
                                       rough_dielectric, soilmodels,
                                       two_layer_gaussian_correlated_surface)

G = np.load(os.path.join(GOLDEN, 'material_gen.npz'))
DX = 0.003


def params():
    pc = make_params(23, 21, 30, 20, 10, 5)
    pc.geom_params.size_z_material = 12
    pc.geom_params.cell_size = DX
    return pc


def close(a, b, rel):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) <= rel * np.max(np.abs(b))


def test_surfaces():
    assert close(gaussian_correlated_surface(41, 37, DX, 0.010, 0.015, 0.002, seed=11), G['gcs'], 1e-12)
    assert close(gaussian_correlated_surface(41, 37, DX, 0.010, 0.015, 0.002, seed=11,
                                             rabus_compat=True), G['gcs_rabus'], 1e-12)
    fast = gaussian_correlated_surface_fast(41, 37, DX, 0.010, 0.015, 0.002, np.random.default_rng(12))
    assert fast.dtype == np.float32 and close(fast, G['gcs_fast'], 1e-5)
    assert close(two_layer_gaussian_correlated_surface(41, 37, DX, 0.010, 0.012, 0.002, 0.6, seed=13),
                 G['two_layer'], 1e-12)
    assert close(two_layer_gaussian_correlated_surface(41, 37, DX, 0.010, 0.012, 0.002, 1.0, seed=14),
                 G['two_layer_full'], 1e-12)


def test_hallikainen():
    m = HallikainenSoilModel()
    got_c = np.array([m.get_epsilon(*c) for c in G['hall_cases']])
    got_f = np.array([hallikainen_soil_model(*c) for c in G['hall_cases']])
    assert close(got_c, G['hall_class'], 1e-14)
    assert close(got_f, G['hall_func'], 1e-14)
    with pytest.raises(ValueError):
        m.get_epsilon(0.2, 0.3, 0.2, 20e9)
    with pytest.raises(ValueError):
        m.get_epsilon(1.2, 0.3, 0.2, 5e9)


def models_equal(gen, tag):
    n = 0
    for i, m in enumerate(gen):
        assert m.relative_permittivity.dtype == np.float32
        assert np.array_equal(m.relative_permittivity, G[f'{tag}_{i}_eps']), (tag, i)
        assert np.allclose(m.conductivity, G[f'{tag}_{i}_sig'], rtol=1e-6, atol=0), (tag, i)
        if f'{tag}_{i}_name' in G.files:
            assert m.name == str(G[f'{tag}_{i}_name'])
        n += 1
    return n


def test_rough_dielectric_seeded():
    assert models_equal(rough_dielectric(params(), 7.0, 0.03, 0.004, 0.02, 0.01, 2, seed=300), 'rough') == 2


def test_soil_models():
    pc = params()
    assert models_equal(soilmodels.one_layer_gaussian(pc, [0.1, 0.3], 0.4, 0.2, 0.004, 0.01, 0.02, 2, 21),
                        'one') == 4
    assert models_equal(soilmodels.one_layer_gaussian(pc, [0.2], 0.4, 0.2, 0.004, 0.01, 0.02, 1, 22,
                                                      grooved=True, rabus_compat=True), 'one_groove') == 1
    assert models_equal(soilmodels.two_layer_gaussian(pc, 0.15, [0.3, 0.35], 0.5, 0.1, 0.003, 0.01, 0.7,
                                                      0.025, 0.01, 1, 23), 'two') == 2
    assert models_equal(soilmodels.gradient_gaussian(pc, 0.1, [0.35], 0.5, 0.1, 0.003, 0.01, 0.7,
                                                     0.025, 0.01, 1, 24), 'grad') == 1
    assert models_equal(soilmodels.gradient_gaussian(pc, 0.1, [0.3], 0.5, 0.1, 0.003, 0.01, 0.7,
                                                     0.025, 0.01, 1, 25, grooved=True), 'grad_groove') == 1
    with pytest.raises(ValueError):
        next(soilmodels.one_layer_gaussian(pc, [0.1], 0.4, 0.2, 0.004, 0.01, 1.0, 1, 1))


@pytest.mark.parametrize('tag', ['bub', 'bub_rand'])
def test_bubbles(tag):
    m = MaterialModel(G[f'{tag}_in_eps'].copy(), G[f'{tag}_in_sig'].copy(), DX, 'b', {})
    if tag == 'bub':
        r = bubbles.add_bubbles(m, G['bub_surf'], 0.15, 0.0065, 3.2, 0.0, 31)
    else:
        r = bubbles.add_bubbles_randsize(m, G['bub_surf'], 0.15, 0.004, 0.008, 3.2, 0.0, 32)
    assert np.array_equal(r.relative_permittivity, G[f'{tag}_eps'])
    assert np.array_equal(r.conductivity, G[f'{tag}_sig'])
    assert bubbles.material_volume(G[f'{tag}_in_eps'], G[f'{tag}_in_sig']) == np.sum(G[f'{tag}_in_eps'] != 1.0)
