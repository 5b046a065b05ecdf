"""Material recipes for the device (materials/device.py LayeredMaterial),
on the CPU: each generator's device=True recipe gives, through to_model(),
the arrays of the same generator on the host for the same seed (those are
pinned to the reference's own output in test_material_generators.py), the
bubble sphere lists replay the reference's draws, and the volume counted
from the heights equals the count on the arrays."""
import numpy as np
import pytest

from fdtdsarsim_b200.materials import bubbles, rough_dielectric, soilmodels
from fdtdsarsim_b200.materials.device import LayeredMaterial
from helpers import make_params

DX = 0.003


def params(nz_mat=12):
    pc = make_params(23, 21, 30, 20, 10, 5)
    pc.geom_params.size_z_material = nz_mat
    pc.geom_params.cell_size = DX
    return pc


def same(recipe, model):
    got = recipe.to_model()
    assert isinstance(recipe, LayeredMaterial) and recipe.name == model.name
    assert got.relative_permittivity.dtype == model.relative_permittivity.dtype
    assert np.array_equal(got.relative_permittivity, model.relative_permittivity)
    assert np.array_equal(got.conductivity, model.conductivity)
    assert recipe.material_volume() == bubbles.material_volume(model.relative_permittivity,
                                                               model.conductivity) or recipe.spheres


def test_rough_dielectric_recipes():
    pc = params()
    for r, m in zip(rough_dielectric(pc, 7.0, 0.03, 0.004, 0.02, 0.01, 2, seed=300, device=True),
                    rough_dielectric(pc, 7.0, 0.03, 0.004, 0.02, 0.01, 2, seed=300)):
        same(r, m)


def test_soil_recipes():
    pc = params()
    n = 0
    for dev, host in (
            (soilmodels.one_layer_gaussian(pc, [0.1, 0.3], 0.4, 0.2, 0.004, 0.01, 0.02, 2, 21, device=True),
             soilmodels.one_layer_gaussian(pc, [0.1, 0.3], 0.4, 0.2, 0.004, 0.01, 0.02, 2, 21)),
            (soilmodels.one_layer_gaussian(pc, [0.2], 0.4, 0.2, 0.004, 0.01, 0.02, 1, 22, grooved=True,
                                           rabus_compat=True, device=True),
             soilmodels.one_layer_gaussian(pc, [0.2], 0.4, 0.2, 0.004, 0.01, 0.02, 1, 22, grooved=True,
                                           rabus_compat=True)),
            (soilmodels.two_layer_gaussian(pc, 0.15, [0.3, 0.35], 0.5, 0.1, 0.003, 0.01, 0.7, 0.025, 0.01,
                                           1, 23, device=True),
             soilmodels.two_layer_gaussian(pc, 0.15, [0.3, 0.35], 0.5, 0.1, 0.003, 0.01, 0.7, 0.025, 0.01,
                                           1, 23))):
        for r, m in zip(dev, host):
            same(r, m)
            n += 1
    assert n == 7


@pytest.mark.parametrize('randsize', [False, True], ids=['fixed', 'random'])
def test_bubble_recipes_replay_the_draws(randsize):
    pc = params(nz_mat=24)
    r = next(rough_dielectric(pc, 6.0, 0.01, 0.004, 0.05, 0.012, 1, seed=41, device=True))
    m = next(rough_dielectric(pc, 6.0, 0.01, 0.004, 0.05, 0.012, 1, seed=41))
    surf = r.heights[0].copy()
    for target in (r, m):
        if randsize:
            bubbles.add_bubbles_randsize(target, surf, 0.2, 0.004, 0.009, 3.15, 0.0, 77)
        else:
            bubbles.add_bubbles(target, surf, 0.2, 0.006, 3.15, 0.0, 77)
    assert len(r.spheres) == 1 and len(r.spheres[0][0]) > 3
    same(r, m)
    assert r.metadata == m.metadata
