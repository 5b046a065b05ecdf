"""Material blocks made on the device (fdtd_fill_layers, fdtd_paint_spheres,
fdtd_set_materials_staged) against the host: the staged block equals the
recipe's host arrays bit for bit (rough dielectric, one- and two-layer
soils, fixed and random bubbles, float32 and float64), a solve from the
staged block equals one from the uploaded host block, and run_experiment
with recipes writes the result files it writes for the host models."""
import numpy as np
import pytest

from fdtdsarsim_b200 import _native, resultsio
from fdtdsarsim_b200.experiment import run_experiment
from fdtdsarsim_b200.materials import bubbles, rough_dielectric, soilmodels
from fdtdsarsim_b200.parameters import results_filename
from helpers import bits_equal, make_params, native_for, random_problem

pytestmark = pytest.mark.gpu


def recipes(pc):
    out = list(rough_dielectric(pc, 7.0, 0.03, 0.004, 0.02, 0.01, 1, seed=300, device=True))
    out += list(soilmodels.one_layer_gaussian(pc, [0.2], 0.4, 0.2, 0.004, 0.01, 0.02, 1, 21, device=True))
    out += list(soilmodels.two_layer_gaussian(pc, 0.15, [0.3], 0.5, 0.1, 0.003, 0.01, 0.7, 0.025, 0.01,
                                              1, 23, device=True))
    r = next(rough_dielectric(pc, 6.0, 0.01, 0.004, 0.03, 0.012, 1, seed=41, device=True))
    bubbles.add_bubbles(r, r.heights[0].copy(), 0.2, 0.006, 3.15, 0.0, 77)
    bubbles.add_bubbles_randsize(r, r.heights[0].copy(), 0.1, 0.004, 0.009, 1.0, 0.0, 78)
    out.append(r)
    return out


@pytest.mark.parametrize('dtype', ['float32', 'float64'])
def test_staged_blocks_equal_the_host_arrays(dtype):
    pc = make_params(151, 47, 41, 28, 12, 10, dtype=dtype, nz_mat=16)
    pc.geom_params.cell_size = 0.003
    for rec in recipes(pc):
        want = rec.to_model()
        sim = native_for(pc, _native.FDTD_KERNEL_FUSED, (32, 4))
        try:
            rec.stage(sim)
            eps, sig = sim.get_staged_materials(rec.shape[0])
            assert bits_equal(eps, want.relative_permittivity), rec.name
            assert bits_equal(sig, want.conductivity), rec.name
        finally:
            sim.close()


def test_solve_from_a_staged_block_equals_the_uploaded_block():
    pc = make_params(151, 47, 41, 28, 20, 16, nz_mat=16)
    pc.geom_params.cell_size = 0.003
    _, _, _, _, inc = random_problem(pc, 5)
    rec = recipes(pc)[-1]
    m = rec.to_model()
    a, b = native_for(pc, _native.FDTD_KERNEL_FUSED, (32, 4)), native_for(pc, _native.FDTD_KERNEL_FUSED, (32, 4))
    try:
        a.set_materials_eps_sigma(m.relative_permittivity, m.conductivity)
        rec.stage(b)
        b.set_materials_staged()
        for s in (a, b):
            s.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
            s.run(20)
            s.synchronize()
        for c in _native.FIELD_NAMES:
            assert bits_equal(a.get_field(c), b.get_field(c)), c
    finally:
        a.close()
        b.close()


def test_run_experiment_with_recipes_writes_the_same_files(tmp_path):
    from fdtdsarsim_b200 import synthetic
    files = {}
    lam = 2.99792458e8 / 5.4e9
    for tag in ('host', 'device'):
        pc = synthetic.config_params('plain_2x2', 'float32', project_dir=str(tmp_path / tag))
        gen = rough_dielectric(pc, 5.0, 0.02, 0.05 * lam, 0.2 * lam, 0.2 * lam, 2, seed=9,
                               device=tag == 'device')
        run_experiment(pc, gen)
        files[tag] = [results_filename(pc, f'rough_surf_{i}') for i in range(2)]
    for fa, fb in zip(files['host'], files['device']):
        with resultsio.File(fa, 'r') as a, resultsio.File(fb, 'r') as b:
            for name in _native.PHASOR_NAMES:
                assert np.array_equal(a['phasors'][name][()], b['phasors'][name][()]), name
            assert np.array_equal(a['farfield']['e_phi'][()], b['farfield']['e_phi'][()])
