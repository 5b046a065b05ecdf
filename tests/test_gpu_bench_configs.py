"""Parity on the benchmark workloads themselves: the device path, through the
C-ABI, on the grids the bench line is measured on, against the C oracle
(the reference's float32 CPU step, restated; bit-identical to the reference's
fixtures) on every host core.

* plain_16x16 (203 x 761 x 761 cells, snowpack over rough soil, tapered
  plane wave, every step injecting): 16 fused steps, all six fields and the
  24 phasor planes bit for bit, with the shell marched (the default step)
  and with the split-pass shell;
* plain_8x8 (101 x 381 x 381 cells, rough lognormal soil): the full
  1714-step solve, all 24 phasor planes and the fields bit for bit, and the
  backscatter phasor and power (near-to-far transform of the upper plane,
  theta = -theta_inc, r = 2 km) within 1e-4 relative of the oracle's.

The C oracle needs about 2 s (16x16) and 20 s (8x8) on 16 host cores.
"""
import importlib.util
import os
import subprocess

import numpy as np
import pytest

import fdtd_oracle as O
import fdtd_oracle_c as OC
from fdtdsarsim_b200 import _native
from fdtdsarsim_b200.absorbers import cpml_profiles, packed_profiles
from fdtdsarsim_b200.gpu.main_sim import native_geometry
from helpers import bits_equal

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location('bench', os.path.join(ROOT, 'bench.py'))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _oracle(pc):
    if not OC.available():
        subprocess.run(['make', '-C', os.path.join(ROOT, 'oracle')], check=True, capture_output=True)
    g = pc.geom_params
    return OC.COracleSim(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size, g.timestep,
                         pc.inc_beam_params.frequency, pc.processing_params.datatype, cpml_profiles(pc))


def _device(pc, ca, cb, inc, steps, shell):
    sim = _native.NativeSim(native_geometry(pc), 0)
    sim.set_absorbers(packed_profiles(pc))
    sim.set_option(_native.OPT_KERNEL, _native.FDTD_KERNEL_FUSED)
    sim.set_option(_native.OPT_TILE_X, 32)
    sim.set_option(_native.OPT_TILE_Y, 4)
    sim.set_option(_native.OPT_SHELL, shell)
    sim.set_materials(ca, cb)
    sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
    sim.run(steps)
    sim.synchronize()
    return sim


@pytest.fixture(scope='module')
def plain_16x16():
    steps = 16
    pc, ca, cb, inc = _bench().build_workload('plain_16x16', 'float32', steps + 1)
    orc = _oracle(pc)
    orc.run(ca, cb, inc, steps)
    return pc, ca, cb, inc, steps, orc


@pytest.mark.parametrize('shell', [_native.SHELL_MARCH, _native.SHELL_SPLIT], ids=['march', 'split'])
def test_plain_16x16_steps_bit_exact(plain_16x16, shell):
    pc, ca, cb, inc, steps, orc = plain_16x16
    assert (pc.geom_params.size_z, pc.geom_params.size_y, pc.geom_params.size_x) == (203, 761, 761)
    sim = _device(pc, ca, cb, inc, steps, shell)
    try:
        for c in _native.FIELD_NAMES:
            assert bits_equal(sim.get_field(c), getattr(orc, c)), c
        got = sim.get_phasors()
        for name in _native.PHASOR_NAMES:
            assert bits_equal(got[name], orc.ph[name]), name
    finally:
        sim.close()


def _backscatter(pc, ph):
    g, b = pc.geom_params, pc.inc_beam_params
    ff = O.near2far(ph['ex_ph_u'], ph['ey_ph_u'], ph['hx_ph_u'], ph['hy_ph_u'],
                    g.size_x - 2 * g.size_pml, g.size_y - 2 * g.size_pml, g.size_z - 2 * g.size_pml,
                    g.cell_size, 2.0e3, [-b.theta_angle], [b.phi_angle], b.frequency)
    p_h, p_v = O.farfield_power(ff['E_theta'], ff['E_phi'], ff['H_theta'], ff['H_phi'])
    if b.polarization.upper() == 'HH':
        return complex(np.ravel(ff['E_phi'])[0]), float(np.ravel(p_h)[0])
    return complex(np.ravel(ff['E_theta'])[0]), float(np.ravel(p_v)[0])


def test_plain_8x8_full_solve():
    pc, ca, cb, inc = _bench().build_workload('plain_8x8', 'float32', 10 ** 6)
    g = pc.geom_params
    assert (g.size_z, g.size_y, g.size_x, g.size_t) == (101, 381, 381, 1714)
    orc = _oracle(pc)
    orc.run(ca, cb, inc, g.size_t)
    sim = _device(pc, ca, cb, inc, g.size_t, _native.SHELL_MARCH)
    try:
        got = sim.get_phasors()
        for name in _native.PHASOR_NAMES:
            assert bits_equal(got[name], orc.ph[name]), name
        for c in _native.FIELD_NAMES:
            assert bits_equal(sim.get_field(c), getattr(orc, c)), c
        e_dev, p_dev = _backscatter(pc, got)
        e_orc, p_orc = _backscatter(pc, orc.ph)
        assert p_orc > 0
        assert abs(e_dev - e_orc) <= 1e-4 * abs(e_orc)
        assert abs(p_dev - p_orc) <= 1e-4 * p_orc
    finally:
        sim.close()
