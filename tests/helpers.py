"""Shared builders for the parity tests: one seeded problem, run through the
oracle and through the C-ABI."""
import os

import numpy as np
import scipy.constants

import fdtd_oracle as O
from fdtdsarsim_b200 import _native
from fdtdsarsim_b200.absorbers import cpml_profiles, packed_profiles
from fdtdsarsim_b200.materials import MaterialModel, compute_material_arrays
from fdtdsarsim_b200.parameters import ParameterCollection

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
FREQ = 5.4e9
LAM = scipy.constants.c / FREQ


def make_params(nx, ny, nz, tfsf_z, nt, ntp, dtype='float32', cell_wl=0.021, nz_mat=None,
                npml=10):
    pc = ParameterCollection()
    pc.processing_params.processing_type = 'gpu'
    pc.processing_params.datatype = dtype
    pc.inc_beam_params.frequency = FREQ
    pc.inc_beam_params.polarization = 'HH'
    pc.inc_beam_params.theta_angle = 20.0
    g = pc.geom_params
    g.courant = 0.5
    g.size_pml = npml
    g.cell_size = LAM * cell_wl
    g.timestep = g.cell_size * g.courant / scipy.constants.c
    g.size_x, g.size_y, g.size_z = nx, ny, nz
    g.size_z_material = nz_mat if nz_mat is not None else max(1, min(nz - 1, tfsf_z - 2))
    g.tfsf_z = tfsf_z
    g.size_t = nt
    g.size_t_inc = ntp
    g.size_t_pulse = ntp // 2
    g.simulation_duration = 18.0
    return pc


def random_problem(pc, seed):
    """Seeded Ca/Cb (from random eps_r/sigma) and incident planes."""
    g = pc.geom_params
    dtype = pc.processing_params.datatype
    rng = np.random.default_rng(seed)
    shape = (g.size_z_material, g.size_y, g.size_x)
    eps = rng.uniform(1.0, 20.0, size=shape).astype(dtype)
    sig = rng.uniform(0.0, 0.3, size=shape).astype(dtype)
    ca, cb = compute_material_arrays(pc, MaterialModel(eps, sig, g.cell_size))
    inc = {}
    for comp, scale in (('ex', 1.0), ('ey', 1.0), ('hx', 1 / 376.73), ('hy', 1 / 376.73)):
        inc[comp] = (scale * rng.standard_normal((g.size_t_inc, g.size_y, g.size_x))).astype(dtype)
    return eps, sig, ca, cb, inc


def oracle_for(pc):
    g = pc.geom_params
    return O.OracleSim(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size,
                       g.timestep, pc.inc_beam_params.frequency,
                       pc.processing_params.datatype, cpml_profiles(pc))


def native_for(pc, kernel=_native.FDTD_KERNEL_SPLIT, tile=(32, 8), phasor_mode=0, zchunk=0, slab=False,
               shell=None):
    """A NativeSim for pc with the given step path. The fused step's shell
    is marched (SHELL_MARCH) unless ``shell`` says otherwise; ``slab`` (the
    z slabs marched beside split-pass strips) implies the split-pass shell."""
    from fdtdsarsim_b200.gpu.main_sim import native_geometry
    sim = _native.NativeSim(native_geometry(pc), 0)
    sim.set_absorbers(packed_profiles(pc))
    sim.set_option(_native.OPT_KERNEL, kernel)
    if kernel == _native.FDTD_KERNEL_FUSED:
        if shell is None:
            shell = _native.SHELL_SPLIT if slab else _native.SHELL_MARCH
        sim.set_option(_native.OPT_TILE_X, tile[0])
        sim.set_option(_native.OPT_TILE_Y, tile[1])
        sim.set_option(_native.OPT_ZCHUNK, zchunk)
        sim.set_option(_native.OPT_FUSED_SLAB, int(slab))
        sim.set_option(_native.OPT_SHELL, shell)
    sim.set_option(_native.OPT_PHASOR_MODE, phasor_mode)
    return sim


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    return np.array_equal(a.view(np.uint8), b.view(np.uint8))


def rel_err(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a - b)))
