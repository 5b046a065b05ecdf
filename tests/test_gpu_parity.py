"""CUDA path vs the oracle (and vs the reference's own fixtures), through the
C-ABI. In the reference phasor mode the device reproduces the reference's
float32 arithmetic bit for bit, so fields and phasors are compared exactly;
the Kahan mode is held to the 1e-4 relative bar of the metric."""
import os

import numpy as np
import pytest

from fdtdsarsim_b200 import _native
from helpers import (GOLDEN, bits_equal, make_params, native_for, oracle_for, random_problem,
                     rel_err)

pytestmark = pytest.mark.gpu

SPLIT, FUSED = _native.FDTD_KERNEL_SPLIT, _native.FDTD_KERNEL_FUSED

CASES = [
    # nx, ny, nz, tfsf_z, nt, ntp, dtype
    (27, 25, 23, 14, 40, 30, 'float32'),
    (41, 37, 29, 16, 35, 35, 'float32'),     # nx, ny not multiples of anything
    (27, 25, 23, 20, 30, 20, 'float32'),     # injection plane inside the upper CPML
    (33, 23, 25, 12, 25, 10, 'float64'),
]


# Grids wider than one fused tile (128 x cells): several x tiles, a partial
# last tile, an x CPML face that straddles a tile edge (nx = 261: x 251..260,
# tile edge 256), and a pitch that is not a multiple of the tile (nx = 150).
WIDE = [
    (261, 45, 30, 14, 24, 16, 'float32'),
    (150, 61, 37, 20, 20, 20, 'float32'),
    (140, 33, 26, 12, 16, 10, 'float64'),
    # injection plane at the lower / upper end of the fused interior z range
    (300, 70, 40, 10, 12, 8, 'float32'),
    (173, 53, 40, 28, 12, 8, 'float32'),
    # injection plane just below the interior (npml - 1) and just below the
    # upper CPML slab (nz - npml - 1): neither box may march through it
    (41, 37, 29, 9, 20, 15, 'float32'),
    (41, 37, 29, 18, 20, 15, 'float32'),
    # tall grid: the shell march cuts its x and y strips into several z
    # chunks (each recomputing the plane below it)
    (140, 45, 200, 100, 10, 8, 'float32'),
]


def _run_both(case, seed, kernel=SPLIT, tile=(32, 8), phasor_mode=0, steps=None, zchunk=0, shell=None):
    nx, ny, nz, tfsf, nt, ntp, dtype = case
    pc = make_params(nx, ny, nz, tfsf, nt, ntp, dtype=dtype)
    _, _, ca, cb, inc = random_problem(pc, seed)
    orc = oracle_for(pc)
    steps = nt if steps is None else steps
    orc.run(ca, cb, inc, steps)
    sim = native_for(pc, kernel, tile, phasor_mode, zchunk, shell=shell)
    sim.set_materials(ca, cb)
    sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
    sim.run(steps)
    sim.synchronize()
    return orc, sim


@pytest.mark.parametrize('case', CASES)
def test_split_matches_oracle_bit_exact(case):
    orc, sim = _run_both(case, seed=101)
    for c in _native.FIELD_NAMES:
        assert bits_equal(sim.get_field(c), getattr(orc, c)), c
    for k, name in enumerate(_native.PHASOR_NAMES):
        assert bits_equal(sim.get_phasor(k), orc.ph[name]), name
    sim.close()


def _assert_matches(orc, sim):
    for c in _native.FIELD_NAMES:
        assert bits_equal(sim.get_field(c), getattr(orc, c)), c
    for k, name in enumerate(_native.PHASOR_NAMES):
        assert bits_equal(sim.get_phasor(k), orc.ph[name]), name


@pytest.mark.parametrize('shell', [_native.SHELL_MARCH, _native.SHELL_SPLIT], ids=['march', 'split'])
@pytest.mark.parametrize('case', CASES + WIDE)
def test_fused_matches_oracle_bit_exact(case, shell):
    """The fused step with its shell marched (the default: CPML faces,
    domain edges and the injection plane inside a z-march beside the
    interior march) or swept by the split passes."""
    orc, sim = _run_both(case, seed=202, kernel=FUSED, shell=shell)
    _assert_matches(orc, sim)
    sim.close()


@pytest.mark.parametrize('tile_y', [4, 8])
def test_march_shell_tiles(tile_y):
    """The shell march beside interior tiles of other heights, and a grid
    whose interior is narrower than one 128-cell row (8- and 16-lane rows
    in the strips and slabs)."""
    for case in (WIDE[0], (67, 91, 43, 30, 16, 12, 'float32')):
        orc, sim = _run_both(case, seed=404 + tile_y, kernel=FUSED, tile=(32, tile_y),
                             shell=_native.SHELL_MARCH)
        _assert_matches(orc, sim)
        sim.close()


@pytest.mark.parametrize('slab', [1, 2])
@pytest.mark.parametrize('case', CASES + WIDE)
def test_fused_slab_matches_oracle_bit_exact(case, slab):
    """FDTD_OPT_FUSED_SLAB: 1, the CPML z slabs marched by the slab kernel;
    2, the column march (the interior's x-y box over every plane, z faces,
    domain edge planes and injection plane in the march)."""
    pc = make_params(*case[:6], dtype=case[6])
    _, _, ca, cb, inc = random_problem(pc, 71)
    o = oracle_for(pc)
    o.run(ca, cb, inc, pc.geom_params.size_t)
    sim = native_for(pc, FUSED, (32, 4), slab=slab)
    try:
        sim.set_materials(ca, cb)
        sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
        sim.run(pc.geom_params.size_t)
        sim.synchronize()
        for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
            assert bits_equal(sim.get_field(c), getattr(o, c)), c
        for k, name in enumerate(_native.PHASOR_NAMES):
            assert bits_equal(sim.get_phasor(k), o.ph[name]), name
    finally:
        sim.close()


@pytest.mark.parametrize('zchunk', [1, 3, 7])
@pytest.mark.parametrize('case', [WIDE[0], WIDE[3], WIDE[4], WIDE[7]])
def test_column_march_chunks_start_anywhere(case, zchunk):
    """The column march in short z chunks: chunks start on the injection
    plane, the plane above it, inside the CPML slabs and at plane 0; each
    recomputes the plane below it with every plane-uniform term."""
    pc = make_params(*case[:6], dtype=case[6])
    _, _, ca, cb, inc = random_problem(pc, 73 + zchunk)
    o = oracle_for(pc)
    steps = min(pc.geom_params.size_t, 12)
    o.run(ca, cb, inc, steps)
    sim = native_for(pc, FUSED, (32, 4), zchunk=zchunk, slab=2)
    try:
        sim.set_materials(ca, cb)
        sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
        sim.run(steps)
        sim.synchronize()
        for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
            assert bits_equal(sim.get_field(c), getattr(o, c)), c
        for k, name in enumerate(_native.PHASOR_NAMES):
            assert bits_equal(sim.get_phasor(k), o.ph[name]), name
    finally:
        sim.close()


@pytest.mark.parametrize('tile_y,zchunk', [(4, 3), (7, 5), (8, 0), (15, 7), (16, 1)])
def test_fused_tiles_and_chunks(tile_y, zchunk):
    """Every tile height, and z chunks down to one plane (each chunk then
    recomputes the plane below it)."""
    case = WIDE[0] if tile_y != 16 else WIDE[1]
    orc, sim = _run_both(case, seed=303, kernel=FUSED, tile=(32, tile_y), zchunk=zchunk)
    _assert_matches(orc, sim)
    sim.close()


def test_fused_rejects_unsupported_tiles():
    pc = make_params(27, 25, 23, 14, 10, 5)
    _, _, ca, cb, inc = random_problem(pc, 1)
    for tile in ((16, 8), (32, 5)):
        sim = native_for(pc, FUSED, tile)
        sim.set_materials(ca, cb)
        sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
        with pytest.raises(_native.FdtdError) as ei:
            sim.run(1)
        assert ei.value.code == _native.FDTD_ERR_INVALID
        sim.close()


def test_kernels_can_alternate_within_a_run():
    """Fused steps use the ping-pong field and psi sets, split steps the
    current set in place; switching between them at any step keeps the
    oracle's values."""
    case = WIDE[0]
    nx, ny, nz, tfsf, nt, ntp, dtype = case
    pc = make_params(nx, ny, nz, tfsf, nt, ntp, dtype=dtype)
    _, _, ca, cb, inc = random_problem(pc, 17)
    orc = oracle_for(pc)
    orc.run(ca, cb, inc, nt)
    sim = native_for(pc, FUSED)
    sim.set_materials(ca, cb)
    sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
    done = 0
    for n, k in ((3, FUSED), (2, SPLIT), (5, FUSED), (1, SPLIT), (nt - 11, FUSED)):
        sim.set_option(_native.OPT_KERNEL, k)
        sim.run(n)
        done += n
    sim.synchronize()
    assert done == nt
    _assert_matches(orc, sim)
    sim.close()


def test_fused_runs_in_chunks_and_resets():
    case = WIDE[1]
    nx, ny, nz, tfsf, nt, ntp, dtype = case
    pc = make_params(nx, ny, nz, tfsf, nt, ntp, dtype=dtype)
    _, _, ca, cb, inc = random_problem(pc, 23)
    orc = oracle_for(pc)
    orc.run(ca, cb, inc, nt)
    sim = native_for(pc, FUSED)
    sim.set_materials(ca, cb)
    sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
    for _ in range(2):
        sim.reset()
        for n in (1, 4, 7, nt - 12):
            sim.run(n)
        sim.synchronize()
        _assert_matches(orc, sim)
    sim.close()


@pytest.mark.parametrize('kernel', [SPLIT, FUSED], ids=['split', 'fused'])
@pytest.mark.parametrize('tag', ['f32', 'f32_tfsf_in_pml'])
def test_device_reproduces_reference_fixture(tag, kernel):
    """Same inputs the reference ran on (tests/golden), same CPML profiles:
    fields and 24 phasor planes equal the reference's outputs exactly."""
    g = np.load(os.path.join(GOLDEN, f'mainloop_{tag}.npz'))
    ab = np.load(os.path.join(GOLDEN, 'absorbers.npz'))
    pc = make_params(int(g['nx']), int(g['ny']), int(g['nz']), int(g['tfsf_z']), int(g['nt']),
                     int(g['ntp']))
    assert pc.geom_params.cell_size == float(g['dx'])
    from fdtdsarsim_b200.gpu.main_sim import native_geometry
    sim = _native.NativeSim(native_geometry(pc), 0)
    sim.set_absorbers(np.concatenate([ab[f'float32_0.021_{k}'] for k in
                                      ('be_d', 'bh_d', 'ce_d', 'ch_d', 'be_u', 'bh_u',
                                       'ce_u', 'ch_u')]))
    sim.set_option(_native.OPT_KERNEL, kernel)
    sim.set_option(_native.OPT_ZCHUNK, 4)
    sim.set_materials(g['ca'], g['cb'])
    sim.set_incident(g['inc_ex'], g['inc_ey'], g['inc_hx'], g['inc_hy'])
    sim.run(int(g['nt']))
    sim.synchronize()
    for c in _native.FIELD_NAMES:
        assert bits_equal(sim.get_field(c), g[f'field_{c}']), c
    for k, name in enumerate(_native.PHASOR_NAMES):
        assert bits_equal(sim.get_phasor(k), g[name]), name
    sim.close()


@pytest.mark.parametrize('case', CASES[:2])
def test_kahan_phasors_within_tolerance(case):
    orc, sim = _run_both(case, seed=7, phasor_mode=_native.FDTD_PHASOR_KAHAN)
    for c in _native.FIELD_NAMES:
        assert bits_equal(sim.get_field(c), getattr(orc, c)), c
    for k, name in enumerate(_native.PHASOR_NAMES):
        err = rel_err(sim.get_phasor(k), orc.ph[name])
        assert err < 1e-5, (name, err)   # metric bar: 1e-4 relative
    sim.close()


def test_split_runs_in_chunks_and_resets():
    case = CASES[0]
    nx, ny, nz, tfsf, nt, ntp, dtype = case
    pc = make_params(nx, ny, nz, tfsf, nt, ntp, dtype=dtype)
    _, _, ca, cb, inc = random_problem(pc, 5)
    orc = oracle_for(pc)
    orc.run(ca, cb, inc, nt)
    sim = native_for(pc)
    sim.set_materials(ca, cb)
    sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
    for _ in range(2):
        sim.reset()
        for n in (1, 7, 12, nt - 20):
            sim.run(n)
        sim.synchronize()
        assert sim.step_index() == nt
        for c in _native.FIELD_NAMES:
            assert bits_equal(sim.get_field(c), getattr(orc, c)), c
        assert bits_equal(sim.get_phasor(5), orc.ph['ey_ph_u'])
    with pytest.raises(_native.FdtdError):
        sim.run(1)   # beyond size_t
    sim.close()


def test_eps_sigma_on_device_matches_host_coefficients():
    case = CASES[1]
    nx, ny, nz, tfsf, nt, ntp, dtype = case
    pc = make_params(nx, ny, nz, tfsf, nt, ntp, dtype=dtype)
    eps, sig, ca, cb, inc = random_problem(pc, 9)
    a = native_for(pc)
    a.set_materials(ca, cb)
    b = native_for(pc)
    b.set_materials_eps_sigma(eps, sig)
    for s in (a, b):
        s.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
        s.run(20)
        s.synchronize()
    for c in _native.FIELD_NAMES:
        assert bits_equal(a.get_field(c), b.get_field(c)), c
    a.close()
    b.close()


def test_state_errors():
    pc = make_params(27, 25, 23, 14, 10, 5)
    sim = native_for(pc)
    with pytest.raises(_native.FdtdError) as ei:
        sim.run(1)
    assert ei.value.code == _native.FDTD_ERR_STATE
    with pytest.raises(_native.FdtdError):
        sim.get_phasor(24)
    with pytest.raises(ValueError):
        sim.set_materials(np.zeros((3, 3, 3), np.float32), np.zeros((3, 3, 3), np.float32))
    sim.close()


@pytest.mark.parametrize('pinned', [False, True], ids=['pageable', 'pinned'])
@pytest.mark.parametrize('kernel', [SPLIT, FUSED], ids=['split', 'fused'])
def test_streamed_run_equals_resident_planes(pinned, kernel):
    """fdtd_run_streamed (planes copied 16 steps at a time beside the time
    stepping) steps exactly like a run on planes uploaded beforehand, across
    calls that end inside a transfer group and past the last incident step."""
    import torch
    pc = make_params(150, 41, 33, 16, 60, 45)
    _, _, ca, cb, inc = random_problem(pc, 21)
    comps = [inc[c] for c in ('ex', 'ey', 'hx', 'hy')]
    if pinned:
        comps = [torch.from_numpy(c).pin_memory().numpy() for c in comps]
    a, b = native_for(pc, kernel), native_for(pc, kernel)
    try:
        for s in (a, b):
            s.set_materials(ca, cb)
        a.set_incident(*comps)
        a.run(60)
        a.synchronize()
        for n in (7, 20, 33):
            b.run_streamed(n, *comps)
        for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
            assert bits_equal(a.get_field(c), b.get_field(c)), c
        for k in (4, 7, 13):
            assert bits_equal(a.get_phasor(k), b.get_phasor(k)), k
    finally:
        a.close()
        b.close()


def test_non_finite_check_reports_the_step():
    """FDTD_OPT_CHECK_EVERY: a NaN planted in the host-side initial field
    (no device fault involved) is reported by fdtd_synchronize as
    FDTD_ERR_NONFINITE with the first checked step after it; a clean run
    with the check on passes and steps exactly like one without."""
    pc = make_params(41, 37, 29, 16, 12, 10)
    _, _, ca, cb, inc = random_problem(pc, 33)
    comps = [inc[c] for c in ('ex', 'ey', 'hx', 'hy')]
    a, b = native_for(pc), native_for(pc)
    try:
        for s in (a, b):
            s.set_materials(ca, cb)
            s.set_incident(*comps)
        b.set_option(_native.OPT_CHECK_EVERY, 3)
        a.run(12)
        b.run(12)
        a.synchronize()
        b.synchronize()
        assert bits_equal(a.get_field('ey'), b.get_field('ey'))
        b.reset()
        hz = np.zeros((29, 37, 41), np.float32)
        hz[14, 18, 20] = np.nan
        b.set_field('hz', hz)
        b.run(7)
        with pytest.raises(_native.FdtdError) as ei:
            b.synchronize()
        assert ei.value.code == _native.FDTD_ERR_NONFINITE
        assert 'after step 3' in str(ei.value)
        b.reset()
        b.run(4)
        b.synchronize()
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize('kernel', [SPLIT, FUSED], ids=['split', 'fused'])
def test_graph_chunks_equal_direct_launches(kernel):
    """FDTD_OPT_GRAPH_CHUNK: steps replayed from captured graphs (odd chunk,
    so the fused step's field sets alternate between replays; a tile change
    forces a new capture) equal directly launched steps bit for bit."""
    pc = make_params(150, 41, 33, 16, 40, 30)
    _, _, ca, cb, inc = random_problem(pc, 44)
    comps = [inc[c] for c in ('ex', 'ey', 'hx', 'hy')]
    a, b = native_for(pc, kernel), native_for(pc, kernel)
    try:
        for s in (a, b):
            s.set_materials(ca, cb)
            s.set_incident(*comps)
        b.set_option(_native.OPT_GRAPH_CHUNK, 5)
        for s in (a, b):
            s.run(13)
        if kernel == FUSED:
            for s in (a, b):
                s.set_option(_native.OPT_TILE_Y, 8)
        for s in (a, b):
            s.run(27)
            s.synchronize()
        for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
            assert bits_equal(a.get_field(c), b.get_field(c)), c
        for k in (0, 4, 9, 17):
            assert bits_equal(a.get_phasor(k), b.get_phasor(k)), k
        assert b.step_index() == 40
    finally:
        a.close()
        b.close()


def test_all_phasors_in_one_call():
    """fdtd_get_phasors (one call, into a pageable or a page-locked buffer)
    returns the 24 planes of fdtd_get_phasor bit for bit."""
    import torch
    pc = make_params(41, 37, 29, 16, 12, 10)
    _, _, ca, cb, inc = random_problem(pc, 35)
    sim = native_for(pc, FUSED, (32, 4))
    try:
        sim.set_materials(ca, cb)
        sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
        sim.run(12)
        sim.synchronize()
        pinned = torch.empty(2 * sim.phasors_size(), dtype=torch.float32).pin_memory().numpy()
        for out in (None, pinned.view(np.complex64)):
            got = sim.get_phasors(out)
            for k, name in enumerate(_native.PHASOR_NAMES):
                assert bits_equal(got[name], sim.get_phasor(k)), name
    finally:
        sim.close()
