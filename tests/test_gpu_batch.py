"""Batched sweep (fdtd_batch_*): members of uneven sizes advanced together,
one launch per pass for all members, chunks replayed from a captured CUDA
graph. Each member must end with the oracle's fields and phasors bit for
bit, however the run is cut into calls and graph chunks."""
import pytest

from fdtdsarsim_b200 import _native
from helpers import bits_equal, make_params, native_for, oracle_for, random_problem

pytestmark = pytest.mark.gpu

MODELS = [
    # nx, ny, nz, tfsf_z, nt, ntp
    (27, 25, 23, 14, 30, 20),
    (41, 37, 29, 16, 30, 30),
    (35, 31, 27, 20, 30, 12),     # injection plane inside the upper CPML
    (150, 61, 37, 20, 30, 25),
]


def _members(models, seed, dtype='float32'):
    out = []
    for k, (nx, ny, nz, tfsf, nt, ntp) in enumerate(models):
        pc = make_params(nx, ny, nz, tfsf, nt, ntp, dtype=dtype)
        _, _, ca, cb, inc = random_problem(pc, seed + k)
        orc = oracle_for(pc)
        orc.run(ca, cb, inc, nt)
        sim = native_for(pc)
        sim.set_materials(ca, cb)
        sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
        out.append((orc, sim))
    return out


def _assert_member(orc, sim):
    for c in _native.FIELD_NAMES:
        assert bits_equal(sim.get_field(c), getattr(orc, c)), c
    for k, name in enumerate(_native.PHASOR_NAMES):
        assert bits_equal(sim.get_phasor(k), orc.ph[name]), name


@pytest.mark.parametrize('chunk,calls', [(0, (30,)), (7, (30,)), (4, (3, 10, 17)), (64, (1, 29))])
def test_batch_matches_oracle_for_every_member(chunk, calls):
    members = _members(MODELS, seed=500)
    batch = _native.Batch([s for _, s in members], graph_chunk=chunk)
    for n in calls:
        batch.run(n)
    batch.synchronize()
    for orc, sim in members:
        assert sim.step_index() == 30
        _assert_member(orc, sim)
    batch.close()
    for _, sim in members:
        sim.close()


@pytest.mark.parametrize('kernels', ['fused', 'mixed'])
def test_streams_mode_matches_oracle_for_every_member(kernels):
    """FDTD_OPT_BATCH_STREAMS: every member on its own stream with its own
    kernel (all fused, or fused and split mixed) ends with the oracle's
    fields and phasors; the all-or-nothing step check still applies; the
    mode can be switched between calls."""
    members = _members(MODELS, seed=560)
    sims = [s for _, s in members]
    if kernels == 'mixed':
        for s in sims[::2]:
            s.set_option(_native.OPT_KERNEL, _native.FDTD_KERNEL_SPLIT)
    batch = _native.Batch(sims, graph_chunk=4, streams=True)
    batch.run(7)
    with pytest.raises(_native.FdtdError):
        batch.run(24)             # would pass size_t: nothing runs
    batch.set_streams(False)
    batch.run(9)
    batch.set_streams(True)
    batch.run(14)
    batch.synchronize()
    for orc, sim in members:
        assert sim.step_index() == 30
        _assert_member(orc, sim)
    with pytest.raises(_native.FdtdError):
        _native.check(_native.lib.fdtd_batch_set_option(batch.h, _native.OPT_BATCH_STREAMS, 2))
    batch.close()


def test_batch_float64_members():
    members = _members(MODELS[:2], seed=520, dtype='float64')
    batch = _native.Batch([s for _, s in members], graph_chunk=8)
    batch.run(30)
    for orc, sim in members:
        _assert_member(orc, sim)
    batch.close()


def test_members_mix_own_steps_and_batch_steps():
    """A member that ran fused steps on its own (its current field set
    changed) joins the batch afterwards; the batch rebuilds its table."""
    members = _members(MODELS, seed=540)
    sims = [s for _, s in members]
    sims[1].set_option(_native.OPT_KERNEL, _native.FDTD_KERNEL_FUSED)
    sims[1].run(3)
    sims[3].set_option(_native.OPT_KERNEL, _native.FDTD_KERNEL_FUSED)
    sims[3].run(3)
    batch = _native.Batch(sims, graph_chunk=5)
    with pytest.raises(_native.FdtdError):
        batch.run(28)   # members 1 and 3 would pass size_t
    for s in (0, 2):
        sims[s].run(3)
    batch.run(20)
    sims[1].run(7)
    batch.run(0)
    for s in (0, 2, 3):
        sims[s].run(7)
    for orc, sim in members:
        assert sim.step_index() == 30
        _assert_member(orc, sim)
    batch.close()


def test_batch_rejects_bad_members():
    pc32 = make_params(27, 25, 23, 14, 10, 5)
    pc64 = make_params(27, 25, 23, 14, 10, 5, dtype='float64')
    a, b = native_for(pc32), native_for(pc64)
    with pytest.raises(_native.FdtdError):
        _native.Batch([a, b])
    with pytest.raises(_native.FdtdError):
        _native.Batch([a, a])
    with pytest.raises(_native.FdtdError):
        _native.Batch([])
    batch = _native.Batch([a])
    with pytest.raises(_native.FdtdError) as ei:
        batch.run(1)   # materials not set
    assert ei.value.code == _native.FDTD_ERR_STATE
    with pytest.raises(_native.FdtdError) as ei:
        a.close()      # a member outlives its batch
    assert ei.value.code == _native.FDTD_ERR_STATE and a.h is not None
    batch.close()
    a.close()
    assert a.h is None


# members for the tile queue: uneven grids, two wide enough for an interior
# box (x 32..), one with its injection plane in the upper CPML
QUEUE_MODELS = MODELS + [(261, 45, 30, 14, 30, 16), (173, 53, 40, 28, 30, 20)]


@pytest.mark.parametrize('chunk,calls', [(0, (30,)), (7, (30,)), (4, (3, 10, 17)), (64, (1, 29))])
def test_queue_mode_matches_oracle_for_every_member(chunk, calls):
    """FDTD_BATCH_QUEUE: every member's fused step, one persistent launch
    walking the interior z-march tiles of all members (longest first) and
    the batched split passes over all their shells. Odd calls flip every
    member's current field set, even graph chunks keep it; every member
    ends with the oracle's bits."""
    members = _members(QUEUE_MODELS, seed=580)
    batch = _native.Batch([s for _, s in members], graph_chunk=chunk, mode=_native.BATCH_QUEUE)
    for n in calls:
        batch.run(n)
    batch.synchronize()
    for orc, sim in members:
        assert sim.step_index() == 30
        _assert_member(orc, sim)
    batch.close()
    for _, sim in members:
        sim.close()


def test_queue_mode_interleaves_with_other_modes_and_own_steps():
    """The tile queue after a member's own steps, between split-pass and
    member-stream calls, in float32 and float64 members."""
    for dtype, models in (('float32', QUEUE_MODELS), ('float64', MODELS[:2] + QUEUE_MODELS[-1:])):
        members = _members(models, seed=600, dtype=dtype)
        sims = [s for _, s in members]
        for s in sims:
            s.set_option(_native.OPT_KERNEL, _native.FDTD_KERNEL_FUSED)
            s.run(1)
        batch = _native.Batch(sims, graph_chunk=6, mode=_native.BATCH_QUEUE)
        batch.run(9)
        batch.set_mode(_native.BATCH_SPLIT)
        batch.run(5)
        batch.set_mode(_native.BATCH_QUEUE)
        batch.run(8)
        batch.set_mode(_native.BATCH_STREAMS)
        batch.run(3)
        batch.set_mode(_native.BATCH_QUEUE)
        batch.run(4)
        batch.synchronize()
        for orc, sim in members:
            assert sim.step_index() == 30
            _assert_member(orc, sim)
        with pytest.raises(_native.FdtdError):
            batch.set_mode(3)
        batch.close()
        for s in sims:
            s.close()
