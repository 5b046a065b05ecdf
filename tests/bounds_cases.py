"""Cases for the bounds-checked build (run by test_gpu_bounds.py in a child
process with FDTDSARSIM_B200_LIBRARY=check): tiny and ragged grids through
every step path, each compared with the oracle bit for bit; any access a
kernel makes outside its allocation or shared array is reported by
synchronize as FDTD_ERR_BOUNDS. Prints one JSON line."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, os.path.join(ROOT, 'sar-pixel-simulator_b200'), os.path.join(ROOT, 'oracle')):
    if p not in sys.path:
        sys.path.insert(0, p)

from fdtdsarsim_b200 import _native  # noqa: E402
from helpers import bits_equal, make_params, native_for, oracle_for, random_problem  # noqa: E402

SPLIT, FUSED = _native.FDTD_KERNEL_SPLIT, _native.FDTD_KERNEL_FUSED

# nx, ny, nz, tfsf_z, nt, ntp, dtype
GRIDS = [
    (23, 23, 23, 12, 10, 8, 'float32'),      # the smallest grid npml 10 allows
    (133, 27, 29, 14, 10, 8, 'float32'),     # nx just past a 128-cell tile
    (129, 25, 31, 10, 10, 8, 'float32'),     # injection plane at the interior's first plane
    (37, 141, 25, 20, 10, 8, 'float32'),     # tall in y, odd sizes
    (45, 41, 75, 48, 8, 6, 'float32'),       # z ranges cut into several chunks
    (165, 37, 33, 21, 8, 6, 'float64'),
]
PATHS = [
    ('split', dict(kernel=SPLIT)),
    ('fused_split_shell', dict(kernel=FUSED, tile=(32, 4), shell=_native.SHELL_SPLIT)),
    ('fused_march_shell', dict(kernel=FUSED, tile=(32, 8), shell=_native.SHELL_MARCH)),
    ('fused_zchunk_3', dict(kernel=FUSED, tile=(32, 4), zchunk=3, shell=_native.SHELL_MARCH)),
    ('fused_column', dict(kernel=FUSED, tile=(32, 4), slab=2, shell=_native.SHELL_SPLIT)),
    ('fused_column_zchunk_3', dict(kernel=FUSED, tile=(32, 4), zchunk=3, slab=2, shell=_native.SHELL_SPLIT)),
]


def problem(case, seed):
    nx, ny, nz, tfsf, nt, ntp, dtype = case
    pc = make_params(nx, ny, nz, tfsf, nt, ntp, dtype=dtype)
    _, _, ca, cb, inc = random_problem(pc, seed)
    orc = oracle_for(pc)
    orc.run(ca, cb, inc, nt)
    return pc, ca, cb, inc, orc


def same(orc, sim):
    ok = all(bits_equal(sim.get_field(c), getattr(orc, c)) for c in _native.FIELD_NAMES)
    return ok and all(bits_equal(sim.get_phasor(k), orc.ph[n]) for k, n in enumerate(_native.PHASOR_NAMES))


def main():
    out = {'library': _native.LIB_NAME, 'checked': _native.bounds_check_enabled(), 'runs': []}
    problems = [problem(c, 900 + k) for k, c in enumerate(GRIDS)]
    for case, (pc, ca, cb, inc, orc) in zip(GRIDS, problems):
        for name, kw in PATHS:
            sim = native_for(pc, **kw)
            rec = {'grid': list(case[:4]), 'dtype': case[6], 'path': name}
            try:
                sim.set_materials(ca, cb)
                sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
                sim.run(case[4])
                sim.synchronize()
                rec['bit_exact'] = same(orc, sim)
                rec['error'] = None
            except _native.FdtdError as e:
                rec['bit_exact'] = False
                rec['error'] = f'{e.code}: {e}'
            sim.close()
            out['runs'].append(rec)
    # every float32 grid at once through the batch tile queue
    members = [(p, case) for p, case in zip(problems, GRIDS) if case[6] == 'float32']
    sims = []
    for (pc, ca, cb, inc, _), case in members:
        sim = native_for(pc)
        sim.set_materials(ca, cb)
        sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
        sims.append(sim)
    nt = min(case[4] for _, case in members)
    rec = {'path': 'batch_queue', 'members': len(sims)}
    try:
        batch = _native.Batch(sims, graph_chunk=4, mode=_native.BATCH_QUEUE)
        batch.run(nt)
        batch.synchronize()
        batch.close()
        for s in sims:
            s.synchronize()
        rec['error'] = None
        rec['steps'] = nt
    except _native.FdtdError as e:
        rec['error'] = f'{e.code}: {e}'
    for s in sims:
        s.close()
    out['runs'].append(rec)
    print(json.dumps(out))


if __name__ == '__main__':
    main()
