"""Time the reference's own CPU solver (``fdtdsarsim.cpu.main_sim.MainSimCpu``,
numba kernels on a thread pool) beside this repository's C restatement of
its step (``oracle/fdtd_oracle.c``) on the same host -- a measurement recipe,
not part of the product or the tests.

The reference is imported from its checkout (``/root/reference``) with the
in-memory h5py / matplotlib stand-ins of ``tests/golden/_refshims.py``. Both
solvers run the 8x8 wavelength geometry (101 x 381 x 381 cells) on the same
seeded coefficients and incident planes; per-step time is the difference
between a run of ``2 + STEPS`` steps and a run of 2 steps, after a first
run that compiles numba's kernels, on all host cores and on one.

    python oracle/reference_speed.py            # per-step rates, 8x8 wavelength geometry
    python oracle/reference_speed.py --full     # whole solves of the 2x2 (31x39x39) and
                                                # 4x4 (55x133x133) wavelength geometries
"""
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF = '/root/reference'
STEPS = 4

sys.path.insert(0, os.path.join(ROOT, 'tests', 'golden'))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, 'sar-pixel-simulator_b200'))


def reference_step_s(pc, ca, cb, inc, threads):
    import h5py
    from fdtdsarsim.cpu.main_sim import MainSimCpu
    from fdtdsarsim.parameters import inc_filename
    g = pc.geom_params
    times = {}
    for nt in (2, 2, 2 + STEPS):   # the first run compiles the numba kernels
        with tempfile.TemporaryDirectory() as proj:
            pc.processing_params.project_dir = proj
            pc.processing_params.threads_per_proc = threads
            g.size_t = nt
            with h5py.File(inc_filename(pc), 'w') as f:
                for c in ('ex', 'ey', 'hx', 'hy'):
                    f.create_dataset(c, data=inc[c])
                grp = f.create_group('phasors')
                for c in ('ex', 'ey', 'hx', 'hy'):
                    grp.create_dataset(f'{c}_inc_phasor',
                                       data=np.zeros((g.size_y - 20, g.size_x - 20), np.complex64))
            sim = MainSimCpu(pc, mpi=True)
            t0 = time.perf_counter()
            sim.run(ca, cb, f'case{nt}', {})
            times[nt] = time.perf_counter() - t0
    return (times[2 + STEPS] - times[2]) / STEPS


def oracle_step_s(pc, ca, cb, inc, threads):
    import fdtd_oracle_c as OC
    from fdtdsarsim_b200.absorbers import cpml_profiles
    g = pc.geom_params
    sim = OC.COracleSim(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size, g.timestep,
                        pc.inc_beam_params.frequency, 'float32', cpml_profiles(pc), nthreads=threads)
    sim.step(ca, cb, inc)
    t0 = time.perf_counter()
    for _ in range(STEPS):
        sim.step(ca, cb, inc)
    return (time.perf_counter() - t0) / STEPS


def main():
    import _refshims
    _refshims.install()
    sys.path.insert(0, REF)
    from fdtdsarsim_b200 import synthetic
    from fdtdsarsim_b200.materials import compute_material_arrays
    pc = synthetic.config_params('plain_8x8', 'float32')
    g = pc.geom_params
    rng = np.random.default_rng(2024)
    ca, cb = compute_material_arrays(pc, synthetic.rough_lognormal_soil(pc, rng))
    g.size_t_inc = 2 + STEPS
    inc = synthetic.plane_wave_incident(pc, g.size_t_inc, 'float32')
    # the reference's parameter object, with this geometry
    from fdtdsarsim.parameters import ParameterCollection
    rpc = ParameterCollection()
    for grp in ('geom_params', 'inc_beam_params', 'processing_params'):
        for k, v in vars(getattr(pc, grp)).items():
            setattr(getattr(rpc, grp), k, v)
    rpc.processing_params.processing_type = 'cpu'
    cells = g.size_x * g.size_y * g.size_z
    cores = os.cpu_count() or 1
    out = {'grid': [g.size_z, g.size_y, g.size_x], 'cells': cells, 'steps': STEPS, 'cores': cores}
    for threads in (cores, 1):
        r = reference_step_s(rpc, ca, cb, inc, threads)
        o = oracle_step_s(pc, ca, cb, inc, threads)
        out[f'threads{threads}'] = {
            'reference_mcell_s': round(cells / r / 1e6, 1), 'c_port_mcell_s': round(cells / o / 1e6, 1),
            'reference_s_per_step': round(r, 4), 'c_port_s_per_step': round(o, 4)}
    print(json.dumps(out))


def full_solves():
    """Wall time of whole reference solves (all size_t steps, all host cores,
    numba compiled beforehand) of the two small benchmark geometries."""
    import _refshims
    _refshims.install()
    sys.path.insert(0, REF)
    import h5py
    from fdtdsarsim.cpu.main_sim import MainSimCpu
    from fdtdsarsim.parameters import ParameterCollection, inc_filename
    from fdtdsarsim_b200 import synthetic
    from fdtdsarsim_b200.materials import compute_material_arrays
    out = {'cores': os.cpu_count()}
    for name in ('plain_2x2', 'adjoint_4x4'):
        pc = synthetic.config_params(name, 'float32')
        g = pc.geom_params
        rng = np.random.default_rng(7)
        ca, cb = compute_material_arrays(pc, synthetic.uniform_rough_soil(pc, rng))
        inc = synthetic.plane_wave_incident(pc, g.size_t_inc, 'float32')
        rpc = ParameterCollection()
        for grp in ('geom_params', 'inc_beam_params', 'processing_params'):
            for k, v in vars(getattr(pc, grp)).items():
                setattr(getattr(rpc, grp), k, v)
        rpc.processing_params.processing_type = 'cpu'
        rpc.processing_params.threads_per_proc = os.cpu_count()
        nt = g.size_t
        runs = {}
        for tag, steps in (('compile', 2), ('full', nt)):
            with tempfile.TemporaryDirectory() as proj:
                rpc.processing_params.project_dir = proj
                rpc.geom_params.size_t = steps
                with h5py.File(inc_filename(rpc), 'w') as f:
                    for c in ('ex', 'ey', 'hx', 'hy'):
                        f.create_dataset(c, data=inc[c])
                    grp = f.create_group('phasors')
                    for c in ('ex', 'ey', 'hx', 'hy'):
                        grp.create_dataset(f'{c}_inc_phasor', data=np.zeros(
                            (g.size_y - 20, g.size_x - 20), np.complex64))
                sim = MainSimCpu(rpc, mpi=True)
                t0 = time.perf_counter()
                sim.run(ca, cb, tag, {})
                runs[tag] = time.perf_counter() - t0
        out[name] = {'grid': [g.size_z, g.size_y, g.size_x], 'size_t': nt,
                     'reference_solve_s': round(runs['full'], 2)}
    print(json.dumps(out))


if __name__ == '__main__':
    if '--full' in sys.argv:
        full_solves()
    else:
        main()
