"""FDTD time-stepping throughput on B200 (Mcell-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload plain_16x16|plain_8x8] [--kernel auto|split|fused]

One step is one Yee time step (H + CPML + injection + E + CPML + injection +
six phasor planes) of the whole grid. The default workload is the full-size
plain solve: 16x16 wavelengths, 3 wavelengths of material, cell 0.021 wl
(203 x 761 x 761 cells, 5.4 GHz, VV), float32, with a seeded synthetic
snowpack-over-rough-soil material and seeded synthetic incident planes.

``value`` is device time of exactly K steps with all inputs resident in HBM
(CUDA events on the launching stream, max over ranks). ``e2e`` is the same
metric through the C-ABI with host buffers: Ca/Cb upload, per-step incident
planes from pinned host memory, K steps, and the 24 phasor planes read back.
With N GPUs every rank runs its own replica (the reference farms whole
material models to workers; nothing is exchanged inside a model).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, 'sar-pixel-simulator_b200'))

BYTES_PER_CELL = {'float32': 56, 'float64': 112}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='plain_16x16',
                    choices=['plain_16x16', 'plain_8x8', 'batch64', 'adjoint_4x4', 'incident_16x16'])
    ap.add_argument('--fd-cells', type=int, default=32, help='adjoint_4x4: cells checked by FD')
    ap.add_argument('--profile-region', action='store_true',
                    help='adjoint_4x4: run one extra gradient between cudaProfilerStart/Stop')
    ap.add_argument('--models', type=int, default=64, help='batch64: number of models')
    ap.add_argument('--kernel', default='auto', choices=['auto', 'split', 'fused'])
    ap.add_argument('--tile-y', type=int, default=None, help='fused kernel rows per tile')
    ap.add_argument('--shell', default=None, choices=['march', 'split'],
                    help='fused kernel: shell marched or swept by the split passes')
    ap.add_argument('--zchunk', type=int, default=0, help='fused kernel z planes per block (0: auto)')
    ap.add_argument('--slab', type=int, default=None, choices=[0, 1, 2],
                    help='fused kernel: march the CPML z slabs (1), the whole z extent of the '
                         "interior's x-y box (2), or sweep the slabs with the shell (0)")
    ap.add_argument('--dtype', default='float32', choices=['float32', 'float64'])
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--cpu-steps', type=int, default=4)
    ap.add_argument('--no-extras', action='store_true',
                    help='plain_16x16 at N=1: skip the batch64, adjoint_4x4 and fp64_error records')
    return ap.parse_args()


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def build_workload(name, dtype, nsteps_inc, seed=2024, with_model=False):
    """(params, Ca, Cb, incident planes) of a plain-solve workload, and the
    material model (eps_r, sigma of the material planes) with with_model.
    Host modules only: the device library is not loaded here."""
    from fdtdsarsim_b200 import synthetic
    from fdtdsarsim_b200.materials import compute_material_arrays
    pc = synthetic.config_params(name, dtype)
    g = pc.geom_params
    rng = np.random.default_rng(seed)
    if name == 'plain_16x16':
        model = synthetic.snowpack_over_rough_soil(pc, rng)
    else:
        model = synthetic.rough_lognormal_soil(pc, rng)
    ca, cb = compute_material_arrays(pc, model)
    # The timed window covers steps t < size_t_inc of a full solve, so every
    # timed step injects, as the first 1372 steps of the real solve do. Only
    # the planes of the steps that run are synthesised (a tapered plane wave
    # with the geometry's frequency, polarisation and angle).
    n = min(g.size_t_inc, nsteps_inc)
    inc = synthetic.plane_wave_incident(pc, n, dtype)
    g.size_t_inc = n
    if with_model:
        return pc, ca, cb, inc, model
    return pc, ca, cb, inc


def workload_desc(pc, name):
    g = pc.geom_params
    return {
        'workload': f'{name}: plain solve {g.size_z}x{g.size_y}x{g.size_x} cells '
                    f'(nz x ny x nx), cell {g.cell_size:.6g} m, '
                    f'{pc.inc_beam_params.polarization}, theta 20 deg, 5.4 GHz',
        'grid': [g.size_z, g.size_y, g.size_x],
        'cells': g.size_z * g.size_y * g.size_x,
        'size_t_full_solve': g.size_t,
        'npml': g.size_pml,
        'materials': 'synthetic seeded (snowpack of ice spheres over rough soil)'
        if name == 'plain_16x16' else 'synthetic seeded (rough lognormal soil)',
        'incident': 'tapered plane wave (geometry frequency, polarisation, angle), injected every timed step',
        'l2': 'inputs larger than L2 (fields alone %.2f GB, L2 126 MB)' % (
            6 * g.size_z * g.size_y * g.size_x
            * (4 if pc.processing_params.datatype == 'float32' else 8) / 1e9),
    }


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix='.csv')
            os.close(fd)
            self.fh = open(self.path, 'w')
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.device), f'--query-gpu={self.QUERY}',
                 '--format=csv,noheader,nounits', '-lms', '100'], stdout=self.fh,
                stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(',')]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace('.', '').isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == 'active'})
        return {'sm_mhz': statistics.median(sm) if sm else None,
                'sm_max_mhz': max(mx) if mx else None, 'reasons': reasons,
                'samples': len(rows)}


def measured_peak_hbm():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as fh:
            return float(json.load(fh)['hbm_gbs']), 'measured'
    except (OSError, KeyError, ValueError, TypeError):
        return 6650.0, 'fallback'


def committed_traffic(kernel_name, workload):
    """dram bytes per launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, 'profiles', 'traffic.json')
    try:
        with open(path) as fh:
            d = json.load(fh)
        return d.get(workload, {}).get(kernel_name)
    except (OSError, ValueError):
        return None


# ---------------------------------------------------------------------------
# CPU baseline (the oracle: CPU restatement of the reference's algorithm)
# ---------------------------------------------------------------------------
def cpu_baseline(pc, ca, cb, inc, steps, warmup=1):
    """The oracle (CPU restatement of the reference's step) on the host: the
    C restatement on every host core when it is built (make -C oracle), else
    the numpy oracle on one core. `steps` full-grid steps after `warmup`
    untimed ones (the first touches every array)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import fdtd_oracle as O
    from fdtdsarsim_b200.absorbers import cpml_profiles
    g = pc.geom_params
    args = (g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size, g.timestep,
            pc.inc_beam_params.frequency, pc.processing_params.datatype, cpml_profiles(pc))
    try:
        import fdtd_oracle_c as OC
        if not OC.available():
            subprocess.run(['make', '-C', os.path.join(ROOT, 'oracle')], check=True,
                           capture_output=True)
        cores = os.cpu_count() or 1
        sim = OC.COracleSim(*args, nthreads=cores)
        what = f'C oracle, {cores} threads'
    except Exception:   # no compiler on the host: the numpy oracle
        cores = 1
        sim = O.OracleSim(*args)
        what = 'numpy oracle, one thread'
    for _ in range(max(1, warmup)):
        sim.step(ca, cb, inc)  # untimed; the first touches every array
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step(ca, cb, inc)
    dt = time.perf_counter() - t0
    cells = g.size_x * g.size_y * g.size_z
    return {'value': cells * steps / dt / 1e6, 'unit': 'Mcell-updates/s', 'cores': cores,
            'kind': 'port',
            'sample': f'{steps} time steps of the full {g.size_z}x{g.size_y}x{g.size_x} grid '
                      f'({what}), after {max(1, warmup)} untimed'}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def init_replicas(backend='nccl', timeout_s=120):
    """(rank, world, local) of this process from the launcher's environment
    (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_ADDR/PORT); with more than one
    rank, a process group on ``backend`` with a short timeout, so that ranks
    waiting for a lost peer end with an error. Replicas only: the group
    carries barriers and the max-over-ranks timing, no data."""
    import datetime
    import torch
    import torch.distributed as dist
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        kw = {'device_id': torch.device('cuda', local)} if backend == 'nccl' else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return rank, world, local


def max_over_ranks(x, world, device):
    """The largest of every rank's value (the job's time is its slowest
    replica's)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units, steps, ms, world):
    """Whole-job Mcell-updates/s: every rank processed ``units`` cells for
    ``steps`` steps in at most ``ms`` milliseconds."""
    return world * units * steps / (ms / 1e3) / 1e6


def step_launches(choice):
    """Kernel launches of one step: split H pass, E pass, phasors; fused
    with the marched shell: interior march, shell march, phasors; fused with
    the split-pass shell: interior march (and z-slab march), shell H pass,
    shell E pass, phasors."""
    from fdtdsarsim_b200 import _native
    if choice['kernel'] == _native.FDTD_KERNEL_SPLIT:
        return 3
    if choice.get('shell', _native.SHELL_SPLIT) == _native.SHELL_MARCH:
        return 3
    return 4 + int(bool(choice.get('slab', 0)))


def shell_name(choice):
    from fdtdsarsim_b200 import _native
    if choice['kernel'] == _native.FDTD_KERNEL_SPLIT:
        return None
    return 'march' if choice.get('shell', _native.SHELL_SPLIT) == _native.SHELL_MARCH else 'split_passes'


def run_ours(a):
    import torch
    import torch.distributed as dist
    rank, world, local = init_replicas('nccl')
    torch.cuda.set_device(local)
    from fdtdsarsim_b200 import _native
    from fdtdsarsim_b200.absorbers import packed_profiles
    from fdtdsarsim_b200.gpu.main_sim import native_geometry
    from fdtdsarsim_b200 import tuning

    pc, ca, cb, inc, model = build_workload(a.workload, a.dtype, a.warmup + a.steps + 1, with_model=True)
    g = pc.geom_params
    cells = g.size_x * g.size_y * g.size_z
    geom = native_geometry(pc)
    kernel = {'auto': None, 'split': _native.FDTD_KERNEL_SPLIT,
              'fused': _native.FDTD_KERNEL_FUSED}[a.kernel]
    tuned = None
    if kernel is None and a.tile_y is None:
        # measure the candidates on this geometry (a few steps each)
        choice, tuned = tuning.autotune(geom, local, save=False)
    else:
        choice = tuning.choose(geom, kernel=kernel,
                               tile=None if a.tile_y is None else (32, a.tile_y))
        choice['zchunk'] = a.zchunk
        if a.shell is not None:
            choice['shell'] = _native.SHELL_MARCH if a.shell == 'march' else _native.SHELL_SPLIT
        if a.slab is not None:
            choice['slab'] = a.slab

    def new_sim():
        sim = _native.NativeSim(geom, local)
        sim.set_absorbers(packed_profiles(pc))
        tuning.apply(sim, choice)
        return sim

    sim = new_sim()
    # time on the stream the library launches on
    stream = torch.cuda.ExternalStream(sim.stream())
    sim.set_materials(ca, cb)
    sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up
    sim.run(a.warmup)
    sim.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    sim.run(a.steps)
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = t_start.elapsed_time(t_end)
    ms_max = max_over_ranks(ms, world, 'cuda')
    value = job_rate(cells, a.steps, ms_max, world)
    launches_per_step = step_launches(choice)
    gpu_launches = launches_per_step * a.steps + 1

    # live per-kernel timing for the roofline (separate pass, same state)
    sim.reset()
    sim.run(a.warmup)
    sim.synchronize()
    sim.clear_kernel_time()
    sim.set_option(_native.OPT_TIMING, 1)
    nprof = min(a.steps, 60)
    sim.run(nprof)
    step_ms, step_n = sim.kernel_time(_native.TIME_STEP)
    ph_ms, ph_n = sim.kernel_time(_native.TIME_PHASOR)
    sim.set_option(_native.OPT_TIMING, 0)
    kname = 'fused_step' if choice['kernel'] == _native.FDTD_KERNEL_FUSED else 'split_h_e'
    avg_ms = step_ms / max(step_n, 1)
    alg_bytes = cells * BYTES_PER_CELL[a.dtype]
    peak, peak_kind = measured_peak_hbm()
    achieved = alg_bytes / (avg_ms / 1e3) / 1e9
    roofline = {'bound': 'hbm', 'achieved': round(achieved, 1), 'peak': peak, 'unit': 'GB/s',
                'frac': round(achieved / peak, 4), 'traffic': committed_traffic(kname, a.workload),
                'kernel': kname, 'peak_source': peak_kind,
                'algorithmic_bytes_per_launch': alg_bytes,
                'avg_launch_ms': round(avg_ms, 4),
                'phasor_kernel_avg_ms': round(ph_ms / max(ph_n, 1), 4),
                'step_share_of_device_time': round(step_ms / max(step_ms + ph_ms, 1e-9), 4)}
    sim.close()
    del sim

    # end to end through the C-ABI with host buffers, as run_experiment
    # drives it (MainSimGpu.run_eps_sigma): the material block's eps_r and
    # sigma go up and the device makes Ca, Cb; the incident planes stream
    # from pinned memory beside the steps; the 24 phasor planes come back
    e2e = None
    if not a.no_e2e:
        pin = {}
        for k, v in inc.items():
            t = torch.from_numpy(v).pin_memory()
            pin[k] = t.numpy()
        dt = np.dtype(a.dtype)
        eps_p = torch.from_numpy(np.ascontiguousarray(model.relative_permittivity, dt)).pin_memory().numpy()
        sig_p = torch.from_numpy(np.ascontiguousarray(model.conductivity, dt)).pin_memory().numpy()
        sim2 = new_sim()
        ph_buf = torch.empty(2 * sim2.phasors_size(), dtype=torch.float32 if a.dtype == 'float32'
                             else torch.float64).pin_memory().numpy().view(sim2.cdtype)
        sim2.synchronize()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim2.set_materials_eps_sigma(eps_p, sig_p)          # returns when Ca/Cb are made
        t_mat = time.perf_counter()
        sim2.run_streamed(a.steps, pin['ex'], pin['ey'], pin['hx'], pin['hy'])
        sim2.synchronize()
        t_run = time.perf_counter()
        phs = sim2.get_phasors(ph_buf)
        t1 = time.perf_counter()
        el = max_over_ranks(t1 - t0, world, 'cuda')
        esz = np.dtype(a.dtype).itemsize
        # bytes copied: the material block once, then the incident planes of
        # the steps that ran (t < size_t_inc), four components each
        streamed = min(a.steps, g.size_t_inc)
        h2d = eps_p.nbytes + sig_p.nbytes + 4 * streamed * g.size_x * g.size_y * esz
        d2h = sum(p.nbytes for p in phs.values())
        e2e = {'value': round(world * cells * a.steps / el / 1e6, 1), 'unit': 'Mcell-updates/s',
               'h2d_bytes_per_step': int(h2d / a.steps), 'd2h_bytes_per_step': int(d2h / a.steps),
               'phases_ms': {'materials': round((t_mat - t0) * 1e3, 2),
                             'steps_with_incident_streaming': round((t_run - t_mat) * 1e3, 2),
                             'phasor_readback': round((t1 - t_run) * 1e3, 2)},
               'includes': f'eps_r/sigma upload of the {eps_p.shape[0]}-plane material block (Ca/Cb '
                           f'made on the device, as run_experiment does), incident planes of '
                           f'{streamed} steps from pinned host memory beside the stepping, '
                           f'{a.steps} steps, 24 phasor planes read back into pinned memory; '
                           'wall clock'}
        sim2.close()
        pin = eps_p = sig_p = ph_buf = phs = None   # page-locked buffers

    base = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        base = cpu_baseline(pc, ca, cb, inc, a.cpu_steps)

    # the batched, adjoint and float64 claims, measured in the same run
    # (after the timed region; each with its own clock record)
    extras = {}
    if rank == 0 and world == 1 and a.workload == 'plain_16x16' and not a.no_extras:
        del ca, cb, inc, model
        for key, fn in (('batch64', lambda: batch_record(a, 64, a.steps, a.warmup)),
                        ('adjoint_4x4', lambda: adjoint_record(a, 32)),
                        ('fp64_error', lambda: fp64_record('plain_16x16'))):
            t0 = time.perf_counter()
            try:
                extras[key] = fn()
            except Exception as ex:   # recorded in the line, the headline stands
                extras[key] = {'error': f'{type(ex).__name__}: {ex}'}
            extras[key]['wall_s'] = round(time.perf_counter() - t0, 1)

    if rank == 0:
        line = {
            'metric': 'Mcell-updates/s', 'value': round(value, 1), 'unit': 'Mcell-updates/s',
            'n_gpus': world, 'steps': a.steps, 'warmup': a.warmup,
            'ms_per_step': round(ms_max / a.steps, 4), 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f32' if a.dtype == 'float32' else 'f64',
            'data': 'synthetic (seeded materials of the named shapes, tapered plane-wave incident planes)',
            'config': dict(workload_desc(pc, a.workload),
                           parallelism=f'replicas x{world}' if world > 1 else 'single GPU',
                           kernel=kname, tile=[choice['tile_x'], choice['tile_y']]
                           if choice['kernel'] == _native.FDTD_KERNEL_FUSED else None,
                           zchunk=choice.get('zchunk', 0), z_slabs_fused=int(choice.get('slab', 0)),
                           shell=shell_name(choice),
                           autotuned=None if tuned is None else
                           [{'ms': t, 'kernel': 'fused' if c['kernel'] else 'split',
                             'tile_y': c['tile_y'], 'zchunk': c['zchunk'], 'slab': c.get('slab', 0),
                             'shell': shell_name(c)}
                            for t, c in tuned]),
            'roofline': roofline, 'cpu_baseline': base, 'e2e': e2e,
            'gpu_launches': gpu_launches, 'clocks': clk,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# reference arm: the reference's CPU algorithm (oracle port) on host cores
# ---------------------------------------------------------------------------
def run_reference(a):
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    if rank != 0:
        return
    pc, ca, cb, inc = build_workload(a.workload, a.dtype, a.warmup + a.steps + 2)
    g = pc.geom_params
    cells = g.size_x * g.size_y * g.size_z
    steps = max(1, min(a.steps, a.cpu_steps))
    warm = max(1, min(a.warmup, 3))   # a bounded sample: at most 3 untimed steps
    base = cpu_baseline(pc, ca, cb, inc, steps, warm)
    line = {
        'impl': 'reference', 'metric': 'Mcell-updates/s', 'value': round(base['value'], 2),
        'unit': 'Mcell-updates/s', 'n_gpus': world, 'steps': steps, 'warmup': warm,
        'ms_per_step': round(cells / (base['value'] * 1e6) * 1e3, 2), 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32' if a.dtype == 'float32' else 'f64',
        'data': 'synthetic (seeded materials of the named shapes, tapered plane-wave incident planes)',
        'config': workload_desc(pc, a.workload),
        'cpu_baseline': base,
        'e2e': {'value': round(base['value'], 2), 'unit': 'Mcell-updates/s',
                'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# batched sweep: 64 uneven vegetation models, batched vs one after another
# ---------------------------------------------------------------------------
def batch_models(n, nsteps_inc, seed=4040, dtype='float32'):
    """n seeded models of the batched configuration: x-y uniform in 2..8
    wavelengths, depth 0.5..2 wavelengths, cell 0.03 wavelength, HH and VV
    alternating, dielectric cylinders over flat soil. The material fraction
    grows with the depth (0.4 at 0.5 wl, 0.7 from 1.25 wl) so that the
    injection plane stays below the upper phasor plane."""
    from fdtdsarsim_b200 import synthetic
    from fdtdsarsim_b200.materials import compute_material_arrays
    from fdtdsarsim_b200.parameters import set_geom_params
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        sx, sy = rng.uniform(2.0, 8.0, size=2)
        depth = rng.uniform(0.5, 2.0)
        mf = float(min(0.7, 0.4 + 0.4 * (depth - 0.5)))
        pol = 'HH' if k % 2 == 0 else 'VV'
        pc = synthetic.base_params(dtype, pol=pol, mf=mf, illum=sx)
        set_geom_params(pc, sx, sy, depth, pc.geom_params.simulation_duration, 0.03, 'wavelength')
        g = pc.geom_params
        model = synthetic.vegetation_model(pc, rng, name=f'veg{k:02d}')
        ca, cb = compute_material_arrays(pc, model)
        n = min(g.size_t_inc, nsteps_inc)
        inc = synthetic.plane_wave_incident(pc, n, dtype)
        g.size_t_inc = n
        out.append((pc, ca, cb, inc))
    return out


def batch_record(a, n_models, steps, warmup, check_members=(0, 21, 42)):
    """batch64: n_models uneven models advanced together (both batch modes,
    the faster is the result) and one after another (each model's own time
    loop on one stream). Members of the batched run are compared bit for
    bit with the same models' sequential solves."""
    import torch
    torch.cuda.set_device(0)
    from fdtdsarsim_b200 import _native, tuning
    from fdtdsarsim_b200.absorbers import packed_profiles
    from fdtdsarsim_b200.gpu.main_sim import native_geometry

    models = batch_models(n_models, warmup + steps + 1, dtype=a.dtype)
    cells = [pc.geom_params.size_x * pc.geom_params.size_y * pc.geom_params.size_z
             for pc, _, _, _ in models]
    total = int(sum(cells))
    sims, choices = [], []
    for pc, ca, cb, inc in models:
        geom = native_geometry(pc)
        sim = _native.NativeSim(geom, 0)
        sim.set_absorbers(packed_profiles(pc))
        choice = tuning.choose(geom)
        choices.append(choice)
        tuning.apply(sim, choice)
        sim.set_materials(ca, cb)
        sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
        sims.append(sim)
    check_members = [k for k in check_members if k < len(sims)]

    def timed(stream, fn):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def snapshot():
        return {k: {c: sims[k].get_field(c) for c in ('ex', 'hz')} for k in check_members}

    # batched, two modes: (split) every member each step, one launch per
    # pass, graph chunks; (streams) every member's own step path on its own
    # stream, side by side. The faster is the batched result.
    batch = _native.Batch(sims)
    bstream = torch.cuda.ExternalStream(batch.stream())
    batch.run(warmup)
    batch.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    ms_split = timed(bstream, lambda: batch.run(steps))
    snap_split = snapshot()
    for s in sims:
        s.reset()
    batch.set_streams(True)
    batch.run(warmup)
    batch.synchronize()
    ms_streams = timed(bstream, lambda: batch.run(steps))
    snap_streams = snapshot()
    for s in sims:
        s.reset()
    batch.set_mode(_native.BATCH_QUEUE)
    batch.run(warmup)
    batch.synchronize()
    ms_queue = timed(bstream, lambda: batch.run(steps))
    snap_queue = snapshot()
    batch.close()
    times = {'split': ms_split, 'streams': ms_streams, 'queue': ms_queue}
    mode = min(times, key=times.get)
    ms_b = times[mode]

    # one after another: each model's own time loop (its default kernel), on
    # one stream so the solves do not overlap
    for s in sims:
        s.reset()
    seq = torch.cuda.Stream()
    for s in sims:
        s.set_stream(seq.cuda_stream)
        s.run(warmup)
    ms_s = timed(seq, lambda: [s.run(steps) for s in sims])
    clk = clocks.stop()
    snap_seq = snapshot()
    same = all(np.array_equal(snap[k][c].view(np.uint8), snap_seq[k][c].view(np.uint8))
               for snap in (snap_split, snap_streams, snap_queue) for k in check_members
               for c in ('ex', 'hz'))
    for s in sims:
        s.close()

    value = total * steps / (ms_b / 1e3) / 1e6
    seq_value = total * steps / (ms_s / 1e3) / 1e6
    peak, peak_kind = measured_peak_hbm()
    achieved = total * BYTES_PER_CELL[a.dtype] * steps / (ms_b / 1e3) / 1e9
    nx = [pc.geom_params.size_x for pc, _, _, _ in models]
    nz = [pc.geom_params.size_z for pc, _, _, _ in models]
    return {
        'metric': 'Mcell-updates/s', 'value': round(value, 1), 'unit': 'Mcell-updates/s',
        'n_gpus': 1, 'steps': steps, 'warmup': warmup, 'ms_per_step': round(ms_b / steps, 4),
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32' if a.dtype == 'float32' else 'f64',
        'data': 'synthetic (seeded vegetation models, tapered plane-wave incident planes)',
        'config': {'workload': f'batch{n_models}: {n_models} vegetation models, x-y 2-8 wl, depth '
                               f'0.5-2 wl, cell 0.03 wl, HH/VV, 5.4 GHz',
                   'models': n_models, 'cells_total': total,
                   'nx_range': [int(min(nx)), int(max(nx))], 'nz_range': [int(min(nz)), int(max(nz))],
                   'l2': 'inputs larger than L2 (fields of all models)',
                   'batched': {'streams': 'every model on its own stream, its default kernel, side by side',
                               'split': 'split step of every model per launch, 64-step graph chunks',
                               'queue': "every model's fused step: one persistent launch walking a tile "
                                        'queue over all interior z-march tiles, one launch per split pass '
                                        'over all shells, one phasor launch; 64-step graph chunks'}[mode],
                   'modes_ms_per_step': {k: round(v / steps, 4) for k, v in times.items()}},
        'sequential': {'value': round(seq_value, 1), 'ms_per_step': round(ms_s / steps, 4),
                       'kernel': 'each model alone, its default kernel, one shared stream'},
        'speedup_vs_sequential': round(ms_s / ms_b, 3),
        'members_equal_sequential': {'members': check_members, 'fields': ['ex', 'hz'],
                                     'modes': ['split', 'streams', 'queue'], 'bit_exact': bool(same)},
        'roofline': {'bound': 'hbm', 'achieved': round(achieved, 1), 'peak': peak, 'unit': 'GB/s',
                     'frac': round(achieved / peak, 4), 'traffic': None, 'peak_source': peak_kind,
                     'kernel': {'streams': 'fused_step (member streams)', 'split': 'batch_split_step',
                                'queue': 'batch_queue'}[mode]},
        'cpu_baseline': None, 'e2e': None,
        'gpu_launches': {'streams': sum(step_launches(c) for c in choices) * steps,
                         'split': 3 * steps + 1,
                         'queue': 2 * steps + 1}[mode],
        'clocks': clk,
    }


def run_batch(a):
    print(json.dumps(batch_record(a, a.models, a.steps, a.warmup)))


# ---------------------------------------------------------------------------
# adjoint: cost of the gradient against one forward solve, and its accuracy
# ---------------------------------------------------------------------------
def adjoint_record(a, fd_cells):
    """adjoint_4x4: the gradient's cost against one forward solve and its
    accuracy against central differences of float64 solves and against the
    float64 adjoint."""
    import torch
    torch.cuda.set_device(0)
    from fdtdsarsim_b200 import synthetic
    from fdtdsarsim_b200.adjoint import BackscatterGradient

    def problem(dtype):
        pc = synthetic.config_params('adjoint_4x4', dtype)
        g = pc.geom_params
        rng = np.random.default_rng(5050)
        model = synthetic.uniform_rough_soil(pc, rng)
        return pc, model, synthetic.plane_wave_incident(pc, g.size_t_inc, dtype)

    pc, model, inc = problem('float32')
    g = pc.geom_params
    eps = model.relative_permittivity.astype(np.float64)
    sig = model.conductivity.astype(np.float64)
    from fdtdsarsim_b200 import tuning
    from fdtdsarsim_b200.gpu.main_sim import native_geometry
    tuned, _ = tuning.autotune(native_geometry(pc), 0)   # cached for the runners below
    run = BackscatterGradient(pc, inc, checkpoint_every=64)
    run.value(eps, sig)   # warm-up
    run.value_and_grad(eps, sig)
    clocks = ClockSampler(0)
    clocks.start()

    def wall(fn, reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            out = fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps, out
    t_fwd, J = wall(lambda: run.value(eps, sig), 3)
    t_adj, (J2, ge, gs) = wall(lambda: run.value_and_grad(eps, sig), 3)
    clk = clocks.stop()
    if a.profile_region:
        # one more gradient between cudaProfilerStart/Stop, for
        # `ncu --profile-from-start off` (no effect without a profiler)
        torch.cuda.profiler.start()
        run.value_and_grad(eps, sig)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()

    # float64 adjoint and central differences of float64 forward solves
    pc64, _, inc64 = problem('float64')
    inc64 = {k: v.astype(np.float64) for k, v in inc.items()}
    run64 = BackscatterGradient(pc64, inc64, checkpoint_every=64)
    J64, ge64, gs64 = run64.value_and_grad(eps, sig)
    rng = np.random.default_rng(7)
    mask = np.abs(ge64) > 1e-3 * np.abs(ge64).max()
    cells = np.argwhere(mask)
    picks = cells[rng.choice(len(cells), size=min(fd_cells, len(cells)), replace=False)]
    err32, err64 = [], []
    for z, y, x in picks:
        for base, g32, g64, is_eps in ((eps, ge, ge64, True), (sig, gs, gs64, False)):
            if base[z, y, x] == 0:
                continue   # sigma 0 (air): no relative step
            h = 1e-3 * base[z, y, x]
            b1, b2 = base.copy(), base.copy()
            b1[z, y, x] += h
            b2[z, y, x] -= h
            if is_eps:
                fd = (run64.value(b1, sig) - run64.value(b2, sig)) / (2 * h)
            else:
                fd = (run64.value(eps, b1) - run64.value(eps, b2)) / (2 * h)
            err32.append(abs(g32[z, y, x] - fd) / abs(fd))
            err64.append(abs(g64[z, y, x] - fd) / abs(fd))
    finite = bool(np.isfinite(ge).all() and np.isfinite(gs).all())
    norm_rel = float(np.linalg.norm(ge - ge64) / np.linalg.norm(ge64)) if finite else None
    cells_total = g.size_x * g.size_y * g.size_z
    line = {
        'metric': 'adjoint gradient time / forward solve time', 'value': round(t_adj / t_fwd, 3),
        'unit': 'ratio', 'higher_is_better': False, 'n_gpus': 1,
        'dtype': 'f32', 'data': 'synthetic (seeded rough soil, eps_r U(5,12), sigma U(0.005,0.05); '
                                'tapered plane-wave incident planes)',
        'config': {'workload': f'adjoint_4x4: {g.size_z}x{g.size_y}x{g.size_x} cells, nt {g.size_t}, '
                               f'HH backscatter power at theta -20 deg, checkpoint every 64',
                   'cells': cells_total, 'size_t': g.size_t},
        'forward_s': round(t_fwd, 4), 'gradient_s': round(t_adj, 4),
        'forward_mcell_updates_per_s': round(cells_total * g.size_t / t_fwd / 1e6, 1),
        'power': J, 'power_f64': J64,
        'fd_check': {'cells': int(len(picks)), 'params': ['eps_r', 'sigma'], 'step': '1e-3 relative',
                     'fd_solver': 'float64 forward solves',
                     'max_rel_err_f32_adjoint': float(max(err32)) if err32 else None,
                     'median_rel_err_f32_adjoint': float(np.median(err32)) if err32 else None,
                     'max_rel_err_f64_adjoint': float(max(err64)) if err64 else None},
        'f32_vs_f64_adjoint_rel_l2': norm_rel, 'gradients_finite': finite,
        'nonfinite_f32': int((~np.isfinite(ge)).sum() + (~np.isfinite(gs)).sum()),
        'kernel': tuned, 'clocks': clk,
    }
    run.close()
    run64.close()
    return line


def run_adjoint(a):
    print(json.dumps(adjoint_record(a, a.fd_cells)))


# ---------------------------------------------------------------------------
# incident beam: the full-size beam of the 16x16 wavelength geometry
# ---------------------------------------------------------------------------
def run_incident(a):
    import torch
    torch.cuda.set_device(0)
    from fdtdsarsim_b200 import synthetic
    from fdtdsarsim_b200.incident import IncidentSimGpu, create_pulse
    pc = synthetic.config_params('plain_16x16', a.dtype)
    g = pc.geom_params
    _, _, pulse_fft, pulse_freqs = create_pulse(pc)
    sim = IncidentSimGpu(pc, 0)
    gi = sim.params.geom_params

    def wall(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, out

    # one untimed pass (module loading, cuFFT set-up), then the timed pass
    sim.make_excitation(pulse_fft, pulse_freqs)
    sim.run()
    clocks = ClockSampler(0)
    clocks.start()
    t_exc, peak = wall(lambda: sim.make_excitation(pulse_fft, pulse_freqs))
    t_run, _ = wall(sim.run)
    clk = clocks.stop()
    t_read, planes = wall(sim.planes)
    sim.close()
    cells = gi.size_x * gi.size_y * gi.size_z
    steps = g.size_t_inc
    # CPU: the C oracle's steps on the same grid (all host cores), and the
    # numpy oracle's excitation on a sample of pulse bins, scaled to all bins
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    base = None
    if not a.no_cpu_baseline:
        ca = np.ones((gi.size_z, gi.size_y, gi.size_x), a.dtype)
        cb = np.full_like(ca, native_cb(sim.params))
        base = cpu_baseline(sim.params, ca, cb, None, a.cpu_steps)
        import incident_oracle as IO
        kx_sample = 4
        t0 = time.perf_counter()
        idx = np.linspace(1, len(pulse_fft) - 1, kx_sample).astype(int)
        kx, ky = IO.spatial_freqs(g.size_x, g.size_y, g.cell_size)
        for i in idx:
            k = (2 * np.pi * pulse_freqs[i]) / 299792458
            spec = IO.taper_k(k, kx, ky, pc.inc_beam_params.theta_angle, pc.inc_beam_params.phi_angle,
                              IO.gauss_radius(pc.inc_beam_params.illumination_width,
                                              pc.inc_beam_params.frequency),
                              pc.inc_beam_params.polarization)
            for c in spec:
                np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(c)))
        per_bin = (time.perf_counter() - t0) / kx_sample
        base['excitation_estimate_s'] = round(per_bin * len(pulse_fft), 1)
        base['excitation_sample'] = (f'taper and 2-D FFT of {kx_sample} of {len(pulse_fft)} pulse bins '
                                     f'(numpy oracle, one thread), scaled to all bins; time-axis '
                                     f'transforms not included')
    mcells = cells * steps / t_run / 1e6
    line = {
        'metric': 'Mcell-updates/s', 'value': round(mcells, 1), 'unit': 'Mcell-updates/s',
        'higher_is_better': True, 'n_gpus': 1, 'steps': steps, 'warmup': 1,
        'ms_per_step': round(t_run / steps * 1e3, 4), 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32' if a.dtype == 'float32' else 'f64',
        'data': 'synthetic (the geometry\'s own incident beam: tapered-wave excitation from its '
                'pulse, vacuum run)',
        'config': {'workload': f'incident_16x16: incident beam of the 16x16 wavelength geometry, '
                               f'grid {gi.size_z}x{gi.size_y}x{gi.size_x}, {steps} steps, source '
                               f'{g.size_t_pulse} steps, {pc.inc_beam_params.polarization}',
                   'grid': [gi.size_z, gi.size_y, gi.size_x], 'cells': cells,
                   'pulse_bins': len(pulse_fft)},
        'excitation_s': round(t_exc, 3), 'run_s': round(t_run, 3),
        'planes_to_host_s': round(t_read, 3),
        'planes_bytes': int(sum(v.nbytes for v in planes.values())),
        'excitation_peak_before_normalisation': peak,
        'cpu_baseline': base, 'clocks': clk,
        'gpu_launches': 4 * steps,
    }
    print(json.dumps(line))


def fp64_record(name='plain_16x16', seed=2024):
    """float32 against float64 for a full solve of a benchmark geometry on
    the device: the same seeded material model (eps_r, sigma rounded to each
    type, Ca/Cb made on the device), each precision's own incident beam made
    on the device (tapered-wave excitation and vacuum run, handed over device
    to device, as run_experiment does), all size_t steps; then the
    backscatter far field (theta = -theta_inc, r = 2 km) and its power."""
    import torch
    torch.cuda.set_device(0)
    from fdtdsarsim_b200 import _native, synthetic, tuning
    from fdtdsarsim_b200.absorbers import packed_profiles
    from fdtdsarsim_b200.gpu.main_sim import native_geometry
    from fdtdsarsim_b200.incident import IncidentSimGpu, create_pulse
    from fdtdsarsim_b200.near2far import FarFieldTransform
    from fdtdsarsim_b200.processresults import farfield_power
    pc = synthetic.config_params(name, 'float64')
    rng = np.random.default_rng(seed)
    model = (synthetic.snowpack_over_rough_soil(pc, rng) if name == 'plain_16x16'
             else synthetic.rough_lognormal_soil(pc, rng))
    out = {}
    clocks = ClockSampler(0)
    clocks.start()
    for dtype in ('float32', 'float64'):
        p = synthetic.config_params(name, dtype)
        g, b = p.geom_params, p.inc_beam_params
        t0 = time.perf_counter()
        inc = IncidentSimGpu(p, 0)
        _, _, pulse_fft, pulse_freqs = create_pulse(p)
        inc.make_excitation(pulse_fft, pulse_freqs)
        inc.run()
        geom = native_geometry(p)
        sim = _native.NativeSim(geom, 0)
        sim.set_absorbers(packed_profiles(p))
        tuning.apply(sim, tuning.choose(geom))
        sim.set_materials_eps_sigma(model.relative_permittivity.astype(dtype),
                                    model.conductivity.astype(dtype))
        sim.set_incident_from(inc.native)
        inc.close()
        sim.run(g.size_t)
        ph = sim.get_phasors()
        sim.synchronize()
        sim.close()
        el = time.perf_counter() - t0
        ff = FarFieldTransform(0)(ph, g.size_x - 2 * g.size_pml, g.size_y - 2 * g.size_pml,
                                  g.size_z - 2 * g.size_pml, g.cell_size, 2.0e3,
                                  np.array([-b.theta_angle]), np.array([b.phi_angle]), b.frequency)
        p_h, p_v = farfield_power(ff['E_theta'], ff['E_phi'], ff['H_theta'], ff['H_phi'])
        hh = str(b.polarization).upper() == 'HH'
        out[dtype] = {'e': complex(np.ravel(ff['E_phi'] if hh else ff['E_theta'])[0]),
                      'p': float(np.ravel(p_h if hh else p_v)[0]),
                      'u': {k: np.asarray(ph[k], np.complex128) for k in
                            ('ex_ph_u', 'ey_ph_u', 'hx_ph_u', 'hy_ph_u')},
                      'seconds': round(el, 2), 'steps': g.size_t}
    clk = clocks.stop()
    a32, a64 = out['float32'], out['float64']
    plane_err = max(float(np.max(np.abs(a32['u'][k] - a64['u'][k])) / max(np.max(np.abs(a64['u'][k])), 1e-300))
                    for k in a64['u'])
    g = pc.geom_params
    return {
        'workload': f'{name}: full solve {g.size_z}x{g.size_y}x{g.size_x}, {g.size_t} steps, '
                    f'{pc.inc_beam_params.polarization}, the geometry\'s own incident beam made on '
                    'the device in each precision',
        'backscatter_power': {'float32': a32['p'], 'float64': a64['p'],
                              'rel_err': abs(a32['p'] - a64['p']) / abs(a64['p'])},
        'backscatter_phasor_rel_err': abs(a32['e'] - a64['e']) / abs(a64['e']),
        'upper_phasor_planes_max_err_of_peak': plane_err,
        'seconds': {'float32': a32['seconds'], 'float64': a64['seconds']},
        'clocks': clk,
    }


def native_cb(params):
    """Cb of the vacuum in the simulation dtype (cpu/incident_sim.py:116)."""
    from fdtdsarsim_b200.gpu.main_sim import native_geometry
    return native_geometry(params).dte0dx


def main():
    a = parse()
    if a.impl == 'reference':
        run_reference(a)
    elif a.workload == 'batch64':
        run_batch(a)
    elif a.workload == 'adjoint_4x4':
        run_adjoint(a)
    elif a.workload == 'incident_16x16':
        run_incident(a)
    else:
        run_ours(a)


if __name__ == '__main__':
    main()
