"""Kernel, tile and z-march depth selection for a geometry.

``choose`` returns the step kernel, the fused tile shape and the z chunk
(planes a fused block marches) to use. It takes, in this order: the caller's
explicit choice, a measured entry from the tuning cache, the built-in
default. ``autotune`` measures the candidates on the device for one
geometry (a few steps each, with the library's per-kernel CUDA events) and
stores the winner in the cache, a JSON file keyed by device name, grid size
and element type (``$FDTDSARSIM_B200_TUNING``, else
``~/.cache/fdtdsarsim_b200/tuning.json``).
"""
import json
import os

import numpy as np

from . import _native

DEFAULT_TILE = (32, 4)

_MARCH, _SPLIT = _native.SHELL_MARCH, _native.SHELL_SPLIT

# (kernel, tile_y, zchunk, slab, shell); zchunk 0 lets the library pick;
# shell: the fused step's shell marched (_MARCH) or swept by the split
# passes (_SPLIT), then slab 1 marches the CPML z slabs, slab 2 the whole
# z extent of the interior's x-y box (the column march)
CANDIDATES = [
    (_native.FDTD_KERNEL_SPLIT, 4, 0, 0, _MARCH),
    (_native.FDTD_KERNEL_FUSED, 4, 0, 0, _MARCH),
    (_native.FDTD_KERNEL_FUSED, 4, 26, 0, _MARCH),
    (_native.FDTD_KERNEL_FUSED, 8, 0, 0, _MARCH),
    (_native.FDTD_KERNEL_FUSED, 4, 0, 0, _SPLIT),
    (_native.FDTD_KERNEL_FUSED, 8, 0, 0, _SPLIT),
    (_native.FDTD_KERNEL_FUSED, 4, 0, 1, _SPLIT),
    (_native.FDTD_KERNEL_FUSED, 4, 0, 2, _SPLIT),
]

# cache entries measured with another candidate set are measured again
_VERSION = 'v3'


def cache_path():
    return os.environ.get('FDTDSARSIM_B200_TUNING',
                          os.path.join(os.path.expanduser('~'), '.cache', 'fdtdsarsim_b200',
                                       'tuning.json'))


def _key(geom, device_name):
    dt = 'f32' if geom.dtype == _native.FDTD_F32 else 'f64'
    return f'{device_name}|{geom.nx}x{geom.ny}x{geom.nz}|npml{geom.npml}|{dt}|{_VERSION}'


def _device_name(device):
    try:
        return _native.device_name(device)
    except _native.FdtdError:   # no device here
        return f'device{device}'


def _load():
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def lookup(geom, device=0):
    return _load().get(_key(geom, _device_name(device)))


def choose(geom, kernel=None, tile=None, device=0, use_cache=True):
    """{'kernel', 'tile_x', 'tile_y', 'zchunk', 'slab', 'shell'} for a geometry."""
    if kernel is None and tile is None and use_cache:
        hit = lookup(geom, device)
        if hit:
            return {'kernel': int(hit['kernel']), 'tile_x': 32, 'tile_y': int(hit['tile_y']),
                    'zchunk': int(hit['zchunk']), 'slab': int(hit.get('slab', 0)),
                    'shell': int(hit.get('shell', _SPLIT))}
    k = _native.FDTD_KERNEL_FUSED if kernel is None else int(kernel)
    tx, ty = tile if tile is not None else DEFAULT_TILE
    return {'kernel': k, 'tile_x': int(tx), 'tile_y': int(ty), 'zchunk': 0, 'slab': 0, 'shell': _SPLIT}


def apply(sim, choice):
    """Set a choice on a NativeSim."""
    sim.set_option(_native.OPT_KERNEL, choice['kernel'])
    if choice['kernel'] == _native.FDTD_KERNEL_FUSED:
        sim.set_option(_native.OPT_TILE_X, choice['tile_x'])
        sim.set_option(_native.OPT_TILE_Y, choice['tile_y'])
        sim.set_option(_native.OPT_ZCHUNK, choice.get('zchunk', 0))
        sim.set_option(_native.OPT_FUSED_SLAB, choice.get('slab', 0))
        sim.set_option(_native.OPT_SHELL, choice.get('shell', _SPLIT))


def autotune(geom, device=0, steps=6, candidates=None, save=True):
    """Time every candidate on this geometry and return (choice, timings).

    The measurement uses vacuum coefficients, CPML profiles of ones and
    zeros and no incident beam: the step kernels' cost does not depend on the
    values (the one value-dependent branch, the IEEE division of tiny CPML
    terms, is taken by subnormal inputs only)."""
    g = _native.Geometry()
    for name, _ in _native.Geometry._fields_:
        setattr(g, name, getattr(geom, name))
    g.nt = steps + 4
    g.nt_inc = 0
    sim = _native.NativeSim(g, device)
    ft = np.float32 if g.dtype == _native.FDTD_F32 else np.float64
    prof = np.concatenate([np.ones(g.npml), np.ones(g.npml), np.zeros(g.npml), np.zeros(g.npml)] * 2)
    sim.set_absorbers(prof.astype(ft))
    ca = np.ones((g.nz, g.ny, g.nx), ft)
    cb = np.full((g.nz, g.ny, g.nx), g.dte0dx, ft)
    sim.set_materials(ca, cb)
    timings = []
    for cand in (candidates or CANDIDATES):
        kernel, ty, zc, slab = cand[:4]
        shell = cand[4] if len(cand) > 4 else _MARCH
        choice = {'kernel': kernel, 'tile_x': 32, 'tile_y': ty, 'zchunk': zc, 'slab': slab,
                  'shell': shell}
        try:
            apply(sim, choice)
            sim.reset()
            sim.run(2)
            sim.synchronize()
            sim.clear_kernel_time()
            sim.set_option(_native.OPT_TIMING, 1)
            sim.run(steps)
            ms, n = sim.kernel_time(_native.TIME_STEP)
            sim.set_option(_native.OPT_TIMING, 0)
        except _native.FdtdError:
            continue
        timings.append((ms / max(n, 1), choice))
    sim.close()
    best = min(timings, key=lambda t: t[0])[1]
    if save:
        path = cache_path()
        data = _load()
        data[_key(geom, _device_name(device))] = dict(best, step_ms=min(t[0] for t in timings))
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + '.tmp'
        with open(tmp, 'w') as fh:
            json.dump(data, fh, indent=1)
        os.replace(tmp, path)
    return best, [(round(ms, 5), c) for ms, c in timings]
