"""Kernel and tile selection for a geometry.

``choose`` returns the step kernel and fused-tile shape to use. Without a
measured entry it falls back to the built-in default; the autotuner in
``autotune`` measures candidates on the device and persists the winner.
"""
from . import _native


DEFAULT_TILE = (32, 4)


def choose(geom, kernel=None, tile=None):
    k = _native.FDTD_KERNEL_FUSED if kernel is None else int(kernel)
    tx, ty = tile if tile is not None else DEFAULT_TILE
    return {'kernel': k, 'tile_x': int(tx), 'tile_y': int(ty)}
