"""The fused step's decomposition (fdtd_fused_plan_boxes, host logic, no
GPU): every cell in exactly one box; the z-marching boxes keep clear of the
x and y CPML faces and of the injection plane (and of the plane below each
z range, which a march recomputes); vector-aligned x starts."""
import numpy as np
import pytest

from fdtdsarsim_b200 import _native

GRIDS = [
    # nx, ny, nz, npml, tfsf_z
    (761, 761, 203, 10, 156), (27, 25, 23, 10, 14), (41, 37, 29, 10, 16), (27, 25, 23, 10, 20),
    (261, 45, 30, 10, 14), (150, 61, 37, 10, 20), (300, 70, 40, 10, 10), (173, 53, 40, 10, 28),
    (133, 133, 55, 10, 40), (39, 39, 31, 10, 14), (25, 25, 25, 2, 5), (67, 91, 43, 10, 30),
    (41, 37, 29, 10, 9), (41, 37, 29, 10, 18), (41, 37, 29, 10, 0), (27, 25, 23, 10, 12),
    (761, 761, 142, 10, -2),
]


@pytest.mark.parametrize('mode', ['shell', 'slab', 'march', 'column'])
@pytest.mark.parametrize('tile_y', [4, 8])
@pytest.mark.parametrize('grid', GRIDS)
def test_boxes_partition_the_grid(grid, tile_y, mode):
    nx, ny, nz, m, tfsf = grid
    slab = {'slab': 1, 'column': 2}.get(mode, 0)
    boxes = _native.fused_plan_boxes(nx, ny, nz, m, tfsf, tile_y, slab=slab, march=mode == 'march')
    # the march plan sends the whole shell to the general march, the others
    # to the split passes
    shell_kind = 3 if mode == 'march' else 2
    assert set(boxes[:, 0]) <= {0, 1, shell_kind}
    if mode not in ('slab', 'column'):
        assert 1 not in boxes[:, 0]
    if mode == 'column' and (boxes[:, 0] == 1).any():
        # the column march replaces the interior march and spans every plane
        assert 0 not in boxes[:, 0]
        assert [tuple(b[5:]) for b in boxes if b[0] == 1] == [(0, nz)]
    count = np.zeros((nz, ny, nx), np.int32)
    for kind, x0, x1, y0, y1, z0, z1 in boxes:
        assert x0 % 4 == 0
        count[z0:z1, y0:y1, x0:x1] += 1
        if kind in (0, 1):
            # no x / y face at the box or at the halo it recomputes
            assert x0 - 1 >= m - 1 and x1 <= nx - m and y0 - 1 >= m - 1 and y1 <= ny - m
            if mode != 'column':   # the column march injects; the others keep clear
                assert not (z0 - 1 <= tfsf < z1), (kind, z0, z1)
        if kind == 0:   # the interior: no z face either
            assert z0 - 1 >= m - 1 and z1 <= nz - m
    assert (count == 1).all()
    if nx - m >= 36:   # room for a 32-aligned interior start
        assert (boxes[:, 0] == (1 if mode == 'column' else 0)).any()
