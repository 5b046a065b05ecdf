"""The CPML terms divide by the constant cell size through a correctly
rounded reciprocal and one FMA correction (Markstein's method). On the
device it must give the IEEE quotient bit for bit: every float input is
checked, and 2^30 sampled doubles."""
import pytest
import scipy.constants

from fdtdsarsim_b200 import _native

pytestmark = pytest.mark.gpu

LAM = scipy.constants.c / 5.4e9


@pytest.mark.parametrize('cell_wl', [0.021, 0.03, 0.05])
def test_float_division_by_cell_size_is_exact_for_every_input(cell_wl):
    tested, bad = _native.check_cell_division('float32', LAM * cell_wl)
    assert tested == 2 ** 32
    assert bad == 0


@pytest.mark.parametrize('cell_size', [LAM * 0.021, 1e-3, 0.7])
def test_double_division_by_cell_size_matches_ieee(cell_size):
    tested, bad = _native.check_cell_division('float64', cell_size)
    assert tested == 2 ** 30
    assert bad == 0
