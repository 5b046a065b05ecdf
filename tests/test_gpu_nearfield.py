"""Near-field Poynting power on the device (fdtd_near_field_power) against
the host evaluation (processresults.near_field_power, bit for bit the
reference's processresults.py:128-257): every face power of a solved
simulation within 1e-6 relative of the largest, in float32 and float64,
for odd and even Simpson sample counts; and MainSimGpu with
device_postprocess writes the same powers that process_results keeps."""
import numpy as np
import pytest

from fdtdsarsim_b200 import _native
from fdtdsarsim_b200.processresults import near_field_power, near_field_power_device
from helpers import make_params, native_for, random_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('case', [
    # nx, ny, nz, tfsf_z, nt, ntp, nz_mat, dtype
    (41, 37, 45, 30, 40, 30, 14, 'float32'),    # nz_ph 25: material rows 14 (even), top 10 (even)
    (43, 39, 44, 30, 40, 30, 13, 'float32'),    # nz_ph 24: 13 (odd) and 10
    (33, 35, 41, 26, 30, 20, 12, 'float64'),
])
def test_device_near_field_power_equals_host(case):
    nx, ny, nz, tfsf, nt, ntp, nz_mat, dtype = case
    pc = make_params(nx, ny, nz, tfsf, nt, ntp, dtype=dtype, nz_mat=nz_mat)
    _, _, ca, cb, inc = random_problem(pc, 77)
    sim = native_for(pc, _native.FDTD_KERNEL_FUSED, (32, 4))
    try:
        sim.set_materials(ca, cb)
        sim.set_incident(inc['ex'], inc['ey'], inc['hx'], inc['hy'])
        sim.run(nt)
        sim.synchronize()
        ph = dict(sim.get_phasors())
        rng = np.random.default_rng(3)
        cd = np.complex64 if dtype == 'float32' else np.complex128
        for c in ('ex', 'ey', 'hx', 'hy'):
            ph[f'{c}_inc_phasor'] = (rng.standard_normal((ny - 20, nx - 20))
                                     + 1j * rng.standard_normal((ny - 20, nx - 20))).astype(cd)
        dx = pc.geom_params.cell_size
        host = near_field_power(ph, dx, nz_mat)
        dev = near_field_power_device(sim, ph, dx, nz_mat)
        scale = max(abs(v) for v in host.values())
        assert scale > 0
        for k, v in host.items():
            assert abs(dev[k] - v) <= 1e-6 * scale, (k, dev[k], v)
    finally:
        sim.close()
