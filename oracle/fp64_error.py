"""Float32 error against a float64 run, per benchmark configuration -- a
measurement recipe on the oracle, not part of the product or the tests.

The device solver is bit-identical to the oracle in float32 and in float64
(tests/test_gpu_parity.py), so the C restatement of the step
(oracle/fdtd_oracle.c, all host cores) run here in both precisions gives
exactly the numbers the device gives. For each configuration: seeded
synthetic materials and tapered plane-wave incident planes made in float64
(the float32 run gets them rounded), a full solve of size_t steps in each
precision, then the backscatter far field (theta = -theta_inc, r = 2 km,
near2far.py:28-156 restated in oracle/fdtd_oracle.py) and its power
(processresults.py:260-271).

    python oracle/fp64_error.py plain_2x2 adjoint_4x4 plain_8x8
    python oracle/fp64_error.py plain_16x16        # about 25 min on 8 cores
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, 'sar-pixel-simulator_b200'))

import fdtd_oracle as O          # noqa: E402
import fdtd_oracle_c as OC       # noqa: E402
from fdtdsarsim_b200 import synthetic                           # noqa: E402
from fdtdsarsim_b200.absorbers import cpml_profiles             # noqa: E402
from fdtdsarsim_b200.materials import MaterialModel, compute_material_arrays  # noqa: E402

MODELS = {'plain_16x16': synthetic.snowpack_over_rough_soil,
          'adjoint_4x4': synthetic.uniform_rough_soil}


def solve(pc, model, inc):
    g = pc.geom_params
    dtype = pc.processing_params.datatype
    m = MaterialModel(model.relative_permittivity.astype(dtype),
                      model.conductivity.astype(dtype), g.cell_size)
    ca, cb = compute_material_arrays(pc, m)
    inc = {c: np.ascontiguousarray(v, dtype=dtype) for c, v in inc.items()}
    sim = OC.COracleSim(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size,
                        g.timestep, pc.inc_beam_params.frequency, dtype, cpml_profiles(pc))
    sim.run(ca, cb, inc, g.size_t)
    return sim.ph


def backscatter(pc, ph):
    g, b = pc.geom_params, pc.inc_beam_params
    ff = O.near2far(ph['ex_ph_u'], ph['ey_ph_u'], ph['hx_ph_u'], ph['hy_ph_u'],
                    g.size_x - 20, g.size_y - 20, g.size_z - 20, g.cell_size, 2.0e3,
                    [-b.theta_angle], [b.phi_angle], b.frequency)
    p_h, p_v = O.farfield_power(ff['E_theta'], ff['E_phi'], ff['H_theta'], ff['H_phi'])
    if b.polarization.upper() == 'HH':
        return complex(ff['E_phi']), float(p_h)
    return complex(ff['E_theta']), float(p_v)


def run(name):
    pc64 = synthetic.config_params(name, 'float64')
    pc32 = synthetic.config_params(name, 'float32')
    g = pc64.geom_params
    make = MODELS.get(name, synthetic.rough_lognormal_soil)
    model = make(pc64, np.random.default_rng(2024))
    inc = synthetic.plane_wave_incident(pc64, g.size_t_inc, 'float64')
    t0 = time.perf_counter()
    ph64 = solve(pc64, model, inc)
    ph32 = solve(pc32, model, inc)
    b64, p64 = backscatter(pc64, ph64)
    b32, p32 = backscatter(pc32, ph32)
    planes = {}
    for k in ('ex_ph_u', 'ey_ph_u', 'hx_ph_u', 'hy_ph_u'):
        ref = ph64[k]
        planes[k] = float(np.max(np.abs(ph32[k] - ref)) / np.max(np.abs(ref)))
    return {'config': name, 'grid': [g.size_z, g.size_y, g.size_x], 'size_t': g.size_t,
            'polarization': pc64.inc_beam_params.polarization,
            'backscatter_power_f64': p64, 'backscatter_power_rel_err': abs(p32 - p64) / abs(p64),
            'backscatter_phasor_rel_err': abs(b32 - b64) / abs(b64),
            'upper_plane_max_rel_err': max(planes.values()),
            'seconds': round(time.perf_counter() - t0, 1)}


if __name__ == '__main__':
    for cfg in sys.argv[1:] or ['plain_2x2', 'adjoint_4x4', 'plain_8x8']:
        print(json.dumps(run(cfg)), flush=True)
