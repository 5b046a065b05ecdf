# fdtdsarsim/experiment.py, get_fdtd_simulator: one more branch, first
if proc_type == 'b200':
    from fdtdsarsim.b200 import MainSimB200
    return MainSimB200

# fdtdsarsim/b200.py
import ctypes, numpy as np, scipy.constants
from fdtdsarsim.absorbers import Absorbers

lib = ctypes.CDLL('libfdtd_b200.so')

class Geometry(ctypes.Structure):           # fdtd_geometry
    _fields_ = [(n, ctypes.c_int32) for n in
                ('nx', 'ny', 'nz', 'npml', 'tfsf_z', 'nt', 'nt_inc', 'dtype')] + \
               [(n, ctypes.c_double) for n in
                ('cell_size', 'timestep', 'frequency', 'db', 'dtm0', 'dte0dx')]

class MainSimB200:
    def __init__(self, params, mpi=False):
        self.params = params
        g, ft = params.geom_params, np.float32       # or float64
        dt, dx = g.timestep, g.cell_size
        geom = Geometry(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z,
                        g.size_t, g.size_t_inc, 0, dx, dt,
                        params.inc_beam_params.frequency,
                        ft(dt / (scipy.constants.mu_0 * dx)), ft(dt / scipy.constants.mu_0),
                        ft(dt / (scipy.constants.epsilon_0 * dx)))
        self.h = ctypes.c_void_p()
        assert lib.fdtd_create(ctypes.byref(geom), int(params.processing_params.gpu_num),
                               ctypes.byref(self.h)) == 0
        a = Absorbers(params)                          # profiles = column 0 of the tiles
        prof = np.concatenate([a.be_d[:, 0, 0], a.bh_d[:, 0, 0], a.ce_d[:, 0, 0],
                               a.ch_d[:, 0, 0], a.be_u[:, 0, 0], a.bh_u[:, 0, 0],
                               a.ce_u[:, 0, 0], a.ch_u[:, 0, 0]]).astype(ft)
        lib.fdtd_set_absorbers(self.h, prof.ctypes.data)

    def run(self, Ca, Cb, material_name, material_meta):
        Ca = np.ascontiguousarray(Ca, dtype=np.float32)   # the handle's element type
        Cb = np.ascontiguousarray(Cb, dtype=np.float32)
        lib.fdtd_reset(self.h)
        lib.fdtd_set_materials(self.h, Ca.ctypes.data, Cb.ctypes.data)
        # incident planes once per experiment: lib.fdtd_set_incident(self.h, ex, ey, hx, hy, nt_inc)
        lib.fdtd_run(self.h, self.params.geom_params.size_t)
        lib.fdtd_synchronize(self.h)
        # 24 phasor planes, reference order: lib.fdtd_get_phasor(self.h, k, out.ctypes.data)
