"""ctypes front end of the C oracle (oracle/fdtd_oracle.c) -- TEST
INFRASTRUCTURE AND CPU BASELINE ONLY.

``COracleSim`` is an ``OracleSim`` whose ``step`` runs the C restatement
with POSIX threads on the same numpy arrays; results are bit-identical to
the numpy oracle (tests/test_oracle_c.py). Build with ``make -C oracle``.
"""
import ctypes
import os

import numpy as np

import fdtd_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_build', 'libfdtd_oracle.so')

_P = ctypes.c_void_p


class _State(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int), ('ny', ctypes.c_int), ('nz', ctypes.c_int),
                ('npml', ctypes.c_int), ('tfsf_z', ctypes.c_int), ('t', ctypes.c_int),
                ('nt_inc', ctypes.c_int), ('dtype', ctypes.c_int), ('nthreads', ctypes.c_int),
                ('db', ctypes.c_double), ('dtm0', ctypes.c_double), ('dte0dx', ctypes.c_double),
                ('dx', ctypes.c_double),
                ('ex', _P), ('ey', _P), ('ez', _P), ('hx', _P), ('hy', _P), ('hz', _P),
                ('ca', _P), ('cb', _P),
                ('psi', _P * 24), ('prof', _P * 8), ('inc', _P * 4), ('ph', _P * 24),
                ('ce', ctypes.c_double), ('se', ctypes.c_double), ('ch', ctypes.c_double),
                ('sh', ctypes.c_double)]


_lib = None


def available():
    return os.path.isfile(LIB_PATH)


def _load():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f'{LIB_PATH} missing: run make -C oracle')
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_step.argtypes = [ctypes.POINTER(_State)]
        _lib.oracle_step.restype = ctypes.c_int
    return _lib


# (face, side, slot) -> numpy auxiliary name
_PSI = [('z', ('d', 'u'), ('Exz', 'Eyz', 'Hxz', 'Hyz')),
        ('x', ('l', 'r'), ('Eyx', 'Ezx', 'Hyx', 'Hzx')),
        ('y', ('f', 'b'), ('Exy', 'Ezy', 'Hxy', 'Hzy'))]
_PROF = ('be_d', 'bh_d', 'ce_d', 'ch_d', 'be_u', 'bh_u', 'ce_u', 'ch_u')


class COracleSim(O.OracleSim):
    """OracleSim stepped by the C restatement on ``nthreads`` threads."""

    def __init__(self, *args, nthreads=None, **kw):
        super().__init__(*args, **kw)
        self.nthreads = int(nthreads or os.cpu_count() or 1)
        _load()

    def step(self, ca, cb, inc):
        ca = np.ascontiguousarray(ca, dtype=self.dtype)
        cb = np.ascontiguousarray(cb, dtype=self.dtype)
        st = _State()
        st.nx, st.ny, st.nz, st.npml, st.tfsf_z = self.nx, self.ny, self.nz, self.npml, self.tfsf_z
        st.t = self.t
        ntp = inc['ex'].shape[0] if inc is not None else 0
        st.nt_inc = ntp
        st.dtype = 0 if self.dtype == np.float32 else 1
        st.nthreads = self.nthreads
        st.db, st.dtm0, st.dte0dx, st.dx = (float(self.Db), float(self.dtm0), float(self.dte0dx),
                                            float(self.dxf))
        for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
            setattr(st, c, getattr(self, c).ctypes.data)
        st.ca, st.cb = ca.ctypes.data, cb.ctypes.data
        k = 0
        for _, sides, slots in _PSI:
            for side in sides:
                for name in slots:
                    st.psi[k] = self.psi[name + side].ctypes.data
                    k += 1
        profs = [np.ascontiguousarray(self.p[n], dtype=self.dtype) for n in _PROF]
        for i, a in enumerate(profs):
            st.prof[i] = a.ctypes.data
        incs = []
        if inc is not None:
            for i, c in enumerate(('ex', 'ey', 'hx', 'hy')):
                a = np.ascontiguousarray(inc[c], dtype=self.dtype)
                incs.append(a)
                st.inc[i] = a.ctypes.data
        for i, name in enumerate(O.PHASOR_NAMES):
            st.ph[i] = self.ph[name].ctypes.data
        st.ce, st.se, st.ch, st.sh = O.phase_factors(self.omega, self.t, self.dt)
        if _load().oracle_step(ctypes.byref(st)) != 0:
            raise RuntimeError('oracle_step failed')
        self.t += 1
