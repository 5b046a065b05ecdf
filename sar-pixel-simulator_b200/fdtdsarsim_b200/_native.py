"""ctypes binding of libfdtd_b200.so (declared in include/fdtd_b200.h).

The library is the only compute path of this package: importing this module
fails loudly when it is missing, and every call that returns a non-zero
status raises :class:`FdtdError` with the library's message.
"""
import ctypes
import os

import numpy as np

# FDTDSARSIM_B200_LIBRARY=check selects the bounds-checked build
# (libfdtd_b200_check.so): every global access of the step kernels checked
# against the live allocations, violations reported as FDTD_ERR_BOUNDS
LIB_NAME = ('libfdtd_b200_check.so' if os.environ.get('FDTDSARSIM_B200_LIBRARY', '') == 'check'
            else 'libfdtd_b200.so')
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

FDTD_OK = 0
FDTD_ERR_INVALID = 1
FDTD_ERR_CUDA = 2
FDTD_ERR_STATE = 3
FDTD_ERR_NONFINITE = 4
FDTD_ERR_NOMEM = 5
FDTD_ERR_BOUNDS = 6

FDTD_F32 = 0
FDTD_F64 = 1

FDTD_KERNEL_SPLIT = 0
FDTD_KERNEL_FUSED = 1

FDTD_PHASOR_REFERENCE = 0
FDTD_PHASOR_KAHAN = 1

OPT_KERNEL = 1
OPT_PHASOR_MODE = 2
OPT_TILE_X = 3
OPT_TILE_Y = 4
OPT_GRAPH_CHUNK = 5
OPT_CHECK_EVERY = 6
OPT_TIMING = 7
OPT_ZCHUNK = 8
OPT_FUSED_SLAB = 9
OPT_BATCH_STREAMS = 10
OPT_SHELL = 11
SHELL_MARCH = 0
SHELL_SPLIT = 1
OPT_BATCH_MODE = 12
BATCH_SPLIT = 0
BATCH_STREAMS = 1
BATCH_QUEUE = 2

TIME_STEP = 0
TIME_PHASOR = 1

POLARIZATIONS = {'HH': 0, 'VV': 1, 'RHCP': 2, 'LHCP': 3}   # FDTD_POL_*

PHASOR_NAMES = (
    'ex_ph_d', 'ey_ph_d', 'hx_ph_d', 'hy_ph_d',
    'ex_ph_u', 'ey_ph_u', 'hx_ph_u', 'hy_ph_u',
    'ey_ph_l', 'ez_ph_l', 'hy_ph_l', 'hz_ph_l',
    'ey_ph_r', 'ez_ph_r', 'hy_ph_r', 'hz_ph_r',
    'ex_ph_f', 'ez_ph_f', 'hx_ph_f', 'hz_ph_f',
    'ex_ph_b', 'ez_ph_b', 'hx_ph_b', 'hz_ph_b',
)
FIELD_NAMES = ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')


class FdtdError(RuntimeError):
    """A libfdtd_b200 call failed; ``code`` is the FDTD_ERR_* status."""

    def __init__(self, code, msg):
        super().__init__(f'libfdtd_b200 error {code}: {msg}')
        self.code = code


class Geometry(ctypes.Structure):
    """Mirror of ``fdtd_geometry``."""
    _fields_ = [
        ('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('nz', ctypes.c_int32),
        ('npml', ctypes.c_int32), ('tfsf_z', ctypes.c_int32), ('nt', ctypes.c_int32),
        ('nt_inc', ctypes.c_int32), ('dtype', ctypes.c_int32),
        ('cell_size', ctypes.c_double), ('timestep', ctypes.c_double),
        ('frequency', ctypes.c_double), ('db', ctypes.c_double), ('dtm0', ctypes.c_double),
        ('dte0dx', ctypes.c_double),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double

# name -> argtypes; every function returns int
SIGNATURES = {
    'fdtd_last_error': [ctypes.c_char_p, _I],
    'fdtd_version': [],
    'fdtd_bounds_check_enabled': [],
    'fdtd_near_field_power': [_P, _P, _I, _P, _P],
    'fdtd_fill_layers': [_P, _I, _I, _P, _P, _P],
    'fdtd_paint_spheres': [_P, _I, _P, _D, _D],
    'fdtd_set_materials_staged': [_P],
    'fdtd_get_staged_materials': [_P, _I, _P, _P],
    'fdtd_device_count': [ctypes.POINTER(_I)],
    'fdtd_device_name': [_I, ctypes.c_char_p, _I],
    'fdtd_create': [ctypes.POINTER(Geometry), _I, ctypes.POINTER(_P)],
    'fdtd_destroy': [_P],
    'fdtd_set_option': [_P, _I, _I],
    'fdtd_get_option': [_P, _I, ctypes.POINTER(_I)],
    'fdtd_set_absorbers': [_P, _P],
    'fdtd_set_materials': [_P, _P, _P],
    'fdtd_set_materials_eps_sigma': [_P, _P, _P, _I],
    'fdtd_set_incident': [_P, _P, _P, _P, _P, _I],
    'fdtd_reset': [_P],
    'fdtd_run': [_P, _I],
    'fdtd_run_streamed': [_P, _I, _P, _P, _P, _P],
    'fdtd_synchronize': [_P],
    'fdtd_step_index': [_P, ctypes.POINTER(ctypes.c_int64)],
    'fdtd_get_stream': [_P, ctypes.POINTER(_P)],
    'fdtd_set_stream': [_P, _P],
    'fdtd_get_kernel_time': [_P, _I, ctypes.POINTER(_D), ctypes.POINTER(_I)],
    'fdtd_clear_kernel_time': [_P],
    'fdtd_get_phasor': [_P, _I, _P],
    'fdtd_get_phasors': [_P, _P],
    'fdtd_get_field': [_P, _I, _P],
    'fdtd_set_field': [_P, _I, _P],
    'fdtd_near2far': [_P, _P, _P, _P, _I, _I, _I, _I, _D, _D, _P, _I, _P, _I, _D, _I, _P],
    'fdtd_grad_forward': [_P, _I],
    'fdtd_grad_backward': [_P, _P, _P, _I, _P, _P],
    'fdtd_batch_create': [ctypes.POINTER(_P), _I, ctypes.POINTER(_P)],
    'fdtd_batch_destroy': [_P],
    'fdtd_batch_set_option': [_P, _I, _I],
    'fdtd_batch_run': [_P, _I],
    'fdtd_batch_synchronize': [_P],
    'fdtd_batch_get_stream': [_P, ctypes.POINTER(_P)],
    'fdtd_check_cell_division': [_I, _D, _I, ctypes.POINTER(ctypes.c_int64),
                                 ctypes.POINTER(ctypes.c_int64)],
    'fdtd_near2far_noalloc': [_P, _P, _P, _P, _I, _I, _I, _I, _D, _D, _P, _I, _P, _I, _D, _I, _P],
    'fdtd_fused_plan_boxes': [_I, _I, _I, _I, _I, _I, _I, _I, _P, _I, ctypes.POINTER(_I)],
    'fdtd_incident_create': [ctypes.POINTER(Geometry), _I, _I, ctypes.POINTER(_P)],
    'fdtd_incident_destroy': [_P],
    'fdtd_incident_set_option': [_P, _I, _I],
    'fdtd_incident_set_absorbers': [_P, _P],
    'fdtd_incident_make_excitation': [_P, _P, _P, _I, _D, _D, _I, _D, ctypes.POINTER(_D)],
    'fdtd_incident_set_excitation': [_P, _P, _P],
    'fdtd_incident_get_excitation': [_P, _P, _P],
    'fdtd_incident_run': [_P],
    'fdtd_incident_get_planes': [_P, _P, _P, _P, _P],
    'fdtd_incident_get_phasors': [_P, _P, _P, _P, _P],
    'fdtd_set_incident_from': [_P, _P],
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f'{LIB_PATH} is missing: build it with `python sar-pixel-simulator_b200/build.py'
            f'{" --bounds-check" if LIB_NAME.endswith("_check.so") else ""}` (there is no CPU fallback)')
    lib = ctypes.CDLL(LIB_PATH)
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = ctypes.c_int
    return lib


lib = _load()


def last_error():
    buf = ctypes.create_string_buffer(1024)
    lib.fdtd_last_error(buf, len(buf))
    return buf.value.decode(errors='replace')


def check(rc):
    if rc != FDTD_OK:
        raise FdtdError(rc, last_error())


def device_count():
    n = ctypes.c_int(0)
    check(lib.fdtd_device_count(ctypes.byref(n)))
    return n.value


def device_name(device=0):
    """The CUDA device's name (fdtd_device_name)."""
    buf = ctypes.create_string_buffer(256)
    check(lib.fdtd_device_name(int(device), buf, len(buf)))
    return buf.value.decode(errors='replace')


def ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def dtype_code(dtype):
    dt = np.dtype(dtype)
    if dt == np.float32:
        return FDTD_F32
    if dt == np.float64:
        return FDTD_F64
    raise ValueError('Invalid dtype specifier')


class NativeSim:
    """Owning wrapper of one ``fdtd_sim`` handle."""

    def __init__(self, geom: Geometry, device: int = 0):
        self.geom = geom
        self.dtype = np.float32 if geom.dtype == FDTD_F32 else np.float64
        self.cdtype = np.complex64 if geom.dtype == FDTD_F32 else np.complex128
        h = ctypes.c_void_p()
        check(lib.fdtd_create(ctypes.byref(geom), int(device), ctypes.byref(h)))
        self.h = h
        self.nx_ph = geom.nx - 2 * geom.npml
        self.ny_ph = geom.ny - 2 * geom.npml
        self.nz_ph = geom.nz - 2 * geom.npml

    def close(self):
        """Free the handle (FdtdError while it is a member of an open
        Batch; the handle then stays valid)."""
        if getattr(self, 'h', None) is not None and self.h.value:
            check(lib.fdtd_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _arr(self, a, shape=None):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        if shape is not None and a.shape != tuple(shape):
            raise ValueError(f'expected shape {tuple(shape)}, got {a.shape}')
        return a

    def set_option(self, opt, value):
        check(lib.fdtd_set_option(self.h, int(opt), int(value)))

    def get_option(self, opt):
        v = ctypes.c_int(0)
        check(lib.fdtd_get_option(self.h, int(opt), ctypes.byref(v)))
        return v.value

    def set_absorbers(self, packed):
        a = self._arr(packed, (8 * self.geom.npml,))
        check(lib.fdtd_set_absorbers(self.h, ptr(a)))

    def set_materials(self, ca, cb):
        g = self.geom
        shape = (g.nz, g.ny, g.nx)
        a, b = self._arr(ca, shape), self._arr(cb, shape)
        check(lib.fdtd_set_materials(self.h, ptr(a), ptr(b)))

    def set_materials_eps_sigma(self, eps_r, sigma):
        g = self.geom
        e, s = self._arr(eps_r), self._arr(sigma)
        if e.shape != s.shape or e.ndim != 3 or e.shape[1:] != (g.ny, g.nx):
            raise ValueError(f'eps/sigma must both be (nz_mat, {g.ny}, {g.nx})')
        check(lib.fdtd_set_materials_eps_sigma(self.h, ptr(e), ptr(s), int(e.shape[0])))

    def set_incident(self, ex, ey, hx, hy):
        g = self.geom
        shape = (g.nt_inc, g.ny, g.nx)
        arrs = [self._arr(c, shape) for c in (ex, ey, hx, hy)]
        check(lib.fdtd_set_incident(self.h, *[ptr(a) for a in arrs], int(g.nt_inc)))

    def reset(self):
        check(lib.fdtd_reset(self.h))

    def run(self, nsteps):
        check(lib.fdtd_run(self.h, int(nsteps)))

    def run_streamed(self, nsteps, ex, ey, hx, hy):
        g = self.geom
        shape = (g.nt_inc, g.ny, g.nx)
        arrs = [self._arr(c, shape) for c in (ex, ey, hx, hy)]
        check(lib.fdtd_run_streamed(self.h, int(nsteps), *[ptr(a) for a in arrs]))

    def synchronize(self):
        check(lib.fdtd_synchronize(self.h))

    def step_index(self):
        t = ctypes.c_int64(0)
        check(lib.fdtd_step_index(self.h, ctypes.byref(t)))
        return t.value

    def stream(self):
        s = ctypes.c_void_p()
        check(lib.fdtd_get_stream(self.h, ctypes.byref(s)))
        return s.value

    def set_stream(self, stream_handle):
        check(lib.fdtd_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)))

    def kernel_time(self, kind):
        ms = ctypes.c_double(0)
        n = ctypes.c_int(0)
        check(lib.fdtd_get_kernel_time(self.h, int(kind), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def clear_kernel_time(self):
        check(lib.fdtd_clear_kernel_time(self.h))

    def phasor_shape(self, k):
        if k < 8:
            return (self.ny_ph, self.nx_ph)
        if k < 16:
            return (self.nz_ph, self.ny_ph)
        return (self.nz_ph, self.nx_ph)

    def get_phasor(self, k):
        out = np.zeros(self.phasor_shape(k), self.cdtype)
        check(lib.fdtd_get_phasor(self.h, int(k), ptr(out)))
        return out

    def phasors_size(self):
        """Complex elements of the 24 phasor planes together."""
        return sum(int(np.prod(self.phasor_shape(k))) for k in range(24))

    def get_phasors(self, out=None):
        """All 24 phasor planes by name, read in one call
        (fdtd_get_phasors). ``out``: an optional flat buffer of
        phasors_size() complex elements (page-locked memory makes the
        transfer direct); the planes are views of it."""
        n = self.phasors_size()
        if out is None:
            out = np.empty(n, self.cdtype)
        if out.dtype != self.cdtype or out.size != n or not out.flags['C_CONTIGUOUS']:
            raise ValueError(f'phasor buffer must be {n} contiguous {np.dtype(self.cdtype).name}')
        check(lib.fdtd_get_phasors(self.h, ptr(out)))
        planes, off = {}, 0
        for k, name in enumerate(PHASOR_NAMES):
            shape = self.phasor_shape(k)
            m = int(np.prod(shape))
            planes[name] = out[off:off + m].reshape(shape)
            off += m
        return planes

    def get_field(self, comp):
        g = self.geom
        k = FIELD_NAMES.index(comp) if isinstance(comp, str) else int(comp)
        out = np.zeros((g.nz, g.ny, g.nx), self.dtype)
        check(lib.fdtd_get_field(self.h, k, ptr(out)))
        return out

    def set_field(self, comp, arr):
        g = self.geom
        k = FIELD_NAMES.index(comp) if isinstance(comp, str) else int(comp)
        a = self._arr(arr, (g.nz, g.ny, g.nx))
        check(lib.fdtd_set_field(self.h, k, ptr(a)))

    def grad_forward(self, checkpoint_every):
        """Reset and run all size_t steps keeping checkpoints
        (fdtd_grad_forward)."""
        check(lib.fdtd_grad_forward(self.h, int(checkpoint_every)))

    def grad_backward(self, dj_dre, dj_dim, nz_out):
        """dJ/dCa, dJ/dCb of the first nz_out planes from dJ/d(Re, Im) of the
        four upper-plane phasors, each (4, ny_ph, nx_ph) float64
        (fdtd_grad_backward)."""
        g = self.geom
        shape = (4, g.ny - 2 * g.npml, g.nx - 2 * g.npml)
        re = np.ascontiguousarray(dj_dre, dtype=np.float64)
        im = np.ascontiguousarray(dj_dim, dtype=np.float64)
        if re.shape != shape or im.shape != shape:
            raise ValueError(f'phasor gradients must have shape {shape}')
        gca = np.empty((int(nz_out), g.ny, g.nx), np.float64)
        gcb = np.empty_like(gca)
        check(lib.fdtd_grad_backward(self.h, ptr(re), ptr(im), int(nz_out), ptr(gca), ptr(gcb)))
        return gca, gcb

    def get_fields(self):
        return {c: self.get_field(c) for c in FIELD_NAMES}

    def fill_layers(self, nz_mat, heights, eps_r, sigma):
        """Stage a material block made on the device from interface height
        maps (fdtd_fill_layers); heights: (nlayers, ny, nx) cells."""
        g = self.geom
        h = np.ascontiguousarray(np.asarray(heights, dtype=np.float64).reshape(-1, g.ny, g.nx))
        e = np.ascontiguousarray(eps_r, dtype=np.float64)
        s = np.ascontiguousarray(sigma, dtype=np.float64)
        if e.shape != (h.shape[0] + 1,) or s.shape != e.shape:
            raise ValueError('eps_r and sigma need one value per layer and one above')
        check(lib.fdtd_fill_layers(self.h, int(nz_mat), int(h.shape[0]), ptr(h), ptr(e), ptr(s)))

    def paint_spheres(self, spheres, eps_r, sigma):
        """Paint (n, 5) spheres (zc, yc, xc, rc, ri in cells) into the
        staged block (fdtd_paint_spheres)."""
        sp = np.ascontiguousarray(np.asarray(spheres, dtype=np.float64).reshape(-1, 5))
        check(lib.fdtd_paint_spheres(self.h, int(sp.shape[0]), ptr(sp), float(eps_r), float(sigma)))

    def set_materials_staged(self):
        check(lib.fdtd_set_materials_staged(self.h))

    def get_staged_materials(self, nz_mat):
        g = self.geom
        e = np.empty((nz_mat, g.ny, g.nx), self.dtype)
        s = np.empty_like(e)
        check(lib.fdtd_get_staged_materials(self.h, int(nz_mat), ptr(e), ptr(s)))
        return e, s

    def near_field_power(self, inc_phasors, size_z_material, weights):
        """The 11 face powers of fdtd_near_field_power (incident, left /
        right / front / back bottom and top, down, up) from the current
        phasors; inc_phasors: ex, ey, hx, hy incident phasor planes (ny_ph,
        nx_ph); weights: the concatenated Simpson weights."""
        cd = np.complex64 if self.dtype == np.float32 else np.complex128
        inc = np.ascontiguousarray(np.stack([np.asarray(inc_phasors[k]) for k in
                                             ('ex_inc_phasor', 'ey_inc_phasor', 'hx_inc_phasor',
                                              'hy_inc_phasor')]), dtype=cd)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        out = np.zeros(11, np.float64)
        check(lib.fdtd_near_field_power(self.h, ptr(inc), int(size_z_material), ptr(w), ptr(out)))
        return out

    def set_incident_from(self, inc):
        """The first nt_inc planes recorded by a NativeIncident run, device
        to device (fdtd_set_incident_from)."""
        check(lib.fdtd_set_incident_from(self.h, inc.h))


class NativeIncident:
    """Owning wrapper of one ``fdtd_incident`` handle: the excitation and
    the vacuum run that record the incident beam. ``geom`` is the incident
    grid (nz its height, nt the recorded steps, dte0dx the vacuum's Cb)."""

    def __init__(self, geom: Geometry, nt_pulse: int, device: int = 0):
        self.geom = geom
        self.dtype = np.float32 if geom.dtype == FDTD_F32 else np.float64
        self.cdtype = np.complex64 if geom.dtype == FDTD_F32 else np.complex128
        self.nt_pulse = min(int(nt_pulse), int(geom.nt))
        h = ctypes.c_void_p()
        check(lib.fdtd_incident_create(ctypes.byref(geom), int(nt_pulse), int(device), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, 'h', None) is not None and self.h.value:
            lib.fdtd_incident_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, opt, value):
        check(lib.fdtd_incident_set_option(self.h, int(opt), int(value)))

    def set_absorbers(self, packed):
        a = np.ascontiguousarray(packed, dtype=self.dtype)
        if a.shape != (8 * self.geom.npml,):
            raise ValueError(f'expected {8 * self.geom.npml} profile values, got {a.shape}')
        check(lib.fdtd_incident_set_absorbers(self.h, ptr(a)))

    def make_excitation(self, k_vals, pulse_fft, theta_deg, phi_deg, pol, gauss_radius):
        """Excitation on the device from the pulse bins' wavenumbers and
        spectrum; returns the peak magnitude before normalisation."""
        if pol not in POLARIZATIONS:
            raise ValueError('Invalid polarization value')
        k = np.ascontiguousarray(k_vals, dtype=np.float64)
        pf = np.ascontiguousarray(pulse_fft, dtype=np.complex128)
        if k.shape != pf.shape or k.ndim != 1:
            raise ValueError('wavenumbers and pulse spectrum must be 1-D of one length')
        peak = ctypes.c_double(0)
        check(lib.fdtd_incident_make_excitation(self.h, ptr(k), ptr(pf), int(k.size), float(theta_deg),
                                                float(phi_deg), POLARIZATIONS[pol], float(gauss_radius),
                                                ctypes.byref(peak)))
        return peak.value

    def _exc_shape(self):
        return (self.nt_pulse, self.geom.ny, self.geom.nx)

    def set_excitation(self, ex_imag, ey_imag):
        a = np.ascontiguousarray(ex_imag, dtype=self.dtype)
        b = np.ascontiguousarray(ey_imag, dtype=self.dtype)
        if a.shape != self._exc_shape() or b.shape != self._exc_shape():
            raise ValueError(f'excitation must be {self._exc_shape()}')
        check(lib.fdtd_incident_set_excitation(self.h, ptr(a), ptr(b)))

    def get_excitation(self):
        a = np.zeros(self._exc_shape(), self.dtype)
        b = np.zeros(self._exc_shape(), self.dtype)
        check(lib.fdtd_incident_get_excitation(self.h, ptr(a), ptr(b)))
        return a, b

    def run(self):
        check(lib.fdtd_incident_run(self.h))

    def get_planes(self):
        g = self.geom
        out = {c: np.zeros((g.nt, g.ny, g.nx), self.dtype) for c in ('ex', 'ey', 'hx', 'hy')}
        check(lib.fdtd_incident_get_planes(self.h, *[ptr(out[c]) for c in ('ex', 'ey', 'hx', 'hy')]))
        return out

    def get_phasors(self):
        g = self.geom
        shape = (g.ny - 2 * g.npml, g.nx - 2 * g.npml)
        out = {c: np.zeros(shape, self.cdtype) for c in ('ex', 'ey', 'hx', 'hy')}
        check(lib.fdtd_incident_get_phasors(self.h, *[ptr(out[c]) for c in ('ex', 'ey', 'hx', 'hy')]))
        return {f'{c}_inc_phasor': v for c, v in out.items()}


def near2far(ex_u, ey_u, hx_u, hy_u, nx, ny, nz, dx, r, thetas_deg, phis_deg, freq, device=0,
             allocate=True):
    """Device near-to-far transform; returns E_theta, E_phi, H_theta, H_phi as
    (nphi, ntheta) complex128 arrays. With ``allocate=False`` it runs
    fdtd_near2far_noalloc, which uses the library's static device scratch
    instead of allocating (for callers that may not allocate device memory;
    sizes are capped, see include/fdtd_b200.h)."""
    ex_u = np.asarray(ex_u)
    in_dtype = FDTD_F32 if ex_u.dtype == np.complex64 else FDTD_F64
    cdt = np.complex64 if in_dtype == FDTD_F32 else np.complex128
    planes = [np.ascontiguousarray(p, dtype=cdt) for p in (ex_u, ey_u, hx_u, hy_u)]
    for p in planes:
        if p.shape != (ny, nx):
            raise ValueError(f'phasor planes must be ({ny}, {nx}), got {p.shape}')
    th = np.ascontiguousarray(thetas_deg, dtype=np.float64)
    ph = np.ascontiguousarray(phis_deg, dtype=np.float64)
    out = np.zeros((4, ph.size, th.size), np.complex128)
    fn = lib.fdtd_near2far if allocate else lib.fdtd_near2far_noalloc
    check(fn(*[ptr(p) for p in planes], in_dtype, int(nx), int(ny), int(nz),
                            float(dx), float(r), ptr(th), int(th.size), ptr(ph), int(ph.size),
                            float(freq), int(device), ptr(out)))
    return {'E_theta': out[0], 'E_phi': out[1], 'H_theta': out[2], 'H_phi': out[3]}


def check_cell_division(dtype, cell_size, device=0):
    """(tested, mismatches): the library's division by the cell size
    against IEEE division on the device (fdtd_check_cell_division)."""
    tested, bad = ctypes.c_int64(0), ctypes.c_int64(0)
    check(lib.fdtd_check_cell_division(dtype_code(dtype), float(cell_size), int(device),
                                       ctypes.byref(tested), ctypes.byref(bad)))
    return tested.value, bad.value


def bounds_check_enabled():
    """True when the loaded library is the bounds-checked build."""
    return bool(lib.fdtd_bounds_check_enabled())


def fused_plan_boxes(nx, ny, nz, npml, tfsf_z, tile_y=4, zchunk=0, slab=False, march=False):
    """(kind, x0, x1, y0, y1, z0, z1) rows of the fused step's boxes
    (fdtd_fused_plan_boxes; host computation, no device needed): kind 0
    interior march, 1 CPML z slab march (with ``slab=2`` the column march),
    2 split-pass shell box, 3 general march shell box. ``march`` gives the
    plan with the shell marched; otherwise the split-pass shell, with
    ``slab`` 1 the z slabs marched, 2 the column march
    (FDTD_OPT_FUSED_SLAB)."""
    out = np.zeros((64, 7), np.int32)
    n = ctypes.c_int(0)
    mode = 2 if march else (3 if int(slab) == 2 else int(bool(slab)))
    check(lib.fdtd_fused_plan_boxes(int(nx), int(ny), int(nz), int(npml), int(tfsf_z), int(tile_y),
                                    int(zchunk), mode, ptr(out), out.shape[0], ctypes.byref(n)))
    return out[:n.value].copy()


class Batch:
    """Several NativeSim members advanced together (fdtd_batch_*): by
    default one launch per pass for all members each step, chunks of steps
    replayed from a captured CUDA graph; with ``streams=True`` every member
    runs its own step path on its own stream, side by side; with
    ``mode=BATCH_QUEUE`` every member takes its fused step: one persistent
    launch per step walks a tile queue over all members' interior tiles and
    one launch per split pass sweeps all their shells. Members keep their
    own state and readback calls."""

    def __init__(self, sims, graph_chunk=None, streams=False, mode=None):
        self.sims = list(sims)   # keeps the members alive while the batch exists
        arr = (_P * len(self.sims))(*[s.h for s in self.sims])
        self.h = _P()
        check(lib.fdtd_batch_create(arr, len(self.sims), ctypes.byref(self.h)))
        if graph_chunk is not None:
            self.set_graph_chunk(graph_chunk)
        if streams:
            self.set_streams(True)
        if mode is not None:
            self.set_mode(mode)

    def set_mode(self, mode):
        """BATCH_SPLIT, BATCH_STREAMS or BATCH_QUEUE (FDTD_OPT_BATCH_MODE)."""
        check(lib.fdtd_batch_set_option(self.h, OPT_BATCH_MODE, int(mode)))

    def set_graph_chunk(self, steps):
        check(lib.fdtd_batch_set_option(self.h, OPT_GRAPH_CHUNK, int(steps)))

    def set_streams(self, on):
        check(lib.fdtd_batch_set_option(self.h, OPT_BATCH_STREAMS, int(bool(on))))

    def run(self, nsteps):
        check(lib.fdtd_batch_run(self.h, int(nsteps)))

    def synchronize(self):
        check(lib.fdtd_batch_synchronize(self.h))

    def stream(self):
        p = _P()
        check(lib.fdtd_batch_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def close(self):
        if self.h:
            lib.fdtd_batch_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
