"""CPU oracle for the FDTD time-stepping path -- TEST INFRASTRUCTURE ONLY.

This module restates, in vectorised numpy, the algorithm of the reference
package ``fdtdsarsim`` (wyatt-sfu/sar-pixel-simulator) for one Yee time step
with CPML absorbers, one-plane incident injection and running phasor DFTs.
The CUDA path's results are compared against it: only ``tests/``, ``__graft_entry__.smoke``
and ``bench.py`` (its CPU-baseline leg) may import it, and never as the thing
that is measured or shipped.

Every floating-point operation keeps the reference's evaluation order and
precision, so that in float32 the oracle reproduces the reference bit for
bit (the reference's numba kernels do not contract multiply-adds):

* field updates: ``cpu/field_updates.py:18-63`` (E) and ``:198-240`` (H);
* CPML: ``cpu/field_updates.py:66-191`` (E) and ``:243-366`` (H), applied
  in the reference's face order z (down/up), x (left/right), y (front/back)
  (``cpu/fdtd_sim.py:51-133``);
* incident injection: ``cpu/main_sim.py:147-161`` (all x, all y);
* phasors: ``cpu/field_updates.py:373-461``; the phase factor is evaluated in
  float64 (complex128 in the reference) and each accumulation is the float64
  sum of the stored phasor and the new term, rounded back to the phasor's
  storage precision;
* loop order: ``cpu/main_sim.py:140-195``.

Parity is pinned against fixtures produced by running the reference itself
(``tests/golden/make_golden.py``); ``tests/test_oracle_golden.py`` checks it.
"""
import math

import numpy as np

PHASOR_NAMES = [
    'ex_ph_d', 'ey_ph_d', 'hx_ph_d', 'hy_ph_d',
    'ex_ph_u', 'ey_ph_u', 'hx_ph_u', 'hy_ph_u',
    'ey_ph_l', 'ez_ph_l', 'hy_ph_l', 'hz_ph_l',
    'ey_ph_r', 'ez_ph_r', 'hy_ph_r', 'hz_ph_r',
    'ex_ph_f', 'ez_ph_f', 'hx_ph_f', 'hz_ph_f',
    'ex_ph_b', 'ez_ph_b', 'hx_ph_b', 'hz_ph_b',
]

# scipy.constants (CODATA 2022) values used by the reference's main loop
# (cpu/main_sim.py:98-99, 127-130)
MU0 = 1.25663706127e-06
EPS0_CODATA = 8.8541878188e-12


def phase_factors(omega, t, dt):
    """(cos, sin) of the E and H phase angles used at step ``t``.

    The reference evaluates ``np.exp(-1j*omega*t*dt)`` and
    ``np.exp(-1j*omega*(t-0.5)*dt)`` in complex128
    (cpu/field_updates.py:387,395); the imaginary part of the argument is
    ``(-omega*t)*dt`` and the real part is zero.
    """
    th_e = (-omega * t) * dt
    th_h = (-omega * (t - 0.5)) * dt
    return math.cos(th_e), math.sin(th_e), math.cos(th_h), math.sin(th_h)


def _acc(ph, mean, c, s):
    """ph += mean * (c + i s), float64 sum rounded to ph's precision."""
    rdt = ph.real.dtype
    m = mean.astype(np.float64)
    ph.real = (ph.real.astype(np.float64) + m * c).astype(rdt)
    ph.imag = (ph.imag.astype(np.float64) + m * s).astype(rdt)


class OracleSim:
    """Reference-faithful FDTD state machine on numpy arrays.

    Args:
        nx, ny, nz, npml, tfsf_z: grid geometry (cells)
        dx, dt: cell size [m] and time step [s] (Python floats)
        freq: phasor frequency [Hz]
        dtype: 'float32' or 'float64'
        profiles: dict of the eight 1-D CPML coefficient profiles
            be_d, bh_d, ce_d, ch_d (down/left/front) and be_u, bh_u, ce_u,
            ch_u (up/right/back), each of length npml
    """

    def __init__(self, nx, ny, nz, npml, tfsf_z, dx, dt, freq, dtype,
                 profiles):
        self.nx, self.ny, self.nz, self.npml = nx, ny, nz, npml
        self.tfsf_z = tfsf_z
        self.dtype = np.dtype(dtype)
        ft = self.dtype.type
        self.dt = dt
        self.omega = 2.0 * np.pi * freq
        self.Db = ft(dt / (MU0 * dx))
        self.dtm0 = ft(dt / MU0)
        self.dxf = ft(dx)
        self.dte0dx = ft(dt / (EPS0_CODATA * dx))
        self.p = {k: np.asarray(v, dtype=self.dtype) for k, v in profiles.items()}
        self.reset()

    def reset(self):
        nx, ny, nz, npml, dt = self.nx, self.ny, self.nz, self.npml, self.dtype
        for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz'):
            setattr(self, c, np.zeros((nz, ny, nx), dt))
        self.psi = {}
        for n in ('Exz', 'Eyz', 'Hxz', 'Hyz'):
            for s in ('d', 'u'):
                self.psi[n + s] = np.zeros((npml, ny, nx), dt)
        for n in ('Eyx', 'Ezx', 'Hyx', 'Hzx'):
            for s in ('l', 'r'):
                self.psi[n + s] = np.zeros((nz, ny, npml), dt)
        for n in ('Exy', 'Ezy', 'Hxy', 'Hzy'):
            for s in ('f', 'b'):
                self.psi[n + s] = np.zeros((nz, npml, nx), dt)
        cdt = np.complex64 if dt == np.float32 else np.complex128
        self.nx_ph, self.ny_ph, self.nz_ph = nx - 2 * npml, ny - 2 * npml, nz - 2 * npml
        self.ph = {}
        for name in PHASOR_NAMES:
            face = name[-1]
            if face in 'du':
                shape = (self.ny_ph, self.nx_ph)
            elif face in 'lr':
                shape = (self.nz_ph, self.ny_ph)
            else:
                shape = (self.nz_ph, self.nx_ph)
            self.ph[name] = np.zeros(shape, cdt)
        self.t = 0

    # ------------------------------------------------------------------
    # H half step (cpu/field_updates.py:198-240, 243-366)
    # ------------------------------------------------------------------
    def h_update(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        ex, ey, ez, hx, hy, hz = self.ex, self.ey, self.ez, self.hx, self.hy, self.hz
        Db = self.Db
        s = np.s_[0:nz - 1, 0:ny - 1, 1:nx - 1]
        dez = ez[0:nz - 1, 1:ny, 1:nx - 1] - ez[s]
        dey = ey[1:nz, 0:ny - 1, 1:nx - 1] - ey[s]
        hx[s] -= Db * (dez - dey)
        s = np.s_[0:nz - 1, 1:ny - 1, 0:nx - 1]
        dex = ex[1:nz, 1:ny - 1, 0:nx - 1] - ex[s]
        dez = ez[0:nz - 1, 1:ny - 1, 1:nx] - ez[s]
        hy[s] -= Db * (dex - dez)
        s = np.s_[1:nz - 1, 0:ny - 1, 0:nx - 1]
        dex = ex[1:nz - 1, 1:ny, 0:nx - 1] - ex[s]
        dey = ey[1:nz - 1, 0:ny - 1, 1:nx] - ey[s]
        hz[s] -= Db * (dey - dex)

    def h_cpml(self):
        nx, ny, nz, m = self.nx, self.ny, self.nz, self.npml
        ex, ey, ez, hx, hy, hz = self.ex, self.ey, self.ez, self.hx, self.hy, self.hz
        P, p, dx, dtm0 = self.psi, self.p, self.dxf, self.dtm0
        # down / up: z faces, psi over z in [0, m-1), y in [0, ny-1), x in [0, nx-1)
        for side, z0 in (('d', 0), ('u', nz - m)):
            b = p['bh_' + side][0:m - 1, None, None]
            c = p['ch_' + side][0:m - 1, None, None]
            f = np.s_[z0:z0 + m - 1, 0:ny - 1, 0:nx - 1]
            fu = np.s_[z0 + 1:z0 + m, 0:ny - 1, 0:nx - 1]
            q = np.s_[0:m - 1, 0:ny - 1, 0:nx - 1]
            P['Hyz' + side][q] = b * P['Hyz' + side][q] + c * (ex[fu] - ex[f]) / dx
            P['Hxz' + side][q] = b * P['Hxz' + side][q] + c * (ey[fu] - ey[f]) / dx
            hy[f] -= dtm0 * P['Hyz' + side][q]
            hx[f] += dtm0 * P['Hxz' + side][q]
        # left / right: x faces, z in [0, nz-1), y in [0, ny-1), x in [0, m-1)
        for side, x0, pk in (('l', 0, 'd'), ('r', nx - m, 'u')):
            b = p['bh_' + pk][None, None, 0:m - 1]
            c = p['ch_' + pk][None, None, 0:m - 1]
            f = np.s_[0:nz - 1, 0:ny - 1, x0:x0 + m - 1]
            fr = np.s_[0:nz - 1, 0:ny - 1, x0 + 1:x0 + m]
            q = np.s_[0:nz - 1, 0:ny - 1, 0:m - 1]
            P['Hzx' + side][q] = b * P['Hzx' + side][q] + c * (ey[fr] - ey[f]) / dx
            P['Hyx' + side][q] = b * P['Hyx' + side][q] + c * (ez[fr] - ez[f]) / dx
            hz[f] -= dtm0 * P['Hzx' + side][q]
            hy[f] += dtm0 * P['Hyx' + side][q]
        # front / back: y faces, z in [0, nz-1), y in [0, m-1), x in [0, nx-1)
        for side, y0, pk in (('f', 0, 'd'), ('b', ny - m, 'u')):
            b = p['bh_' + pk][None, 0:m - 1, None]
            c = p['ch_' + pk][None, 0:m - 1, None]
            f = np.s_[0:nz - 1, y0:y0 + m - 1, 0:nx - 1]
            fb = np.s_[0:nz - 1, y0 + 1:y0 + m, 0:nx - 1]
            q = np.s_[0:nz - 1, 0:m - 1, 0:nx - 1]
            P['Hxy' + side][q] = b * P['Hxy' + side][q] + c * (ez[fb] - ez[f]) / dx
            P['Hzy' + side][q] = b * P['Hzy' + side][q] + c * (ex[fb] - ex[f]) / dx
            hx[f] -= dtm0 * P['Hxy' + side][q]
            hz[f] += dtm0 * P['Hzy' + side][q]

    # ------------------------------------------------------------------
    # E half step (cpu/field_updates.py:18-63, 66-191)
    # ------------------------------------------------------------------
    def e_update(self, ca, cb):
        nx, ny, nz = self.nx, self.ny, self.nz
        ex, ey, ez, hx, hy, hz = self.ex, self.ey, self.ez, self.hx, self.hy, self.hz
        s = np.s_[1:nz - 1, 1:ny - 1, 0:nx - 1]
        scaled = ex[s] * ca[s]
        dhz = hz[s] - hz[1:nz - 1, 0:ny - 2, 0:nx - 1]
        dhy = hy[s] - hy[0:nz - 2, 1:ny - 1, 0:nx - 1]
        ex[s] = scaled + (cb[s] * (dhz - dhy))
        s = np.s_[1:nz - 1, 0:ny - 1, 1:nx - 1]
        scaled = ey[s] * ca[s]
        dhx = hx[s] - hx[0:nz - 2, 0:ny - 1, 1:nx - 1]
        dhz = hz[s] - hz[1:nz - 1, 0:ny - 1, 0:nx - 2]
        ey[s] = scaled + (cb[s] * (dhx - dhz))
        s = np.s_[0:nz - 1, 1:ny - 1, 1:nx - 1]
        scaled = ez[s] * ca[s]
        dhx = hx[s] - hx[0:nz - 1, 0:ny - 2, 1:nx - 1]
        dhy = hy[s] - hy[0:nz - 1, 1:ny - 1, 0:nx - 2]
        ez[s] = scaled + (cb[s] * (dhy - dhx))

    def e_cpml(self, cb):
        nx, ny, nz, m = self.nx, self.ny, self.nz, self.npml
        ex, ey, ez, hx, hy, hz = self.ex, self.ey, self.ez, self.hx, self.hy, self.hz
        P, p, dx = self.psi, self.p, self.dxf
        # down: psi z in [1, m) -> field z in [1, m); up: psi z in [0, m-1)
        # -> field z in [nz-m, nz-1)
        for side, q0, z0 in (('d', 1, 1), ('u', 0, nz - m)):
            b = p['be_' + side][q0:q0 + m - 1, None, None]
            c = p['ce_' + side][q0:q0 + m - 1, None, None]
            f = np.s_[z0:z0 + m - 1, 0:ny - 1, 0:nx - 1]
            fd = np.s_[z0 - 1:z0 + m - 2, 0:ny - 1, 0:nx - 1]
            q = np.s_[q0:q0 + m - 1, 0:ny - 1, 0:nx - 1]
            P['Eyz' + side][q] = b * P['Eyz' + side][q] + c * (hx[f] - hx[fd]) / dx
            P['Exz' + side][q] = b * P['Exz' + side][q] + c * (hy[f] - hy[fd]) / dx
            ey[f] += cb[f] * dx * P['Eyz' + side][q]
            ex[f] -= cb[f] * dx * P['Exz' + side][q]
        for side, q0, x0, pk in (('l', 1, 1, 'd'), ('r', 0, nx - m, 'u')):
            b = p['be_' + pk][None, None, q0:q0 + m - 1]
            c = p['ce_' + pk][None, None, q0:q0 + m - 1]
            f = np.s_[0:nz - 1, 0:ny - 1, x0:x0 + m - 1]
            fl = np.s_[0:nz - 1, 0:ny - 1, x0 - 1:x0 + m - 2]
            q = np.s_[0:nz - 1, 0:ny - 1, q0:q0 + m - 1]
            P['Ezx' + side][q] = b * P['Ezx' + side][q] + c * (hy[f] - hy[fl]) / dx
            P['Eyx' + side][q] = b * P['Eyx' + side][q] + c * (hz[f] - hz[fl]) / dx
            ez[f] += cb[f] * dx * P['Ezx' + side][q]
            ey[f] -= cb[f] * dx * P['Eyx' + side][q]
        for side, q0, y0, pk in (('f', 1, 1, 'd'), ('b', 0, ny - m, 'u')):
            b = p['be_' + pk][None, q0:q0 + m - 1, None]
            c = p['ce_' + pk][None, q0:q0 + m - 1, None]
            f = np.s_[0:nz - 1, y0:y0 + m - 1, 0:nx - 1]
            ff = np.s_[0:nz - 1, y0 - 1:y0 + m - 2, 0:nx - 1]
            q = np.s_[0:nz - 1, q0:q0 + m - 1, 0:nx - 1]
            P['Exy' + side][q] = b * P['Exy' + side][q] + c * (hz[f] - hz[ff]) / dx
            P['Ezy' + side][q] = b * P['Ezy' + side][q] + c * (hx[f] - hx[ff]) / dx
            ex[f] += cb[f] * dx * P['Exy' + side][q]
            ez[f] -= cb[f] * dx * P['Ezy' + side][q]

    # ------------------------------------------------------------------
    # phasors (cpu/field_updates.py:373-461)
    # ------------------------------------------------------------------
    def phasors(self, t):
        m, nx, ny, nz = self.npml, self.nx, self.ny, self.nz
        cE, sE, cH, sH = phase_factors(self.omega, t, self.dt)
        ex, ey, ez, hx, hy, hz = self.ex, self.ey, self.ez, self.hx, self.hy, self.hz
        ph = self.ph
        Z = np.s_[m + 1:m + self.nz_ph]
        Zd = np.s_[m:m + self.nz_ph - 1]
        Y = np.s_[m + 1:m + self.ny_ph]
        Yd = np.s_[m:m + self.ny_ph - 1]
        X = np.s_[m + 1:m + self.nx_ph]
        Xd = np.s_[m:m + self.nx_ph - 1]
        for side, px in (('l', m + 1), ('r', nx - m - 1)):
            _acc(ph['ey_ph_' + side][1:, 1:], 0.5 * (ey[Z, Y, px] + ey[Z, Yd, px]).astype(np.float64), cE, sE)
            _acc(ph['ez_ph_' + side][1:, 1:], 0.5 * (ez[Z, Y, px] + ez[Zd, Y, px]).astype(np.float64), cE, sE)
            _acc(ph['hy_ph_' + side][1:, 1:], 0.25 * (hy[Z, Y, px] + hy[Z, Y, px - 1] + hy[Zd, Y, px]
                                                      + hy[Zd, Y, px - 1]).astype(np.float64), cH, sH)
            _acc(ph['hz_ph_' + side][1:, 1:], 0.25 * (hz[Z, Y, px] + hz[Z, Y, px - 1] + hz[Z, Yd, px]
                                                      + hz[Z, Yd, px - 1]).astype(np.float64), cH, sH)
        for side, py in (('f', m + 1), ('b', ny - m - 1)):
            _acc(ph['ex_ph_' + side][1:, 1:], 0.5 * (ex[Z, py, X] + ex[Z, py, Xd]).astype(np.float64), cE, sE)
            _acc(ph['ez_ph_' + side][1:, 1:], 0.5 * (ez[Z, py, X] + ez[Zd, py, X]).astype(np.float64), cE, sE)
            _acc(ph['hx_ph_' + side][1:, 1:], 0.25 * (hx[Z, py, X] + hx[Z, py - 1, X] + hx[Zd, py, X]
                                                      + hx[Zd, py - 1, X]).astype(np.float64), cH, sH)
            _acc(ph['hz_ph_' + side][1:, 1:], 0.25 * (hz[Z, py, X] + hz[Z, py - 1, X] + hz[Z, py, Xd]
                                                      + hz[Z, py - 1, Xd]).astype(np.float64), cH, sH)
        for side, pz in (('d', m + 1), ('u', nz - m - 1)):
            _acc(ph['ex_ph_' + side][1:, 1:], 0.5 * (ex[pz, Y, X] + ex[pz, Y, Xd]).astype(np.float64), cE, sE)
            _acc(ph['ey_ph_' + side][1:, 1:], 0.5 * (ey[pz, Y, X] + ey[pz, Yd, X]).astype(np.float64), cE, sE)
            _acc(ph['hx_ph_' + side][1:, 1:], 0.25 * (hx[pz, Y, X] + hx[pz, Yd, X] + hx[pz - 1, Y, X]
                                                      + hx[pz - 1, Yd, X]).astype(np.float64), cH, sH)
            _acc(ph['hy_ph_' + side][1:, 1:], 0.25 * (hy[pz, Y, X] + hy[pz, Y, Xd] + hy[pz - 1, Y, X]
                                                      + hy[pz - 1, Y, Xd]).astype(np.float64), cH, sH)

    # ------------------------------------------------------------------
    # one full step (cpu/main_sim.py:140-195)
    # ------------------------------------------------------------------
    def step(self, ca, cb, inc):
        """Advance one time step. ``inc`` maps 'ex','ey','hx','hy' to
        (ntp, ny, nx) arrays; injection happens while t < ntp."""
        t = self.t
        ntp = inc['ex'].shape[0] if inc is not None else 0
        self.h_update()
        self.h_cpml()
        if t < ntp:
            self.hx[self.tfsf_z, :, :] += self.Db * inc['ey'][t, :, :]
            self.hy[self.tfsf_z, :, :] -= self.Db * inc['ex'][t, :, :]
        self.e_update(ca, cb)
        self.e_cpml(cb)
        if t < ntp:
            self.ey[self.tfsf_z, :, :] += self.dte0dx * inc['hx'][t, :, :]
            self.ex[self.tfsf_z, :, :] -= self.dte0dx * inc['hy'][t, :, :]
        self.phasors(t)
        self.t = t + 1

    def run(self, ca, cb, inc, nt):
        for _ in range(nt):
            self.step(ca, cb, inc)

    def fields(self):
        return {c: getattr(self, c) for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')}


# ----------------------------------------------------------------------
# near-to-far transform (near2far.py:28-156)
# ----------------------------------------------------------------------
def simpson_weights(n, dx):
    """Composite Simpson 1/3 weights for an odd number of samples.

    scipy.integrate.simpson (scipy 1.18, the reference's dependency,
    near2far.py:26) reduces to this rule when the sample count is odd,
    which it always is for the phasor planes (nx, ny forced odd,
    utils/rounding.py:4-15).
    """
    if n % 2 != 1 or n < 3:
        raise ValueError('odd sample count >= 3 required')
    w = np.ones(n)
    w[1:-1:2] = 4.0
    w[2:-1:2] = 2.0
    return w * dx / 3.0


def near2far(ex_u, ey_u, hx_u, hy_u, nx, ny, nz, dx, r, thetas_deg, phis_deg,
             freq):
    """Far-field E/H (theta, phi components) from the top phasor plane.

    Restates FarFieldTransform.__call__ (near2far.py:28-112) and
    _integrate_z_plane (near2far.py:114-156): J = (-Hy, Hx), M = (Ey, -Ex)
    on the plane z = z_loc[-1]; N and L potentials by 2-D Simpson
    integration (x first, then y); outputs have shape (nphi, ntheta)
    squeezed like the reference.
    """
    eta0 = 376.730313668
    c0 = 299792458
    lam = c0 / freq
    k = 2.0 * np.pi / lam
    th = np.deg2rad(np.asarray(thetas_deg, dtype=np.float64))
    ph = np.deg2rad(np.asarray(phis_deg, dtype=np.float64))
    x_loc = np.arange(-(nx - 1) // 2, ((nx - 1) // 2) + 1) * dx
    y_loc = np.arange(-(ny - 1) // 2, ((ny - 1) // 2) + 1) * dx
    z_loc = np.arange(-(nz - 1) // 2, ((nz - 1) // 2) + 1) * dx
    z_val = z_loc[-1]
    Jx = -np.asarray(hy_u, dtype=np.complex128)
    Jy = np.asarray(hx_u, dtype=np.complex128)
    Mx = np.asarray(ey_u, dtype=np.complex128)
    My = -np.asarray(ex_u, dtype=np.complex128)
    wx = simpson_weights(nx, dx)
    wy = simpson_weights(ny, dx)
    xx, yy = np.meshgrid(x_loc, y_loc)
    ffw = 1j * k * np.exp(-1j * k * r) / (4.0 * np.pi * r)
    shape = (ph.shape[0], th.shape[0])
    out = {n: np.zeros(shape, np.complex128) for n in ('E_theta', 'E_phi', 'H_theta', 'H_phi')}
    for i, p_ in enumerate(ph):
        for j, t_ in enumerate(th):
            e = np.exp(1j * k * (xx * np.sin(t_) * np.cos(p_) + yy * np.sin(t_) * np.sin(p_)
                                 + z_val * np.cos(t_)))
            ct, st, cp, sp = np.cos(t_), np.sin(t_), np.cos(p_), np.sin(p_)
            del st

            def integ(f):
                return wy @ (f @ wx)
            Nt = integ((Jx * ct * cp + Jy * ct * sp) * e)
            Np = integ((-Jx * sp + Jy * cp) * e)
            Lt = integ((Mx * ct * cp + My * ct * sp) * e)
            Lp = integ((-Mx * sp + My * cp) * e)
            out['E_theta'][i, j] = ffw * (-Lp - eta0 * Nt)
            out['E_phi'][i, j] = ffw * (Lt - eta0 * Np)
            out['H_theta'][i, j] = ffw * (Np - Lt / eta0)
            out['H_phi'][i, j] = ffw * (-Nt - Lp / eta0)
    return {k_: np.squeeze(v) for k_, v in out.items()}


def farfield_power(e_theta, e_phi, h_theta, h_phi):
    """(horizontal, vertical) scattered power (processresults.py:260-271)."""
    return (0.5 * np.real(-e_phi * np.conj(h_theta)),
            0.5 * np.real(e_theta * np.conj(h_phi)))
