"""CPU oracle for the incident-beam generation -- TEST INFRASTRUCTURE ONLY.

Restates in numpy how the reference package ``fdtdsarsim``
(wyatt-sfu/sar-pixel-simulator) makes the incident beam that a main
simulation injects. The CUDA path's results are compared against it (only
``tests/`` may import it); it is never the thing that is measured or shipped.

* ``create_pulse``: the Gaussian-tapered complex carrier and its FFT
  (``incidentbeam.py:174-204``);
* ``taper_k``: Braunisch's tapered wave in the spatial-frequency domain
  (``incidentbeam.py:317-433``);
* ``create_inc_excitation``: per temporal frequency, the 2-D FFT of the
  tapered spectrum weighted by the pulse spectrum, the inverse FFT along
  time, and the normalisation to a peak magnitude of 10
  (``incidentbeam.py:206-298``). The stages keep the reference's storage
  precision: the weighted spectra are stored in the complex type of the
  simulation and the time-axis inverse FFT runs in it;
* ``IncidentOracle``: the vacuum FDTD run of ``cpu/incident_sim.py:67-171``
  (E update, E CPML, hard source on plane nz // 2 + 4, H update, H CPML,
  read-out of plane nz // 2, incident phasors of
  ``cpu/field_updates.py:465-491``), on the step functions of
  ``fdtd_oracle.OracleSim``.

Parity: the FDTD run is pinned bit for bit against planes and phasors that
the reference itself produced (``tests/golden/incident_*.npz``, made by
``tests/golden/make_golden.py``) from the reference's own excitation; the
excitation is pinned against the reference's to a tolerance (the reference
evaluates its transcendental functions in numba, this file in numpy).
"""
import math

import numpy as np

from fdtd_oracle import EPS0_CODATA, MU0, OracleSim, _acc

C0 = 299792458.0


def create_pulse(dt, nt_inc, nt_pulse, duration, freq):
    """(time_vals, pulse, pulse_fft, pulse_freqs) of incidentbeam.py:174-199."""
    time_vals = np.linspace(0.0, dt * (nt_inc - 1), num=nt_inc, endpoint=True)
    sig = duration / freq / (2.0 * np.sqrt(2.0 * np.log(10.0)))
    om = 2.0 * np.pi * freq
    pulse = 1.0 * np.exp(-(time_vals - (dt * nt_pulse / 2)) ** 2 / (sig ** 2)) \
        * np.exp(1j * om * time_vals)
    return time_vals, pulse, np.fft.fft(pulse), np.fft.fftfreq(pulse.size, dt)


def spatial_freqs(nx, ny, dx):
    """kx, ky (ny, nx) in the reference's centred order (incidentbeam.py:235-244)."""
    kx = np.fft.fftshift(np.broadcast_to(2 * np.pi * np.fft.fftfreq(nx, dx), (ny, nx)), axes=1)
    ky = np.fft.fftshift(np.broadcast_to((2 * np.pi * np.fft.fftfreq(ny, dx))[:, None], (ny, nx)),
                         axes=0)
    return np.ascontiguousarray(kx), np.ascontiguousarray(ky)


_POL = {'HH': (1.0, 0.0), 'VV': (0.0, 1.0), 'RHCP': (-1j, 1.0), 'LHCP': (1j, 1.0)}


def taper_k(k, kx, ky, theta_deg, phi_deg, radius, pol):
    """(x, y) spectral components of the tapered wave at wavenumber k
    (incidentbeam.py:317-433, equations 4-16 of Braunisch)."""
    if pol not in _POL:
        raise ValueError('Invalid polarization value')
    kp = np.hypot(kx, ky)
    kz = np.conj(np.sqrt((k ** 2 - kp ** 2).astype(np.complex64)))   # complex64, as the reference
    th, ph = np.radians(theta_deg), np.radians(phi_deg)
    kix = k * np.sin(th) * np.cos(ph)
    kiy = k * np.sin(th) * np.sin(ph)
    kip = np.hypot(kix, kiy)
    kiz = np.sqrt(k ** 2 - kip ** 2)
    gauss = ((radius ** 2) / (4 * np.pi)) * np.exp(-(radius ** 2) * (((kx - kix) ** 2) + ((ky - kiy) ** 2)) / 4)
    pos = kp > 0.0
    safe = np.where(pos, kp, 1.0)
    hor_x = np.where(pos, ky / safe, np.sin(ph)).astype(np.complex128)
    hor_y = np.where(pos, -kx / safe, -np.cos(ph)).astype(np.complex128)
    ver_x = np.where(pos, (kz * kx) / (k * safe), np.cos(ph))
    ver_y = np.where(pos, (kz * ky) / (k * safe), np.sin(ph))
    ver_z = np.where(pos, kp / k, 0.0).astype(np.complex128)
    if kip > 0:
        hix, hiy = kiy / kip, -kix / kip
        vix, viy, viz = (kiz * kix) / (k * kip), (kiz * kiy) / (k * kip), kip / k
    else:
        hix, hiy = np.sin(ph), -np.cos(ph)
        vix, viy, viz = np.cos(ph), np.sin(ph), 0.0
    eh_, ev_ = _POL[pol]
    eh = eh_ * ((hix * hor_x) + (hiy * hor_y)) + ev_ * ((vix * hor_x) + (viy * hor_y))
    ev = eh_ * ((hix * ver_x) + (hiy * ver_y)) + ev_ * ((vix * ver_x) + (viy * ver_y) + (viz * ver_z))
    return gauss * ((eh * hor_x) + (ev * ver_x)), gauss * ((eh * hor_y) + (ev * ver_y))


def gauss_radius(illumination_width, freq):
    """Footprint radius of the taper (incidentbeam.py:231-233)."""
    width = illumination_width * C0 / freq
    return width / (2.0 * np.sqrt(2.0 * np.log(10.0)))


def create_inc_excitation(nx, ny, dx, pulse_fft, pulse_freqs, theta_deg, phi_deg, pol, radius,
                          dtype='float32'):
    """(pulse_ex, pulse_ey) complex (nt_inc, ny, nx), normalised to a peak
    magnitude of 10 (incidentbeam.py:206-298)."""
    cdt = np.complex64 if np.dtype(dtype) == np.float32 else np.complex128
    nt = len(pulse_fft)
    kx, ky = spatial_freqs(nx, ny, dx)
    all_k = (2 * np.pi * pulse_freqs) / C0
    out = [np.zeros((nt, ny, nx), cdt), np.zeros((nt, ny, nx), cdt)]
    for i in range(nt):
        if all_k[i] == 0.0:
            continue
        spec = taper_k(all_k[i], kx, ky, theta_deg, phi_deg, radius, pol)
        for c in range(2):
            out[c][i] = 1.0 * pulse_fft[i] * np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(spec[c])))
    for c in range(2):
        out[c] = np.fft.ifft(out[c], axis=0).astype(cdt)
    peak = max(np.abs(out[0]).max(), np.abs(out[1]).max())
    scale = 10.0 / float(peak)
    return (out[0] * scale).astype(cdt), (out[1] * scale).astype(cdt)


def incident_height(cell_size, freq):
    """Cells of the incident grid along z: int(3 wavelengths / cell)
    (cpu/incident_sim.py:33-37)."""
    lam = 299792458 / freq
    return int(3.0 * lam / cell_size)


class IncidentOracle(OracleSim):
    """The incident-beam FDTD run (cpu/incident_sim.py:67-171) in vacuum:
    Ca = 1, Cb = dt / (eps0 dx) with scipy's eps0."""

    def __init__(self, nx, ny, nz, npml, dx, dt, freq, dtype, profiles):
        super().__init__(nx, ny, nz, npml, nz // 2, dx, dt, freq, dtype, profiles)
        ft = self.dtype.type
        self.ca = np.ones((nz, ny, nx), self.dtype)
        self.cb = ft(dt / (EPS0_CODATA * dx)) * np.ones((nz, ny, nx), self.dtype)
        self.Db = ft(dt / (MU0 * dx))
        self.dtm0 = ft(dt / MU0)
        self.feed_in = nz // 2 + 4
        self.read_out = self.feed_in - 4
        cdt = np.complex64 if self.dtype == np.float32 else np.complex128
        self.inc_ph = {c: np.zeros((ny - 2 * npml, nx - 2 * npml), cdt) for c in ('ex', 'ey', 'hx', 'hy')}

    def incident_phasors(self, t):
        """cpu/field_updates.py:465-491: E averaged with phase
        exp(-i omega (t - 1/2) dt), H with exp(-i omega t dt)."""
        m, z = self.npml, self.read_out
        th_e = (-self.omega * (t - 0.5)) * self.dt
        th_h = (-self.omega * t) * self.dt
        cE, sE, cH, sH = math.cos(th_e), math.sin(th_e), math.cos(th_h), math.sin(th_h)
        ny_ph, nx_ph = self.inc_ph['ex'].shape
        Y = np.s_[m + 1:m + ny_ph]
        Yd = np.s_[m:m + ny_ph - 1]
        X = np.s_[m + 1:m + nx_ph]
        Xd = np.s_[m:m + nx_ph - 1]
        ex, ey, hx, hy = self.ex, self.ey, self.hx, self.hy
        _acc(self.inc_ph['ex'][1:, 1:], 0.5 * (ex[z, Y, X] + ex[z, Y, Xd]).astype(np.float64), cE, sE)
        _acc(self.inc_ph['ey'][1:, 1:], 0.5 * (ey[z, Y, X] + ey[z, Yd, X]).astype(np.float64), cE, sE)
        _acc(self.inc_ph['hx'][1:, 1:], 0.25 * (hx[z, Y, X] + hx[z, Yd, X] + hx[z - 1, Y, X]
                                                + hx[z - 1, Yd, X]).astype(np.float64), cH, sH)
        _acc(self.inc_ph['hy'][1:, 1:], 0.25 * (hy[z, Y, X] + hy[z, Y, Xd] + hy[z - 1, Y, X]
                                                + hy[z - 1, Y, Xd]).astype(np.float64), cH, sH)

    def run_incident(self, exc_ex_imag, exc_ey_imag, ntp):
        """Run ntp steps injecting the excitation's imaginary parts
        (nt_pulse, ny, nx) while t < nt_pulse; returns the recorded planes
        {'ex', 'ey', 'hx', 'hy'} (ntp, ny, nx)."""
        npulse = exc_ex_imag.shape[0]
        rec = {c: np.zeros((ntp, self.ny, self.nx), self.dtype) for c in ('ex', 'ey', 'hx', 'hy')}
        for t in range(ntp):
            self.e_update(self.ca, self.cb)
            self.e_cpml(self.cb)
            if t < npulse:
                self.ex[self.feed_in, 1:-1, 0:-1] = exc_ex_imag[t, 1:-1, 0:-1]
                self.ey[self.feed_in, 1:-1, 0:-1] = exc_ey_imag[t, 1:-1, 0:-1]
            self.h_update()
            self.h_cpml()
            for c in ('ex', 'ey', 'hx', 'hy'):
                rec[c][t] = getattr(self, c)[self.read_out]
            self.incident_phasors(t)
        return rec
