"""Float64 numpy discrete adjoint of the FDTD step -- TEST INFRASTRUCTURE.

The reference has no gradient; this module is the CPU check for the
library's adjoint kernels. It differentiates exactly the forward step of
``oracle/fdtd_oracle.OracleSim`` (H update, H CPML, injection, E update,
E CPML, injection, phasors) run in float64, so that it can itself be checked
against central finite differences of that forward step.

Objective: the horizontal backscatter power P_h = 1/2 Re(-E_phi conj(H_theta))
(processresults.py:260-271) at one far-field direction (theta, phi), from
the near-to-far transform of the four upper-plane phasors
(near2far.py:28-156). E_phi and H_theta are linear in those phasors, so the
objective's gradient with respect to the real and imaginary part of each
phasor cell is exact; the running DFT then turns it into a source term on
the upper phasor plane at every step, and the transposed step carries it
back in time. The gradient with respect to Ca and Cb is accumulated on the
way and mapped to eps_r and sigma by the closed form of
``compute_material_arrays`` (materials/materials.py:23-68).
"""
import numpy as np

import fdtd_oracle as O

EPS0_MAT = 8.8541878128e-12   # the constant the reference's material code uses
ETA0 = 376.730313668
C0 = 299792458


def near2far_coefficients(nx_ph, ny_ph, nz_ph, dx, r, theta_deg, phi_deg, freq):
    """Complex coefficient planes (a, b) with E_phi = sum a . p and
    H_theta = sum b . p for p = (ex_u, ey_u, hx_u, hy_u) stacked on axis 0,
    matching oracle.near2far for one direction."""
    lam = C0 / freq
    k = 2.0 * np.pi / lam
    t_, p_ = np.deg2rad(theta_deg), np.deg2rad(phi_deg)
    x_loc = np.arange(-(nx_ph - 1) // 2, ((nx_ph - 1) // 2) + 1) * dx
    y_loc = np.arange(-(ny_ph - 1) // 2, ((ny_ph - 1) // 2) + 1) * dx
    z_val = ((nz_ph - 1) // 2) * dx
    xx, yy = np.meshgrid(x_loc, y_loc)
    e = np.exp(1j * k * (xx * np.sin(t_) * np.cos(p_) + yy * np.sin(t_) * np.sin(p_)
                         + z_val * np.cos(t_)))
    w = np.outer(O.simpson_weights(ny_ph, dx), O.simpson_weights(nx_ph, dx)) * e
    ct, cp, sp = np.cos(t_), np.cos(p_), np.sin(p_)
    ffw = 1j * k * np.exp(-1j * k * r) / (4.0 * np.pi * r)
    # J = (-hy, hx), M = (ey, -ex)
    # Np = sum w (-Jx sp + Jy cp) = sum w (hy sp + hx cp)
    # Lt = sum w (Mx ct cp + My ct sp) = sum w (ey ct cp - ex ct sp)
    zero = np.zeros_like(w)
    dNp = np.stack([zero, zero, w * cp, w * sp])
    dLt = np.stack([-w * ct * sp, w * ct * cp, zero, zero])
    a = ffw * (dLt - ETA0 * dNp)           # E_phi = ffw (Lt - eta0 Np)
    b = ffw * (dNp - dLt / ETA0)           # H_theta = ffw (Np - Lt / eta0)
    return a, b


def objective_and_phasor_grad(p, a, b):
    """P_h and (dJ/dRe p, dJ/dIm p) for p stacked (4, ny_ph, nx_ph)."""
    u = np.sum(a * p)
    v = np.sum(b * p)
    J = 0.5 * np.real(-u * np.conj(v))
    g_re = -0.5 * np.real(a * np.conj(v) + b * np.conj(u))
    g_im = -0.5 * (np.imag(np.conj(a) * v) + np.imag(np.conj(b) * u))
    return J, g_re, g_im


def ca_cb_partials(eps, sig, dt, dx):
    """dCa/deps, dCa/dsig, dCb/deps, dCb/dsig of compute_material_arrays."""
    perm = eps * EPS0_MAT
    x = sig * dt / (2.0 * perm)
    dx_deps = -x / eps
    dx_dsig = dt / (2.0 * perm)
    dca_dx = -2.0 / (1.0 + x) ** 2
    cb0 = dt / (perm * dx)
    dcb_deps = -cb0 / eps / (1.0 + x) - cb0 / (1.0 + x) ** 2 * dx_deps
    dcb_dsig = -cb0 / (1.0 + x) ** 2 * dx_dsig
    return dca_dx * dx_deps, dca_dx * dx_dsig, dcb_deps, dcb_dsig


class AdjointRef:
    """Float64 forward (the oracle) with stored states, then the transposed
    sweep. ``grad(ca, cb, inc, nt)`` returns (J, dJ/dCa, dJ/dCb)."""

    def __init__(self, nx, ny, nz, npml, tfsf_z, dx, dt, freq, profiles, theta_deg, phi_deg,
                 r=2000.0):
        self.sim = O.OracleSim(nx, ny, nz, npml, tfsf_z, dx, dt, freq, 'float64', profiles)
        s = self.sim
        self.a, self.b = near2far_coefficients(s.nx_ph, s.ny_ph, s.nz_ph, dx, r, theta_deg,
                                               phi_deg, freq)

    def _state(self):
        s = self.sim
        st = {c: getattr(s, c).copy() for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')}
        st['psi'] = {k: v.copy() for k, v in s.psi.items()}
        return st

    def forward(self, ca, cb, inc, nt):
        s = self.sim
        s.reset()
        states = [self._state()]
        for _ in range(nt):
            s.step(ca, cb, inc)
            states.append(self._state())
        p = np.stack([s.ph['ex_ph_u'], s.ph['ey_ph_u'], s.ph['hx_ph_u'], s.ph['hy_ph_u']])
        return states, p

    def grad(self, ca, cb, inc, nt):
        s = self.sim
        states, p = self.forward(ca, cb, inc, nt)
        J, g_re, g_im = objective_and_phasor_grad(p, self.a, self.b)
        nx, ny, nz, m = s.nx, s.ny, s.nz, s.npml
        lam = {c: np.zeros((nz, ny, nx)) for c in ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')}
        lpsi = {k: np.zeros_like(v) for k, v in s.psi.items()}
        gca = np.zeros((nz, ny, nx))
        gcb = np.zeros((nz, ny, nx))
        for n in range(nt - 1, -1, -1):
            old, new = states[n], states[n + 1]
            cE, sE, cH, sH = O.phase_factors(s.omega, n, s.dt)
            self._phasor_sources(lam, g_re, g_im, cE, sE, cH, sH, e_part=True)
            self._e_cpml_T(lam, lpsi, gcb, cb, new)
            self._e_update_T(lam, gca, gcb, ca, cb, old, new)
            self._phasor_sources(lam, g_re, g_im, cE, sE, cH, sH, e_part=False)
            self._h_cpml_T(lam, lpsi)
            self._h_update_T(lam)
        return J, gca, gcb

    # -- phasor sources: p += avg(field) (c + i s) on the upper plane -------
    def _phasor_sources(self, lam, g_re, g_im, cE, sE, cH, sH, e_part):
        s = self.sim
        m = s.npml
        pz = s.nz - m - 1
        Y = np.s_[m + 1:m + s.ny_ph]
        Yd = np.s_[m:m + s.ny_ph - 1]
        X = np.s_[m + 1:m + s.nx_ph]
        Xd = np.s_[m:m + s.nx_ph - 1]
        if e_part:
            g = g_re * cE + g_im * sE
            gx, gy = g[0][1:, 1:], g[1][1:, 1:]
            lam['ex'][pz, Y, X] += 0.5 * gx
            lam['ex'][pz, Y, Xd] += 0.5 * gx
            lam['ey'][pz, Y, X] += 0.5 * gy
            lam['ey'][pz, Yd, X] += 0.5 * gy
        else:
            g = g_re * cH + g_im * sH
            gx, gy = g[2][1:, 1:], g[3][1:, 1:]
            for zz in (pz, pz - 1):
                lam['hx'][zz, Y, X] += 0.25 * gx
                lam['hx'][zz, Yd, X] += 0.25 * gx
                lam['hy'][zz, Y, X] += 0.25 * gy
                lam['hy'][zz, Y, Xd] += 0.25 * gy

    # -- E CPML transposed (faces commute) ------------------------------------
    def _e_cpml_T(self, lam, lpsi, gcb, cb, new):
        s = self.sim
        nx, ny, nz, m, dx = s.nx, s.ny, s.nz, s.npml, float(s.dxf)
        p = s.p
        le, lh = lam, lam
        P1 = new['psi']
        for side, q0, z0 in (('d', 1, 1), ('u', 0, nz - m)):
            b = p['be_' + side][q0:q0 + m - 1, None, None]
            c = p['ce_' + side][q0:q0 + m - 1, None, None]
            f = np.s_[z0:z0 + m - 1, 0:ny - 1, 0:nx - 1]
            fd = np.s_[z0 - 1:z0 + m - 2, 0:ny - 1, 0:nx - 1]
            q = np.s_[q0:q0 + m - 1, 0:ny - 1, 0:nx - 1]
            for name, comp, sign, hcomp in (('Eyz', 'ey', 1.0, 'hx'), ('Exz', 'ex', -1.0, 'hy')):
                tot = lpsi[name + side][q] + sign * cb[f] * dx * le[comp][f]
                gcb[f] += sign * dx * P1[name + side][q] * le[comp][f]
                lh[hcomp][f] += c / dx * tot
                lh[hcomp][fd] -= c / dx * tot
                lpsi[name + side][q] = b * tot
        for side, q0, x0, pk in (('l', 1, 1, 'd'), ('r', 0, nx - m, 'u')):
            b = p['be_' + pk][None, None, q0:q0 + m - 1]
            c = p['ce_' + pk][None, None, q0:q0 + m - 1]
            f = np.s_[0:nz - 1, 0:ny - 1, x0:x0 + m - 1]
            fl = np.s_[0:nz - 1, 0:ny - 1, x0 - 1:x0 + m - 2]
            q = np.s_[0:nz - 1, 0:ny - 1, q0:q0 + m - 1]
            for name, comp, sign, hcomp in (('Ezx', 'ez', 1.0, 'hy'), ('Eyx', 'ey', -1.0, 'hz')):
                tot = lpsi[name + side][q] + sign * cb[f] * dx * le[comp][f]
                gcb[f] += sign * dx * P1[name + side][q] * le[comp][f]
                lh[hcomp][f] += c / dx * tot
                lh[hcomp][fl] -= c / dx * tot
                lpsi[name + side][q] = b * tot
        for side, q0, y0, pk in (('f', 1, 1, 'd'), ('b', 0, ny - m, 'u')):
            b = p['be_' + pk][None, q0:q0 + m - 1, None]
            c = p['ce_' + pk][None, q0:q0 + m - 1, None]
            f = np.s_[0:nz - 1, y0:y0 + m - 1, 0:nx - 1]
            ff = np.s_[0:nz - 1, y0 - 1:y0 + m - 2, 0:nx - 1]
            q = np.s_[0:nz - 1, q0:q0 + m - 1, 0:nx - 1]
            for name, comp, sign, hcomp in (('Exy', 'ex', 1.0, 'hz'), ('Ezy', 'ez', -1.0, 'hx')):
                tot = lpsi[name + side][q] + sign * cb[f] * dx * le[comp][f]
                gcb[f] += sign * dx * P1[name + side][q] * le[comp][f]
                lh[hcomp][f] += c / dx * tot
                lh[hcomp][ff] -= c / dx * tot
                lpsi[name + side][q] = b * tot

    # -- E main update transposed ---------------------------------------------
    def _e_update_T(self, lam, gca, gcb, ca, cb, old, new):
        s = self.sim
        nx, ny, nz = s.nx, s.ny, s.nz
        hx, hy, hz = new['hx'], new['hy'], new['hz']
        # ex[s] = ca ex + cb ((hz - hz(y-1)) - (hy - hy(z-1)))
        sl = np.s_[1:nz - 1, 1:ny - 1, 0:nx - 1]
        g = lam['ex'][sl].copy()
        gca[sl] += g * old['ex'][sl]
        gcb[sl] += g * ((hz[sl] - hz[1:nz - 1, 0:ny - 2, 0:nx - 1]) - (hy[sl] - hy[0:nz - 2, 1:ny - 1, 0:nx - 1]))
        f = cb[sl] * g
        lam['hz'][sl] += f
        lam['hz'][1:nz - 1, 0:ny - 2, 0:nx - 1] -= f
        lam['hy'][sl] -= f
        lam['hy'][0:nz - 2, 1:ny - 1, 0:nx - 1] += f
        lam['ex'][sl] = ca[sl] * g
        # ey[s] = ca ey + cb ((hx - hx(z-1)) - (hz - hz(x-1)))
        sl = np.s_[1:nz - 1, 0:ny - 1, 1:nx - 1]
        g = lam['ey'][sl].copy()
        gca[sl] += g * old['ey'][sl]
        gcb[sl] += g * ((hx[sl] - hx[0:nz - 2, 0:ny - 1, 1:nx - 1]) - (hz[sl] - hz[1:nz - 1, 0:ny - 1, 0:nx - 2]))
        f = cb[sl] * g
        lam['hx'][sl] += f
        lam['hx'][0:nz - 2, 0:ny - 1, 1:nx - 1] -= f
        lam['hz'][sl] -= f
        lam['hz'][1:nz - 1, 0:ny - 1, 0:nx - 2] += f
        lam['ey'][sl] = ca[sl] * g
        # ez[s] = ca ez + cb ((hy - hy(x-1)) - (hx - hx(y-1)))
        sl = np.s_[0:nz - 1, 1:ny - 1, 1:nx - 1]
        g = lam['ez'][sl].copy()
        gca[sl] += g * old['ez'][sl]
        gcb[sl] += g * ((hy[sl] - hy[0:nz - 1, 1:ny - 1, 0:nx - 2]) - (hx[sl] - hx[0:nz - 1, 0:ny - 2, 1:nx - 1]))
        f = cb[sl] * g
        lam['hy'][sl] += f
        lam['hy'][0:nz - 1, 1:ny - 1, 0:nx - 2] -= f
        lam['hx'][sl] -= f
        lam['hx'][0:nz - 1, 0:ny - 2, 1:nx - 1] += f
        lam['ez'][sl] = ca[sl] * g

    # -- H CPML transposed ------------------------------------------------------
    def _h_cpml_T(self, lam, lpsi):
        s = self.sim
        nx, ny, nz, m, dx, dtm0 = s.nx, s.ny, s.nz, s.npml, float(s.dxf), float(s.dtm0)
        p = s.p
        for side, z0 in (('d', 0), ('u', nz - m)):
            b = p['bh_' + side][0:m - 1, None, None]
            c = p['ch_' + side][0:m - 1, None, None]
            f = np.s_[z0:z0 + m - 1, 0:ny - 1, 0:nx - 1]
            fu = np.s_[z0 + 1:z0 + m, 0:ny - 1, 0:nx - 1]
            q = np.s_[0:m - 1, 0:ny - 1, 0:nx - 1]
            for name, hcomp, sign, ecomp in (('Hyz', 'hy', -1.0, 'ex'), ('Hxz', 'hx', 1.0, 'ey')):
                tot = lpsi[name + side][q] + sign * dtm0 * lam[hcomp][f]
                lam[ecomp][fu] += c / dx * tot
                lam[ecomp][f] -= c / dx * tot
                lpsi[name + side][q] = b * tot
        for side, x0, pk in (('l', 0, 'd'), ('r', nx - m, 'u')):
            b = p['bh_' + pk][None, None, 0:m - 1]
            c = p['ch_' + pk][None, None, 0:m - 1]
            f = np.s_[0:nz - 1, 0:ny - 1, x0:x0 + m - 1]
            fr = np.s_[0:nz - 1, 0:ny - 1, x0 + 1:x0 + m]
            q = np.s_[0:nz - 1, 0:ny - 1, 0:m - 1]
            for name, hcomp, sign, ecomp in (('Hzx', 'hz', -1.0, 'ey'), ('Hyx', 'hy', 1.0, 'ez')):
                tot = lpsi[name + side][q] + sign * dtm0 * lam[hcomp][f]
                lam[ecomp][fr] += c / dx * tot
                lam[ecomp][f] -= c / dx * tot
                lpsi[name + side][q] = b * tot
        for side, y0, pk in (('f', 0, 'd'), ('b', ny - m, 'u')):
            b = p['bh_' + pk][None, 0:m - 1, None]
            c = p['ch_' + pk][None, 0:m - 1, None]
            f = np.s_[0:nz - 1, y0:y0 + m - 1, 0:nx - 1]
            fb = np.s_[0:nz - 1, y0 + 1:y0 + m, 0:nx - 1]
            q = np.s_[0:nz - 1, 0:m - 1, 0:nx - 1]
            for name, hcomp, sign, ecomp in (('Hxy', 'hx', -1.0, 'ez'), ('Hzy', 'hz', 1.0, 'ex')):
                tot = lpsi[name + side][q] + sign * dtm0 * lam[hcomp][f]
                lam[ecomp][fb] += c / dx * tot
                lam[ecomp][f] -= c / dx * tot
                lpsi[name + side][q] = b * tot

    # -- H main update transposed -------------------------------------------------
    def _h_update_T(self, lam):
        s = self.sim
        nx, ny, nz, Db = s.nx, s.ny, s.nz, float(s.Db)
        # hx[s] -= Db ((ez(y+1) - ez) - (ey(z+1) - ey))
        sl = np.s_[0:nz - 1, 0:ny - 1, 1:nx - 1]
        g = Db * lam['hx'][sl]
        lam['ez'][0:nz - 1, 1:ny, 1:nx - 1] -= g
        lam['ez'][sl] += g
        lam['ey'][1:nz, 0:ny - 1, 1:nx - 1] += g
        lam['ey'][sl] -= g
        # hy[s] -= Db ((ex(z+1) - ex) - (ez(x+1) - ez))
        sl = np.s_[0:nz - 1, 1:ny - 1, 0:nx - 1]
        g = Db * lam['hy'][sl]
        lam['ex'][1:nz, 1:ny - 1, 0:nx - 1] -= g
        lam['ex'][sl] += g
        lam['ez'][0:nz - 1, 1:ny - 1, 1:nx] += g
        lam['ez'][sl] -= g
        # hz[s] -= Db ((ey(x+1) - ey) - (ex(y+1) - ex))
        sl = np.s_[1:nz - 1, 0:ny - 1, 0:nx - 1]
        g = Db * lam['hz'][sl]
        lam['ey'][1:nz - 1, 0:ny - 1, 1:nx] -= g
        lam['ey'][sl] += g
        lam['ex'][1:nz - 1, 1:ny, 0:nx - 1] += g
        lam['ex'][sl] -= g
