"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference ships material generators (rough surfaces, bubbles, soil
models) that are not part of the time-stepping path; these are small,
self-contained stand-ins that produce material blocks with the sizes and
value distributions the benchmark configurations name:

  plain_2x2      2x2 wl, 0.5 wl deep, cell 0.05 wl, flat soil eps 6 / 0.01 S/m
  plain_8x8      8x8 wl, 1.5 wl deep, cell 0.021 wl, rough soil (rms 0.1 wl,
                 corr 0.5 wl), eps_r lognormal (median 8, 5 %), 0.02 S/m
  plain_16x16    16x16 wl, 3 wl deep, cell 0.021 wl, VV: 1.5 wl snowpack of
                 ice spheres (eps 3.15, r 1-3 cells, volume fraction 0.3) over
                 soil (eps 10, 0.05 S/m) with a rough interface (rms 0.05 wl,
                 corr 0.4 wl)
  adjoint_4x4    4x4 wl, 1 wl deep, cell 0.03 wl, rough soil (rms 0.05 wl,
                 corr 0.5 wl), eps_r U(5,12), sigma U(0.005, 0.05) per cell
  batch_model    one of the 64 uneven vegetation models: x-y U(2,8) wl,
                 depth U(0.5,2) wl, cell 0.03 wl, dielectric cylinders
                 (eps 20, 0.3 S/m, r 1-2 cells, length 5-20 cells,
                 0.02 per cubic wl) over flat soil (eps 8, 0.02 S/m)
"""
import numpy as np
import scipy.constants

from .materials.materialmodel import MaterialModel
from .parameters import ParameterCollection, set_geom_params

FREQ = 5.4e9
LAM = scipy.constants.c / FREQ


def base_params(dtype='float32', project_dir='', pol='HH', theta=20.0, mf=0.7,
                sim_duration=18.0, inc_duration=10.0, illum=None):
    pc = ParameterCollection()
    p = pc.processing_params
    p.processing_type = 'gpu'
    p.datatype = dtype
    p.project_dir = project_dir
    b = pc.inc_beam_params
    b.frequency = FREQ
    b.polarization = pol
    b.theta_angle = theta
    b.phi_angle = 0.0
    b.duration = inc_duration
    b.illumination_width = illum if illum is not None else 0.0
    pc.material_params.material_fraction = mf
    pc.geom_params.simulation_duration = sim_duration
    return pc


def config_params(name, dtype='float32', project_dir='', **kw):
    """ParameterCollection of a named benchmark geometry."""
    table = {
        # size_x, size_y, depth, cell (all in wavelengths), pol, mf
        'plain_2x2': (2.0, 2.0, 0.5, 0.05, 'HH', 0.3),
        'plain_8x8': (8.0, 8.0, 1.5, 0.021, 'HH', 0.7),
        'plain_16x16': (16.0, 16.0, 3.0, 0.021, 'VV', 0.7),
        'adjoint_4x4': (4.0, 4.0, 1.0, 0.03, 'HH', 0.6),
    }
    sx, sy, depth, cell, pol, mf = table[name]
    pc = base_params(dtype, project_dir, pol=kw.get('pol', pol), mf=kw.get('mf', mf),
                     illum=kw.get('illum', sx))
    set_geom_params(pc, sx, sy, depth, pc.geom_params.simulation_duration, cell, 'wavelength')
    return pc


def gaussian_surface(nx, ny, dx, corr_len, rms, rng):
    """Height field (ny, nx) [m] with Gaussian autocorrelation: white noise
    filtered in the Fourier domain by a Gaussian of correlation length
    ``corr_len`` [m], rescaled to zero mean and rms ``rms`` [m]."""
    kx = 2 * np.pi * np.fft.fftfreq(nx, dx)
    ky = 2 * np.pi * np.fft.fftfreq(ny, dx)
    k2 = ky[:, None] ** 2 + kx[None, :] ** 2
    filt = np.exp(-k2 * corr_len ** 2 / 8.0)
    noise = rng.standard_normal((ny, nx))
    h = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    h -= h.mean()
    std = h.std()
    return h * (rms / std) if std > 0 else h


def _fill_below(eps, sig, height_cells, e_val, s_val):
    nz = eps.shape[0]
    zc = np.arange(nz)[:, None, None]
    mask = zc <= height_cells[None, :, :]
    eps[mask] = e_val
    sig[mask] = s_val
    return mask


def flat_soil(pc, eps_r=6.0, sigma=0.01):
    g = pc.geom_params
    dt = pc.processing_params.datatype
    shape = (g.size_z_material, g.size_y, g.size_x)
    return MaterialModel(np.full(shape, eps_r, dt), np.full(shape, sigma, dt), g.cell_size,
                         'flat_soil', {'epsilon_r': eps_r, 'conductivity': sigma})


def rough_lognormal_soil(pc, rng, rms_wl=0.1, corr_wl=0.5, median=8.0, spread=0.05,
                         sigma=0.02, name='rough_soil'):
    g = pc.geom_params
    dt = pc.processing_params.datatype
    nz, ny, nx = g.size_z_material, g.size_y, g.size_x
    dx = g.cell_size
    h = gaussian_surface(nx, ny, dx, corr_wl * LAM, rms_wl * LAM, rng) / dx
    h += nz - 1 - 3.0 * rms_wl * LAM / dx
    eps = np.ones((nz, ny, nx), dt)
    sig = np.zeros((nz, ny, nx), dt)
    mask = _fill_below(eps, sig, h, 1.0, sigma)
    ln = rng.normal(np.log(median), spread, size=(nz, ny, nx)).astype(np.float64)
    eps[mask] = np.exp(ln[mask]).astype(dt)
    return MaterialModel(eps, sig, dx, name, {'median_eps': median, 'sigma': sigma})


def _paint_spheres(eps, sig, fraction, rmin, rmax, e_val, s_val, z0, z1, rng):
    """Random balls (radius U(rmin, rmax) cells) in the slab z0 <= z < z1
    until the slab's painted fraction reaches ``fraction``."""
    nz, ny, nx = eps.shape
    slab = (z1 - z0) * ny * nx
    painted = np.zeros(eps.shape, bool)
    count = 0
    offs = {}
    for r in range(int(np.floor(rmin)), int(np.ceil(rmax)) + 1):
        rr = np.arange(-r, r + 1)
        zz, yy, xx = np.meshgrid(rr, rr, rr, indexing='ij')
        offs[r] = (zz, yy, xx, zz ** 2 + yy ** 2 + xx ** 2)
    while count < fraction * slab:
        n = max(64, int((fraction * slab - count) / 20))
        rad = rng.uniform(rmin, rmax, n)
        cz = rng.integers(z0, z1, n)
        cy = rng.integers(0, ny, n)
        cx = rng.integers(0, nx, n)
        for r_int in offs:
            sel = np.nonzero(np.ceil(rad).astype(int) == r_int)[0]
            if sel.size == 0:
                continue
            zz, yy, xx, d2 = offs[r_int]
            inside = d2[None] <= (rad[sel] ** 2)[:, None, None, None]
            Z = (cz[sel][:, None, None, None] + zz[None])
            Y = (cy[sel][:, None, None, None] + yy[None]) % ny
            X = (cx[sel][:, None, None, None] + xx[None]) % nx
            ok = inside & (Z >= z0) & (Z < z1)
            painted[Z[ok], Y[ok], X[ok]] = True
        count = int(painted[z0:z1].sum())
    eps[painted] = e_val
    sig[painted] = s_val
    return count / slab


def snowpack_over_rough_soil(pc, rng, name='snowpack'):
    g = pc.geom_params
    dt = pc.processing_params.datatype
    nz, ny, nx = g.size_z_material, g.size_y, g.size_x
    dx = g.cell_size
    eps = np.ones((nz, ny, nx), dt)
    sig = np.zeros((nz, ny, nx), dt)
    soil_top = nz // 2
    h = gaussian_surface(nx, ny, dx, 0.4 * LAM, 0.05 * LAM, rng) / dx + soil_top
    _fill_below(eps, sig, h, 10.0, 0.05)
    frac = _paint_spheres(eps, sig, 0.3, 1.0, 3.0, 3.15, 0.0, soil_top + 3, nz, rng)
    return MaterialModel(eps, sig, dx, name, {'ice_fraction': frac})


def uniform_rough_soil(pc, rng, name='adjoint_soil'):
    g = pc.geom_params
    dt = pc.processing_params.datatype
    nz, ny, nx = g.size_z_material, g.size_y, g.size_x
    dx = g.cell_size
    h = gaussian_surface(nx, ny, dx, 0.5 * LAM, 0.05 * LAM, rng) / dx + (nz - 1 - 3)
    eps = np.ones((nz, ny, nx), dt)
    sig = np.zeros((nz, ny, nx), dt)
    mask = _fill_below(eps, sig, h, 1.0, 0.0)
    eps[mask] = rng.uniform(5.0, 12.0, size=int(mask.sum())).astype(dt)
    sig[mask] = rng.uniform(0.005, 0.05, size=int(mask.sum())).astype(dt)
    return MaterialModel(eps, sig, dx, name, {})


def vegetation_model(pc, rng, name='veg'):
    """Flat soil (lower third) under randomly oriented dielectric cylinders."""
    g = pc.geom_params
    dt = pc.processing_params.datatype
    nz, ny, nx = g.size_z_material, g.size_y, g.size_x
    dx = g.cell_size
    eps = np.ones((nz, ny, nx), dt)
    sig = np.zeros((nz, ny, nx), dt)
    soil = max(1, nz // 3)
    eps[:soil] = 8.0
    sig[:soil] = 0.02
    vol_wl3 = (nz - soil) * ny * nx * (dx / LAM) ** 3
    n_cyl = rng.poisson(0.02 * vol_wl3)
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing='ij')
    for _ in range(n_cyl):
        r = rng.uniform(1.0, 2.0)
        length = rng.uniform(5.0, 20.0)
        c = np.array([rng.uniform(soil, nz), rng.uniform(0, ny), rng.uniform(0, nx)])
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        half = length / 2 + r
        lo = np.maximum(np.floor(c - half).astype(int), 0)
        hi = np.minimum(np.ceil(c + half).astype(int) + 1, [nz, ny, nx])
        sl = tuple(slice(a, b) for a, b in zip(lo, hi))
        d = np.stack([zz[sl] - c[0], yy[sl] - c[1], xx[sl] - c[2]], axis=-1)
        along = d @ v
        perp2 = np.sum(d * d, axis=-1) - along ** 2
        m = (np.abs(along) <= length / 2) & (perp2 <= r * r)
        eps[sl][m] = 20.0
        sig[sl][m] = 0.3
    return MaterialModel(eps, sig, dx, name, {'n_cylinders': int(n_cyl)})


def plane_wave_incident(pc, nt_planes, dtype=None):
    """Incident planes (nt_planes, ny, nx) 'ex', 'ey', 'hx', 'hy' of a
    tapered plane wave at the geometry's frequency, polarisation and theta
    (phi 0), the kind of excitation the reference's incident beam provides
    (incidentbeam.py:174-433): a carrier sin(2 pi f (t - x sin(theta) / c))
    that ramps up over three periods (raised cosine) and down over the last
    three periods of size_t_inc, times a Gaussian taper across the plane
    (1/e radius 0.4 of each side). H = E / eta0 along the wave's direction.

    Like the reference's beam (whose own Yee ranges leave them at zero),
    ey and hx vanish on the x edges and ex and hy on the y edges of the
    plane. That matters for long runs: on those edges the update applies
    only CPML corrections (no curl update), and that sub-system grows
    exponentially once it is driven; white-noise planes drive it within a
    few hundred steps, with the reference's update as with this one."""
    g = pc.geom_params
    b = pc.inc_beam_params
    dt = pc.processing_params.datatype if dtype is None else dtype
    f = b.frequency
    c = 299792458.0
    eta0 = 376.730313668
    th = np.deg2rad(b.theta_angle)
    dt_ = np.dtype(dt)
    x = (np.arange(g.size_x) - (g.size_x - 1) / 2.0) * g.cell_size
    y = (np.arange(g.size_y) - (g.size_y - 1) / 2.0) * g.cell_size
    t = np.arange(nt_planes) * g.timestep
    tau = t[:, None] - x[None, :] * np.sin(th) / c                       # (nt, nx)
    period = 1.0 / f
    t_end = g.size_t_inc * g.timestep
    ramp = np.clip(tau / (3 * period), 0.0, 1.0)
    ramp = 0.5 * (1.0 - np.cos(np.pi * ramp))
    fall = np.clip((t_end - tau) / (3 * period), 0.0, 1.0)
    fall = 0.5 * (1.0 - np.cos(np.pi * fall))
    carrier = (np.sin(2.0 * np.pi * f * tau) * ramp * fall).astype(dt_)   # (nt, nx)
    wx = 0.4 * g.size_x * g.cell_size
    wy = 0.4 * g.size_y * g.cell_size
    taper = np.exp(-(y[:, None] / wy) ** 2 - (x[None, :] / wx) ** 2).astype(dt_)   # (ny, nx)
    e = (carrier[:, None, :] * taper[None, :, :]).astype(dt)
    zero = np.zeros_like(e)
    if str(b.polarization).upper() == 'VV':
        # E in the plane of incidence (x), H along y
        out = {'ex': (e * np.cos(th)).astype(dt), 'ey': zero,
               'hx': zero, 'hy': (e / eta0).astype(dt)}
    else:
        # HH: E along y, H in the plane of incidence
        out = {'ex': zero, 'ey': e, 'hx': (-e * np.cos(th) / eta0).astype(dt), 'hy': zero}
    for k in ('ey', 'hx'):
        out[k] = out[k].copy()
        out[k][:, :, 0] = 0
        out[k][:, :, -1] = 0
    for k in ('ex', 'hy'):
        out[k] = out[k].copy()
        out[k][:, 0, :] = 0
        out[k][:, -1, :] = 0
    return out
