"""The float64 numpy adjoint (tests/adjoint_ref.py) against central finite
differences of the float64 forward oracle: d P_h / d eps_r and d P_h / d sigma
at material cells. This pins the CPU reference that the device adjoint is
checked against."""
import numpy as np

from adjoint_ref import AdjointRef, ca_cb_partials
from fdtdsarsim_b200.absorbers import cpml_profiles
from fdtdsarsim_b200.materials import MaterialModel, compute_material_arrays
from helpers import make_params


def _problem(seed=31, nt=40):
    pc = make_params(25, 23, 27, 14, nt, 30, dtype='float64')
    g = pc.geom_params
    rng = np.random.default_rng(seed)
    shape = (g.size_z_material, g.size_y, g.size_x)
    eps = rng.uniform(2.0, 12.0, size=shape)
    sig = rng.uniform(0.0, 0.1, size=shape)
    inc = {c: rng.standard_normal((g.size_t_inc, g.size_y, g.size_x)) * s
           for c, s in (('ex', 1.0), ('ey', 1.0), ('hx', 1 / 376.73), ('hy', 1 / 376.73))}
    ref = AdjointRef(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size, g.timestep,
                     pc.inc_beam_params.frequency, cpml_profiles(pc), theta_deg=-20.0, phi_deg=0.0)
    return pc, eps, sig, inc, ref


def _J(pc, ref, eps, sig, inc, nt):
    ca, cb = compute_material_arrays(pc, MaterialModel(eps, sig, pc.geom_params.cell_size))
    _, p = ref.forward(ca, cb, inc, nt)
    from adjoint_ref import objective_and_phasor_grad
    return objective_and_phasor_grad(p, ref.a, ref.b)[0]


def test_float64_adjoint_matches_central_differences():
    nt = 40
    pc, eps, sig, inc, ref = _problem(nt=nt)
    g = pc.geom_params
    ca, cb = compute_material_arrays(pc, MaterialModel(eps, sig, g.cell_size))
    J, gca, gcb = ref.grad(ca, cb, inc, nt)
    nzm = g.size_z_material
    dca_de, dca_ds, dcb_de, dcb_ds = ca_cb_partials(eps, sig, g.timestep, g.cell_size)
    ge = gca[:nzm] * dca_de + gcb[:nzm] * dcb_de
    gs = gca[:nzm] * dca_ds + gcb[:nzm] * dcb_ds
    rng = np.random.default_rng(5)
    # cells with a sensitivity well above round-off: the upper material layers
    cand = np.argwhere(np.abs(ge) > 1e-6 * np.abs(ge).max())
    picks = cand[rng.choice(len(cand), size=4, replace=False)]
    for z, y, x in picks:
        for which, base, grad in (('eps', eps, ge), ('sig', sig, gs)):
            h = 1e-3 * base[z, y, x] if base[z, y, x] != 0 else 1e-6
            plus, minus = base.copy(), base.copy()
            plus[z, y, x] += h
            minus[z, y, x] -= h
            if which == 'eps':
                fd = (_J(pc, ref, plus, sig, inc, nt) - _J(pc, ref, minus, sig, inc, nt)) / (2 * h)
            else:
                fd = (_J(pc, ref, eps, plus, inc, nt) - _J(pc, ref, eps, minus, inc, nt)) / (2 * h)
            # central-difference truncation (relative ~h^2) plus the round-off
            # of two float64 solves divided by 2h
            tol = 1e-4 * abs(fd) + 1e-14 * abs(J) / h
            assert abs(grad[z, y, x] - fd) <= tol, (which, z, y, x, grad[z, y, x], fd)
    # one directional derivative over every material cell (large signal)
    d_e = rng.standard_normal(eps.shape) * eps
    d_s = rng.standard_normal(sig.shape) * sig
    h = 1e-4
    fd = (_J(pc, ref, eps + h * d_e, sig + h * d_s, inc, nt)
          - _J(pc, ref, eps - h * d_e, sig - h * d_s, inc, nt)) / (2 * h)
    an = float(np.sum(ge * d_e) + np.sum(gs * d_s))
    assert abs(an - fd) <= 1e-6 * abs(fd), (an, fd)
