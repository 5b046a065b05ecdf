"""Device gradient (fdtd_grad_forward / fdtd_grad_backward and the
BackscatterGradient runner) against the float64 numpy adjoint, central
finite differences of device forward solves, across checkpoint periods and
between float32 and float64."""
import numpy as np
import pytest

from adjoint_ref import AdjointRef
from fdtdsarsim_b200 import _native
from fdtdsarsim_b200.absorbers import cpml_profiles
from fdtdsarsim_b200.adjoint import BackscatterGradient, backscatter_power
from fdtdsarsim_b200.materials import MaterialModel, compute_material_arrays
from helpers import make_params

pytestmark = pytest.mark.gpu


def _problem(dtype, nt=40, seed=31, dims=(25, 23, 27, 14)):
    nx, ny, nz, tfsf = dims
    pc = make_params(nx, ny, nz, tfsf, nt, 30, dtype=dtype)
    pc.inc_beam_params.polarization = 'HH'
    g = pc.geom_params
    rng = np.random.default_rng(seed)
    shape = (g.size_z_material, g.size_y, g.size_x)
    eps = rng.uniform(2.0, 12.0, size=shape)
    sig = rng.uniform(0.0, 0.1, size=shape)
    # a tapered plane wave: zero on the plane's edges like the reference's
    # beam (the adjoint holds the edge sub-systems, which such a beam never
    # drives, at zero)
    from fdtdsarsim_b200 import synthetic
    inc = synthetic.plane_wave_incident(pc, g.size_t_inc, dtype)
    return pc, eps, sig, inc


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize('kernel', [_native.FDTD_KERNEL_SPLIT, _native.FDTD_KERNEL_FUSED],
                         ids=['split', 'fused'])
def test_float64_device_adjoint_matches_numpy_adjoint(kernel):
    nt = 40
    pc, eps, sig, inc = _problem('float64', nt)
    g = pc.geom_params
    ref = AdjointRef(g.size_x, g.size_y, g.size_z, g.size_pml, g.tfsf_z, g.cell_size, g.timestep,
                     pc.inc_beam_params.frequency, cpml_profiles(pc), theta_deg=-20.0, phi_deg=0.0)
    ca, cb = compute_material_arrays(pc, MaterialModel(eps, sig, g.cell_size))
    J_ref, gca_ref, gcb_ref = ref.grad(ca, cb, inc, nt)
    run = BackscatterGradient(pc, inc, checkpoint_every=7, kernel=kernel)
    J, ge, gs = run.value_and_grad(eps, sig)
    assert abs(J - J_ref) <= 1e-10 * abs(J_ref)
    run.sim.grad_forward(7)
    p = run._upper_phasors()
    from fdtdsarsim_b200.adjoint import power_and_phasor_grad
    _, g_re, g_im = power_and_phasor_grad(p, run.a, run.b, run.sign)
    gca, gcb = run.sim.grad_backward(g_re, g_im, g.size_z)
    assert _rel(gca, gca_ref) < 1e-9
    assert _rel(gcb, gcb_ref) < 1e-9
    run.close()


def test_tuned_gradient_is_finite_and_matches_float64():
    """A longer solve with a tapered plane wave (stable excitation) on the
    kernel the autotuner picks: every gradient entry finite, float32 within
    1e-3 of float64."""
    from fdtdsarsim_b200 import synthetic, tuning
    from fdtdsarsim_b200.gpu.main_sim import native_geometry
    pc32, eps, sig, _ = _problem('float32', 300, seed=61, dims=(41, 39, 35, 18))
    pc64, _, _, _ = _problem('float64', 300, seed=61, dims=(41, 39, 35, 18))
    tuning.autotune(native_geometry(pc32), save=True)
    inc = synthetic.plane_wave_incident(pc32, pc32.geom_params.size_t_inc)
    r32 = BackscatterGradient(pc32, inc, checkpoint_every=64)
    r64 = BackscatterGradient(pc64, {k: v.astype(np.float64) for k, v in inc.items()},
                              checkpoint_every=64)
    J32, ge32, gs32 = r32.value_and_grad(eps, sig)
    J64, ge64, gs64 = r64.value_and_grad(eps, sig)
    assert np.isfinite(ge32).all() and np.isfinite(gs32).all()
    assert abs(J32 - J64) <= 1e-4 * abs(J64)
    assert _rel(ge32, ge64) < 1e-3
    assert _rel(gs32, gs64) < 1e-3
    r32.close()
    r64.close()


def test_checkpoint_period_does_not_change_the_gradient():
    pc, eps, sig, inc = _problem('float32', 40)
    out = []
    for every in (1, 7, 40, 64):
        run = BackscatterGradient(pc, inc, checkpoint_every=every)
        out.append(run.value_and_grad(eps, sig))
        run.close()
    for J, ge, gs in out[1:]:
        assert J == out[0][0]
        assert np.array_equal(ge, out[0][1]) and np.array_equal(gs, out[0][2])


def test_float32_gradient_close_to_float64():
    pc32, eps, sig, inc = _problem('float32', 60, seed=41)
    pc64, _, _, inc64 = _problem('float64', 60, seed=41)
    r32 = BackscatterGradient(pc32, inc, checkpoint_every=16)
    r64 = BackscatterGradient(pc64, {k: v.astype(np.float64) for k, v in inc.items()},
                              checkpoint_every=16)
    J32, ge32, gs32 = r32.value_and_grad(eps, sig)
    J64, ge64, gs64 = r64.value_and_grad(eps, sig)
    assert abs(J32 - J64) <= 1e-4 * abs(J64)
    assert _rel(ge32, ge64) < 1e-3
    assert _rel(gs32, gs64) < 1e-3
    r32.close()
    r64.close()


def test_gradient_matches_central_differences_on_device():
    """float64 device forward solves, step 1e-3 relative, at material cells
    with a sensitivity above round-off."""
    pc, eps, sig, inc = _problem('float64', 50, seed=51, dims=(31, 29, 33, 18))
    run = BackscatterGradient(pc, inc, checkpoint_every=8)
    J, ge, gs = run.value_and_grad(eps, sig)
    rng = np.random.default_rng(9)
    cand = np.argwhere(np.abs(ge) > 1e-3 * np.abs(ge).max())
    for z, y, x in cand[rng.choice(len(cand), size=6, replace=False)]:
        for base, grad, is_eps in ((eps, ge, True), (sig, gs, False)):
            h = 1e-3 * base[z, y, x]
            b1, b2 = base.copy(), base.copy()
            b1[z, y, x] += h
            b2[z, y, x] -= h
            if is_eps:
                fd = (run.value(b1, sig) - run.value(b2, sig)) / (2 * h)
            else:
                fd = (run.value(eps, b1) - run.value(eps, b2)) / (2 * h)
            tol = 1e-4 * abs(fd) + 1e-14 * abs(J) / h
            assert abs(grad[z, y, x] - fd) <= tol, (is_eps, z, y, x, grad[z, y, x], fd)
    run.close()


def test_autograd_function_returns_the_runner_gradient():
    import torch
    pc, eps, sig, inc = _problem('float32', 30)
    run = BackscatterGradient(pc, inc, checkpoint_every=10)
    J, ge, gs = run.value_and_grad(eps, sig)
    te = torch.tensor(eps, dtype=torch.float64, requires_grad=True)
    ts = torch.tensor(sig, dtype=torch.float64, requires_grad=True)
    P = backscatter_power(te, ts, run)
    (2.0 * P).backward()
    assert float(P.detach()) == J
    assert np.array_equal(te.grad.numpy(), 2.0 * ge)
    assert np.array_equal(ts.grad.numpy(), 2.0 * gs)
    run.close()
