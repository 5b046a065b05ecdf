from fdtdsarsim_b200.adjoint import BackscatterGradient, backscatter_power
runner = BackscatterGradient(params, incident, checkpoint_every=64)   # incident: dict ex, ey, hx, hy
P, dP_deps, dP_dsigma = runner.value_and_grad(eps_r, sigma)           # numpy, material block shape
P = backscatter_power(eps_t, sigma_t, runner); P.backward()            # torch.autograd
