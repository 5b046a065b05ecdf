int size_z_material = nz / 2;
float *inc_phasors;          /* ex, ey, hx, hy incident phasors: 4 x (ny_ph, nx_ph) complex */
double *weights, out11[11];  /* Simpson weights: ny_ph, nx_ph, size_z_material, nz_ph - 1 - size_z_material */
fdtd_near_field_power(sim, inc_phasors, size_z_material, weights, out11);
fdtd_set_option(sim, FDTD_OPT_SHELL, FDTD_SHELL_SPLIT);
if (fdtd_bounds_check_enabled()) { /* libfdtd_b200_check.so */ }
