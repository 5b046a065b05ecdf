fdtd_incident *inc;
fdtd_geometry gi = g;                     /* nz = int(3 wl / dx), nt = size_t_inc, dte0dx = vacuum Cb */
fdtd_incident_create(&gi, size_t_pulse, 0, &inc);
fdtd_incident_set_absorbers(inc, profiles);
fdtd_incident_make_excitation(inc, k_vals, pulse_fft, size_t_inc, theta, phi, FDTD_POL_VV, radius, NULL);
fdtd_incident_run(inc);
fdtd_incident_get_planes(inc, ex, ey, hx, hy);   /* the incident file's datasets */
fdtd_set_incident_from(sim, inc);                 /* or hand them to a main simulation on the device */
fdtd_incident_destroy(inc);
