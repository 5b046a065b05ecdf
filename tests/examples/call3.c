int nz_mat = nz / 2, nlayers = 2, n_spheres = 40;
double *heights, *eps_layers, *sig_layers, *spheres;   /* nlayers x (ny, nx); nlayers + 1; n x 5 */
float *eps_out, *sig_out;
fdtd_fill_layers(sim, nz_mat, nlayers, heights, eps_layers, sig_layers);  /* heights in cells, lowest first */
fdtd_paint_spheres(sim, n_spheres, spheres, 1.0, 0.0);                    /* (zc, yc, xc, rc, ri) in cells */
fdtd_set_materials_staged(sim);                                           /* Ca/Cb from the staged block */
fdtd_get_staged_materials(sim, nz_mat, eps_out, sig_out);                 /* optional: the block back on the host */
