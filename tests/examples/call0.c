#include "fdtd_b200.h"
fdtd_sim *sim;
fdtd_geometry g = {nx, ny, nz, 10, tfsf_z, nt, nt_inc, FDTD_F32,
                   dx, dt, 5.4e9, db, dtm0, dte0dx};
if (fdtd_create(&g, 0, &sim)) { char m[512]; fdtd_last_error(m, 512); /* ... */ }
fdtd_set_absorbers(sim, profiles);          /* 8 x npml floats */
fdtd_set_materials(sim, ca, cb);            /* (nz, ny, nx) */
fdtd_set_incident(sim, ex, ey, hx, hy, nt_inc);
fdtd_run(sim, nt);
fdtd_synchronize(sim);
fdtd_get_phasor(sim, 4, ex_ph_u);           /* complex (ny-20, nx-20) */
fdtd_get_phasors(sim, all24);               /* or all 24 planes packed, one call */
fdtd_destroy(sim);
