fdtd_sim *sims[64];            /* each: create, set_absorbers, set_materials, set_incident */
fdtd_batch *b;
fdtd_batch_create(sims, 64, &b);
fdtd_batch_set_option(b, FDTD_OPT_GRAPH_CHUNK, 64);   /* steps per replayed CUDA graph */
fdtd_batch_set_option(b, FDTD_OPT_BATCH_MODE, FDTD_BATCH_SPLIT);  /* or _STREAMS, _QUEUE */
fdtd_batch_run(b, nt);          /* every member advances nt steps */
fdtd_batch_synchronize(b);
fdtd_get_phasor(sims[i], 4, out);                           /* per member, as before */
fdtd_batch_destroy(b);          /* members stay valid */
