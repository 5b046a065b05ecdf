from fdtdsarsim_b200.gpu.main_sim import MainSimGpu
recipes = fdtd.materials.rough_dielectric(params, 3.2, 0.001, 0.004, 0.05, 0.05, 4, seed=7,
                                          device=True)   # LayeredMaterial recipes
MainSimGpu.device_postprocess = True    # near-field powers from the device's phasors
fdtd.run_experiment(params, recipes)    # each block is filled on the device
