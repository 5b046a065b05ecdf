import sys; sys.path.insert(0, 'sar-pixel-simulator_b200')   # or install the folder
import fdtdsarsim_b200 as fdtd                                 # instead of fdtdsarsim

params = fdtd.load_from_json('params.json')   # "processing_type": "gpu"
materials = fdtd.materials.flat_surface(params, 6.0, 0.01)
fdtd.run_experiment(params, materials)        # results/<name>.hdf5 as before
