from .materialmodel import MaterialModel
from .materials import compute_material_arrays, all_vacuum, flat_surface

__all__ = ['MaterialModel', 'compute_material_arrays', 'all_vacuum', 'flat_surface']
