from .materialmodel import MaterialModel
from .materials import compute_material_arrays, all_vacuum, flat_surface, rough_dielectric
from .roughsurface import (gaussian_correlated_surface, gaussian_correlated_surface_fast,
                           two_layer_gaussian_correlated_surface, correlate_layers)
from .dielectricmodels import HallikainenSoilModel, hallikainen_soil_model
from . import bubbles, soilmodels

__all__ = ['MaterialModel', 'compute_material_arrays', 'all_vacuum', 'flat_surface',
           'rough_dielectric', 'gaussian_correlated_surface', 'gaussian_correlated_surface_fast',
           'two_layer_gaussian_correlated_surface', 'correlate_layers', 'HallikainenSoilModel',
           'hallikainen_soil_model', 'bubbles', 'soilmodels']
