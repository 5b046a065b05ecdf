"""The object every material generator yields (materials/materialmodel.py:10-29)."""
from dataclasses import dataclass

import numpy as np


@dataclass
class MaterialModel:
    """Relative permittivity and conductivity of the material block.

    Arrays are (size_z_material, size_y, size_x); vacuum is stacked on top
    up to size_z when the update coefficients are formed. ``name`` names the
    result file, ``metadata`` is stored with the results.
    """
    relative_permittivity: np.ndarray
    conductivity: np.ndarray
    cell_size: float
    name: str = 'results'
    metadata: dict = None
