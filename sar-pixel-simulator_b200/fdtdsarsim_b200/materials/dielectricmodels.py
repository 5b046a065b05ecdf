"""Complex permittivity of wet soil (materials/dielectricmodels.py).

The empirical model of M. Hallikainen, F. Ulaby, M. Dobson, M. El-Rayes and
L.-K. Wu, "Microwave dielectric behavior of wet soil - part 1: empirical
models and experimental observations", IEEE Trans. Geosci. Remote Sens.,
1985: at each of nine frequencies from 1.4 to 18 GHz,
eps' = a + b mv + c mv^2 and eps'' likewise, with a, b, c linear in the sand
and clay fractions (the paper's Table 2, reproduced below); between the
tabulated frequencies eps' and eps'' are interpolated linearly, and
eps = eps' - j eps''.
"""
import numpy as np

__all__ = ['HallikainenSoilModel', 'hallikainen_soil_model']

FREQ_TABLE = np.array([1.4, 4, 6, 8, 10, 12, 14, 16, 18]) * 1.0e9

# Table 2 of Hallikainen et al. (1985): per frequency (rows of FREQ_TABLE),
# the coefficients (constant, sand, clay) of a, b and c for eps' (_RE) and
# eps'' (_IM).
A_RE = np.array([[2.862, -0.012, 0.001], [2.927, -0.012, -0.001], [1.993, 0.002, 0.015],
                 [1.997, 0.002, 0.018], [2.502, -0.003, -0.003], [2.200, -0.001, 0.012],
                 [2.301, 0.001, 0.009], [2.237, 0.002, 0.009], [1.912, 0.007, 0.021]])
A_IM = np.array([[0.356, -0.003, -0.008], [0.004, 0.001, 0.002], [-0.123, 0.002, 0.003],
                 [-0.201, 0.003, 0.003], [-0.070, 0.000, 0.001], [-0.142, 0.001, 0.003],
                 [-0.096, 0.001, 0.002], [-0.027, -0.001, 0.003], [-0.071, 0.000, 0.003]])
B_RE = np.array([[3.803, 0.462, -0.341], [5.505, 0.371, 0.062], [38.086, -0.176, -0.633],
                 [25.579, -0.017, -0.412], [10.101, 0.221, -0.004], [26.473, 0.013, -0.523],
                 [17.918, 0.084, -0.282], [15.505, 0.076, -0.217], [29.123, -0.190, -0.545]])
B_IM = np.array([[5.507, 0.044, -0.002], [0.951, 0.005, -0.010], [7.502, -0.058, -0.116],
                 [11.266, -0.085, -0.155], [6.620, 0.015, -0.081], [11.868, -0.059, -0.225],
                 [8.583, -0.005, -0.153], [6.179, 0.074, -0.086], [6.938, 0.029, -0.128]])
C_RE = np.array([[119.006, -0.500, 0.633], [114.826, -0.389, -0.547], [10.720, 1.256, 1.522],
                 [39.793, 0.723, 0.941], [77.482, -0.061, -0.135], [34.333, 0.284, 1.062],
                 [50.149, 0.012, 0.387], [48.260, 0.168, 0.289], [6.960, 0.822, 1.195]])
C_IM = np.array([[17.753, -0.313, 0.206], [16.759, 0.192, 0.290], [2.942, 0.452, 0.543],
                 [0.194, 0.584, 0.581], [21.578, 0.293, 0.332], [7.817, 0.570, 0.801],
                 [28.707, 0.297, 0.357], [34.126, 0.143, 0.206], [29.945, 0.275, 0.377]])


def hallikainen_soil_model(mv, sand_frac, clay_frac, freq):
    """Complex relative permittivity of soil with volumetric moisture mv
    (0-1), sand and clay fractions (0-1) at ``freq`` [Hz], without range
    checks (the function form used inside the material fills)."""
    vec = np.array([1.0, sand_frac, clay_frac])
    re = [np.dot(t, vec) for t in (A_RE, B_RE, C_RE)]
    im = [np.dot(t, vec) for t in (A_IM, B_IM, C_IM)]
    eps_re = re[0] + (re[1] * mv) + (re[2] * (mv ** 2))
    eps_im = im[0] + (im[1] * mv) + (im[2] * (mv ** 2))
    return np.interp(freq, FREQ_TABLE, eps_re) - 1j * np.interp(freq, FREQ_TABLE, eps_im)


class HallikainenSoilModel:
    """The Hallikainen model with the range checks of the paper's validity
    (moisture and fractions in [0, 1], 1.4 to 18 GHz)."""

    freq_table = FREQ_TABLE
    a_coeff_re, a_coeff_im = A_RE, A_IM
    b_coeff_re, b_coeff_im = B_RE, B_IM
    c_coeff_re, c_coeff_im = C_RE, C_IM

    def get_epsilon(self, mv: float, sand_frac: float, clay_frac: float, freq: float):
        """Complex relative permittivity (eps' - j eps'')."""
        if mv < 0.0 or mv > 1.0:
            raise ValueError('Volumetric moisture out of bounds (0 < mv < 1)')
        if sand_frac < 0.0 or sand_frac > 1.0:
            raise ValueError('Sand fraction out of bounds (0 < sand_frac < 1')
        if clay_frac < 0.0 or clay_frac > 1.0:
            raise ValueError('Clay fraction out of bounds (0 < clay_frac < 1)')
        if freq < 1.4e9 or freq > 18.0e9:
            raise ValueError('Frequency out of bounds (1.4 GHz < freq < 18 GHz)')
        return hallikainen_soil_model(mv, sand_frac, clay_frac, freq)
