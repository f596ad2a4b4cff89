import numpy as np

from . import I, P, lib


def interpolate_wrap(x, y, B, ud, diag, ld, length, num_interp_params, num_modes, num_bin_all):
    lib().ref_interpolate(P(x, np.float64), P(y, np.float64), P(B, np.float64),
                          P(ud, np.float64), P(diag, np.float64), P(ld, np.float64), I(length),
                          I(num_interp_params), I(num_modes), I(num_bin_all))
