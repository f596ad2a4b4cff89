import ctypes

import numpy as np

from . import D, I, P, lib


class pyFastLISAResponse:
    def __init__(self):
        lib().ref_response_create.restype = ctypes.c_void_p
        self._h = ctypes.c_void_p(lib().ref_response_create())
        self._keep = None

    def add_orbit_information(self, dt, N, n_arr, L_arr, x_arr, links, sc_r, sc_e, armlength):
        self._keep = [np.ascontiguousarray(a) for a in (n_arr, L_arr, x_arr, links, sc_r, sc_e)]
        n_arr, L_arr, x_arr, links, sc_r, sc_e = self._keep
        lib().ref_response_add_orbit_information(
            self._h, D(dt), I(N), P(n_arr, np.float64), P(L_arr, np.float64),
            P(x_arr, np.float64), P(links, np.int32), P(sc_r, np.int32), P(sc_e, np.int32),
            D(armlength))

    def LISA_response_wrap(self, buf, ells, mms, freqs, phi_ref, inc, lam, beta, psi, TDItag,
                           rescaled, tdi2, order_fresnel_stencil, num_modes, length, num_bin_all,
                           includes_amps):
        lib().ref_LISA_response(
            self._h, P(buf, np.float64), P(ells, np.int32), P(mms, np.int32),
            P(freqs, np.float64), P(phi_ref, np.float64), P(inc, np.float64),
            P(lam, np.float64), P(beta, np.float64), P(psi, np.float64), I(TDItag),
            I(int(rescaled)), I(int(tdi2)), I(order_fresnel_stencil), I(num_modes), I(length),
            I(num_bin_all), I(int(includes_amps)))

    def __del__(self):
        try:
            lib().ref_response_destroy(self._h)
        except Exception:
            pass
