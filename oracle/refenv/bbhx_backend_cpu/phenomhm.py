import numpy as np

from . import D, I, P, lib


def waveform_amp_phase_wrap(out, ells, mms, freqs, m1_SI, m2_SI, chi1z, chi2z, distance, f_ref,
                            num_modes, length, num_bin_all, fring, fdamp, run_phenomd):
    lib().ref_waveform_amp_phase(
        P(out, np.float64), P(ells, np.int32), P(mms, np.int32), P(freqs, np.float64),
        P(m1_SI, np.float64), P(m2_SI, np.float64), P(chi1z, np.float64), P(chi2z, np.float64),
        P(distance, np.float64), P(f_ref, np.float64), I(num_modes), I(length), I(num_bin_all),
        P(fring, np.float64), P(fdamp, np.float64), I(int(run_phenomd)))


def get_phenomhm_ringdown_frequencies(fring, fdamp, m1, m2, chi1z, chi2z, ells, mms, num_modes,
                                      num_bin_all):
    lib().ref_get_phenomhm_ringdown_frequencies(
        P(fring, np.float64), P(fdamp, np.float64), P(m1, np.float64), P(m2, np.float64),
        P(chi1z, np.float64), P(chi2z, np.float64), P(ells, np.int32), P(mms, np.int32),
        I(num_modes), I(num_bin_all))


def get_phenomd_ringdown_frequencies(fring, fdamp, m1, m2, chi1z, chi2z, num_bin_all, y_rd, c1_rd,
                                     c2_rd, c3_rd, y_dm, c1_dm, c2_dm, c3_dm, dspin):
    lib().ref_get_phenomd_ringdown_frequencies(
        P(fring, np.float64), P(fdamp, np.float64), P(m1, np.float64), P(m2, np.float64),
        P(chi1z, np.float64), P(chi2z, np.float64), I(num_bin_all), P(y_rd, np.float64),
        P(c1_rd, np.float64), P(c2_rd, np.float64), P(c3_rd, np.float64), P(y_dm, np.float64),
        P(c1_dm, np.float64), P(c2_dm, np.float64), P(c3_dm, np.float64), D(dspin))
