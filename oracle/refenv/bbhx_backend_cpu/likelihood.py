import numpy as np

from . import I, P, lib


def direct_like_wrap(d_h, h_h, data, noise, template_ptrs, inds_start, ind_lengths,
                     data_stream_length, num_bin_all):
    template_ptrs = np.ascontiguousarray(template_ptrs, dtype=np.int64)
    inds_start = np.ascontiguousarray(inds_start, dtype=np.int32)
    ind_lengths = np.ascontiguousarray(ind_lengths, dtype=np.int32)
    lib().ref_direct_like(P(d_h, np.complex128), P(h_h, np.complex128), P(data, np.complex128),
                          P(noise, np.float64), P(template_ptrs), P(inds_start), P(ind_lengths),
                          I(data_stream_length), I(num_bin_all))


def hdyn_wrap(d_h, h_h, residuals, constants, freqs, num_bin_all, length, n_channels):
    lib().ref_hdyn(P(d_h, np.complex128), P(h_h, np.complex128), P(residuals, np.complex128),
                   P(constants, np.complex128), P(freqs, np.float64), I(num_bin_all), I(length),
                   I(n_channels))
