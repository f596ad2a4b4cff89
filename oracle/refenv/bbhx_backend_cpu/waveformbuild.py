import numpy as np

from . import I, P, lib


def InterpTDI_wrap(template_ptrs, data_freqs, freqs, y, c1, c2, c3, t_start, t_end, length,
                   data_length, num_bin_all, num_modes, inds_ptrs, inds_start, ind_lengths):
    template_ptrs = np.ascontiguousarray(template_ptrs, dtype=np.int64)
    inds_ptrs = np.ascontiguousarray(inds_ptrs, dtype=np.int64)
    inds_start = np.ascontiguousarray(inds_start, dtype=np.int32)
    ind_lengths = np.ascontiguousarray(ind_lengths, dtype=np.int32)
    t_start = np.ascontiguousarray(t_start, dtype=np.float64)
    t_end = np.ascontiguousarray(t_end, dtype=np.float64)
    lib().ref_InterpTDI(P(template_ptrs), P(data_freqs, np.float64), P(freqs, np.float64),
                        P(y, np.float64), P(c1, np.float64), P(c2, np.float64), P(c3, np.float64),
                        P(t_start), P(t_end), I(length), I(data_length), I(num_bin_all),
                        I(num_modes), P(inds_ptrs), P(inds_start), P(ind_lengths))


def direct_sum_wrap(templates, buf, num_bin_all, length, n_channels, num_modes, t_start, t_end):
    t_start = np.ascontiguousarray(t_start, dtype=np.float64)
    t_end = np.ascontiguousarray(t_end, dtype=np.float64)
    lib().ref_direct_sum(P(templates, np.complex128), P(buf, np.float64), I(num_bin_all),
                         I(length), I(n_channels), I(num_modes), P(t_start), P(t_end))
