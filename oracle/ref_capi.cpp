/*
 * Test infrastructure (oracle only): a plain C entry-point layer over the reference's
 * own CPU implementation of the waveform -> likelihood path, so Python tests and the
 * CPU baseline can call the UNMODIFIED reference C++ through ctypes.  This file is
 * compiled together with the reference sources where they lie
 * (src/bbhx/cutils/{PhenomHMWaveform,Response,Interpolate,WaveformBuild,Likelihood}.cu,
 * each as C++, the way the reference's CPU backend is built: cutils/CMakeLists.txt:388-396)
 * by oracle/build_ref.py; the result is oracle/_ref/libbbhx_ref.so.
 *
 * Each function forwards to the reference routine named in its comment, with the same
 * argument order as the reference's Cython bindings (the drop-in boundary).
 */
#include "global.h"
#include "PhenomHMWaveform.hh"
#include "Response.hh"
#include "Interpolate.hh"
#include "WaveformBuild.hh"
#include "Likelihood.hh"

extern "C" {

/* PhenomHMWaveform.hh:354-371 */
void ref_waveform_amp_phase(double *out, int *ells, int *mms, double *freqs, double *m1_SI,
                            double *m2_SI, double *chi1z, double *chi2z, double *distance,
                            double *f_ref, int numModes, int length, int numBinAll,
                            double *Mf_RD_lm, double *Mf_DM_lm, int run_phenomd)
{
    waveform_amp_phase(out, ells, mms, freqs, m1_SI, m2_SI, chi1z, chi2z, distance, f_ref,
                       numModes, length, numBinAll, Mf_RD_lm, Mf_DM_lm, run_phenomd);
}

/* PhenomHMWaveform.hh:322-333 */
void ref_get_phenomhm_ringdown_frequencies(double *fring, double *fdamp, double *m1, double *m2,
                                           double *chi1z, double *chi2z, int *ells, int *mms,
                                           int numModes, int numBinAll)
{
    get_phenomhm_ringdown_frequencies_wrap(fring, fdamp, m1, m2, chi1z, chi2z, ells, mms,
                                           numModes, numBinAll);
}

/* PhenomHMWaveform.hh:335-352 */
void ref_get_phenomd_ringdown_frequencies(double *fring, double *fdamp, double *m1, double *m2,
                                          double *chi1z, double *chi2z, int numBinAll,
                                          double *y_rd, double *c1_rd, double *c2_rd,
                                          double *c3_rd, double *y_dm, double *c1_dm,
                                          double *c2_dm, double *c3_dm, double dspin)
{
    get_phenomd_ringdown_frequencies_wrap(fring, fdamp, m1, m2, chi1z, chi2z, numBinAll, y_rd,
                                          c1_rd, c2_rd, c3_rd, y_dm, c1_dm, c2_dm, c3_dm, dspin);
}

/* lisaresponse.pyx:12-13,34-76: pyFastLISAResponse object lifetime and orbit tables */
void *ref_response_create(void) { return (void *)new FastLISAResponse(); }

void ref_response_add_orbit_information(void *h, double dt, int N, double *n_arr, double *L_arr,
                                        double *x_arr, int *links, int *sc_r, int *sc_e,
                                        double armlength)
{
    ((FastLISAResponse *)h)->add_orbit_information(dt, N, n_arr, L_arr, x_arr, links, sc_r, sc_e,
                                                   armlength);
}

void ref_response_destroy(void *h)
{
    FastLISAResponse *r = (FastLISAResponse *)h;
    r->dealloc();
    delete r;
}

/* Response.hh:27-41 */
void ref_LISA_response(void *h, double *buf, int *ells, int *mms, double *freqs, double *phi_ref,
                       double *inc, double *lam, double *beta, double *psi, int TDItag,
                       int rescaled, int tdi2, int order_fresnel_stencil, int numModes, int length,
                       int numBinAll, int includesAmps)
{
    ((FastLISAResponse *)h)
        ->LISA_response(buf, ells, mms, freqs, phi_ref, inc, lam, beta, psi, TDItag,
                        rescaled != 0, tdi2 != 0, order_fresnel_stencil, numModes, length,
                        numBinAll, includesAmps);
}

/* Interpolate.hh:4-6 */
void ref_interpolate(double *freqs, double *y, double *B, double *ud, double *diag, double *ld,
                     int length, int numInterpParams, int numModes, int numBinAll)
{
    interpolate(freqs, y, B, ud, diag, ld, length, numInterpParams, numModes, numBinAll);
}

/* WaveformBuild.hh:6 */
void ref_InterpTDI(long *template_ptrs, double *data_freqs, double *freqs, double *y, double *c1,
                   double *c2, double *c3, double *t_start, double *t_end, int length,
                   int data_length, int numBinAll, int numModes, long *inds_ptrs, int *inds_start,
                   int *ind_lengths)
{
    InterpTDI(template_ptrs, data_freqs, freqs, y, c1, c2, c3, t_start, t_end, length, data_length,
              numBinAll, numModes, inds_ptrs, inds_start, ind_lengths);
}

/* WaveformBuild.hh:8-10 */
void ref_direct_sum(double *templates, double *buf, int numBinAll, int data_length, int nChannels,
                    int numModes, double *t_start, double *t_end)
{
    direct_sum((cmplx *)templates, buf, numBinAll, data_length, nChannels, numModes, t_start,
               t_end);
}

/* Likelihood.hh:11 */
void ref_direct_like(double *d_h, double *h_h, double *data, double *noise, long *template_ptrs,
                     int *inds_start, int *ind_lengths, int data_stream_length, int numBinAll)
{
    direct_like((cmplx *)d_h, (cmplx *)h_h, (cmplx *)data, noise, template_ptrs, inds_start,
                ind_lengths, data_stream_length, numBinAll);
}

/* Likelihood.hh:6-9 */
void ref_hdyn(double *d_h, double *h_h, double *residuals, double *constants, double *freqs,
              int numBinAll, int data_length, int nChannels)
{
    hdyn((cmplx *)d_h, (cmplx *)h_h, (cmplx *)residuals, (cmplx *)constants, freqs, numBinAll,
         data_length, nChannels);
}

} /* extern "C" */
