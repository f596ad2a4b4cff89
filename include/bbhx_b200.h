/*
 * bbhx_b200 -- C ABI of the B200 (sm_100a) implementation of the BBHx batched
 * waveform -> likelihood path.
 *
 * Conventions (all entry points):
 *   - return int status: 0 ok, 1 bad argument, 2 CUDA error, 4 non-finite output,
 *     5 missing orbit tables, 6 size above a fixed limit (3 is unused: nothing in the library
 *     waits on another CTA, stream or device); stream-ordered entry points report non-finite
 *     <d|h> / <h|h> through bbhx_take_status(), the synchronous bbhx_direct_like directly;
 *     bbhx_last_error_string() describes the last failure of the calling thread;
 *   - the last argument is a cudaStream_t passed as void* (NULL = legacy default stream);
 *     work is stream-ordered, nothing synchronises unless stated;
 *   - pointers are DEVICE pointers unless marked [host]; complex arrays are interleaved
 *     (re, im) doubles, layout-compatible with numpy/torch complex128;
 *   - array layouts are the reference's flat layouts: B = binaries, M = modes,
 *     L = sparse length, N = data length, P = interpolated quantities (9).
 *
 * Each entry point names the reference interface it replaces (paths inside the BBHx
 * source tree).  Python binds these with ctypes (bbhx_b200/_lib.py).
 */
#ifndef BBHX_B200_H
#define BBHX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ library */
const char *bbhx_last_error_string(void);

/* Caller-provided workspace: while one is set for the calling thread, every entry point takes
   its scratch (segment tables, partial sums, per-(binary, mode) records, adjoint arrays, ...)
   from [base, base + bytes) of device memory instead of the stream-ordered pool
   (cudaMallocAsync), by a 256-byte aligned bump pointer that is rewound when each call
   releases its scratch.  The workspace serves one stream at a time: calls on other streams must
   not overlap with it.  base 256-byte aligned (null: back to the pool); refused (status 1)
   while scratch is live.  A call that needs more than the workspace holds returns status 2;
   bbhx_workspace_peak() is the largest extent the calling thread's calls have needed since the
   workspace was set, including that failed request, so the caller can size it. */
int bbhx_workspace_set(void *base, size_t bytes);
size_t bbhx_workspace_peak(void);
int bbhx_version(void);
int bbhx_stream_synchronize(void *stream);
/* synchronise the stream; return 4 if any likelihood output written since the previous call on
 * this device (direct fused / multi-group / hdyn / heterodyned fused) was NaN or infinite, and
 * clear that record; 0 otherwise (no reference counterpart: the reference returns NaN silently) */
int bbhx_take_status(void *stream);
int bbhx_pointer_is_device(const void *ptr);
size_t bbhx_mode_coeffs_bytes(void);
size_t bbhx_response_mode_bytes(void);
/* self-test (no reference counterpart): out[4i..4i+3] = sin, cos of x[i] from the hot-loop
 * Cody-Waite + Taylor routine and from CUDA's sincos */
int bbhx_selftest_sincos(const double *x, double *out, int n, void *stream);
/* self-test (no reference counterpart) of the fused kernel's phase recurrence: thread l anchors
 * at grid bin k0 + l of the phase cubic pc [4] (y, c1, c2, c3 about knot xk; grid f = k df) and
 * steps `steps` times by 32 bins; out [2 lanes steps] = (cos, sin) per (lane, step), device */
int bbhx_selftest_recurrence(const double *pc, double xk, double k0, double df, int lanes,
                             int steps, double *out, void *stream);
/* diagnostic (no reference counterpart): algorithmic operation tallies of the FP64 heterodyne
 * point chain (PhenomHM amp / phase / t(f), TDI transfer, phasor, channel products) summed over
 * num_modes x length points, set-up excluded; out [12] device = add/sub, mul, div, compare,
 * sqrt, cbrt, log, exp, pow, atan, sin-cos, other; params [11] device = m1, m2 [Msun], chi1z,
 * chi2z, distance [m], phi_ref, inc, lam, beta, psi, t_ref; one thread, for measurement */
int bbhx_count_point_ops(void *orbits, unsigned long long *out, const double *params,
                         const int *ells, const int *mms, int num_modes, const double *freqs,
                         int length, const double *qnm_table, int qnm_n, double dspin, int TDItag,
                         int rescaled, int tdi2, void *stream);

/* ------------------------------------------------------------------ PhenomHM */
/* replaces get_phenomhm_ringdown_frequencies_wrap (src/bbhx/cutils/PhenomHMWaveform.hh:322-333);
 * masses in solar masses; outputs [B, M] */
int bbhx_get_phenomhm_ringdown_frequencies(double *fringdown, double *fdamp, const double *m1,
                                           const double *m2, const double *chi1z,
                                           const double *chi2z, const int *ells, const int *mms,
                                           int num_modes, int num_bin_all, void *stream);

/* replaces get_phenomd_ringdown_frequencies_wrap (PhenomHMWaveform.hh:335-352); outputs [B] */
int bbhx_get_phenomd_ringdown_frequencies(double *fringdown, double *fdamp, const double *m1,
                                          const double *m2, const double *chi1z,
                                          const double *chi2z, int num_bin_all,
                                          const double *y_rd, const double *c1_rd,
                                          const double *c2_rd, const double *c3_rd,
                                          const double *y_dm, const double *c1_dm,
                                          const double *c2_dm, const double *c3_dm, double dspin,
                                          void *stream);

/* both ringdown sets in the [B, M+1] layout the waveform kernel reads
 * (replaces the two calls + concatenation of src/bbhx/waveforms/phenomhm.py:397-463);
 * qnm_table = 8 rows of table_len: y, c1, c2, c3 (ringdown), y, c1, c2, c3 (damping) */
int bbhx_ringdown_frequencies_all(double *fringdown, double *fdamp, const double *m1,
                                  const double *m2, const double *chi1z, const double *chi2z,
                                  const int *ells, const int *mms, int num_modes, int num_bin_all,
                                  const double *qnm_table, int table_len, double dspin,
                                  int run_phenomd, void *stream);

/* replaces waveform_amp_phase (PhenomHMWaveform.hh:354-371): waveform_out [>=3, B, M, L] */
int bbhx_waveform_amp_phase(double *waveform_out, const int *ells, const int *mms,
                            const double *freqs, const double *m1_SI, const double *m2_SI,
                            const double *chi1z, const double *chi2z, const double *distance,
                            const double *f_ref, int num_modes, int length, int num_bin_all,
                            const double *Mf_RD_lm, const double *Mf_DM_lm, int run_phenomd,
                            void *stream);

/* No counterpart in the reference.  Allocation-free form of bbhx_waveform_amp_phase for
 * callers that must not allocate device memory (a host whose own pool owns the GPU, loops
 * where cudaMalloc's device-wide synchronisation would stall other streams, deployments
 * without the stream-ordered allocator).  Its per-(binary, mode) scratch is a static device
 * array inside the library (8192 records of 848 B, ~6.9 MB held by every GPU that loads the
 * library): num_bin_all * num_modes must be <= 8192 (else status 6, nothing launched).  The
 * first call on a device looks up that array's address (make it before any stream capture)
 * and keeps it for the life of the device's primary context, so a cudaDeviceReset while the
 * library is in use is not supported; all calls share the array, so calls that overlap on the
 * GPU race and must be serialised. */
int bbhx_waveform_amp_phase_noalloc(double *waveform_out, const int *ells, const int *mms,
                                    const double *freqs, const double *m1_SI,
                                    const double *m2_SI, const double *chi1z, const double *chi2z,
                                    const double *distance, const double *f_ref, int num_modes,
                                    int length, int num_bin_all, const double *Mf_RD_lm,
                                    const double *Mf_DM_lm, int run_phenomd, void *stream);

/* split form of waveform_amp_phase: per-(binary, mode) records (B*M * bbhx_mode_coeffs_bytes(),
 * coeffs 16-byte aligned, else status 1), then per-frequency evaluation with the t_ref shift
 * of phenomhm.py:485-507 fused (t_ref may be NULL), or t(f) alone */
int bbhx_phenomhm_setup(void *coeffs, const int *ells, const int *mms, const double *m1_SI,
                        const double *m2_SI, const double *chi1z, const double *chi2z,
                        const double *distance, const double *Mf_RD_lm, const double *Mf_DM_lm,
                        int num_modes, int num_bin_all, int run_phenomd, void *stream);
int bbhx_phenomhm_points(double *waveform_out, const double *freqs, const void *coeffs,
                         const double *t_ref, double t_init, int num_modes, int length,
                         int num_bin_all, void *stream);
int bbhx_phenomhm_tf(double *tf_out, const double *freqs, const void *coeffs, const double *t_ref,
                     int num_modes, int length, int num_bin_all, void *stream);

/* default sparse grid of phenomhm.py:208-224 */
int bbhx_default_freqs(double *freqs, const double *m1, const double *m2, const int *mms,
                       double mf_min, double mf_max, int num_modes, int length, int num_bin_all,
                       void *stream);

/* observation-window regrid of phenomhm.py:513-614 (t(f) crossing of 0 and Tobs, then
 * logspace); err_dev: device int, zeroed by the caller, 1/2 on a failed crossing search */
int bbhx_tf_window_regrid(double *freqs_out, double *fminmax, const double *freqs_in,
                          const double *tf, const double *Tobs, int length, long long num_rows,
                          int *err_dev, void *stream);

/* ------------------------------------------------------------------ response */
/* replaces pyFastLISAResponse / AddOrbits (src/bbhx/cutils/lisaresponse.pyx:12-13,34-76) */
int bbhx_orbits_create(void **handle);
/* n_arr, L_arr, x_arr, links, sc_r, sc_e are [host] arrays (copied to the device) */
int bbhx_orbits_add_orbit_information(void *handle, double dt, int N, const double *n_arr,
                                      const double *L_arr, const double *x_arr, const int *links,
                                      const int *sc_r, const int *sc_e, double armlength);
int bbhx_orbits_destroy(void *handle);

/* replaces FastLISAResponse::LISA_response (src/bbhx/cutils/Response.hh:27-41) */
int bbhx_LISA_response(void *orbits, double *response_out, const int *ells, const int *mms,
                       const double *freqs, const double *phi_ref, const double *inc,
                       const double *lam, const double *beta, const double *psi, int TDItag,
                       int rescaled, int tdi2, int order_fresnel_stencil, int num_modes,
                       int length, int num_bin_all, int includes_amps, void *stream);

/* fused PhenomHM + response into a [9, B, M, L] buffer (waveformbuild.py:516-560 in one pass) */
int bbhx_waveform_response_fused(void *orbits, double *buf, const double *freqs,
                                 const void *coeffs, const int *ells, const int *mms,
                                 const double *phi_ref, const double *inc, const double *lam,
                                 const double *beta, const double *psi, const double *t_ref,
                                 double t_init, int TDItag, int rescaled, int tdi2, int num_modes,
                                 int length, int num_bin_all, void *stream);

/* ------------------------------------------------------------------ spline */
/* replaces interpolate (src/bbhx/cutils/Interpolate.hh:4-6) */
int bbhx_interpolate(const double *freqs, const double *y, double *B_, double *upper_diag,
                     double *diag, double *lower_diag, int length, int num_interp_params,
                     int num_modes, int num_bin_all, void *stream);

/* ------------------------------------------------------------------ templates */
/* replaces InterpTDI (src/bbhx/cutils/WaveformBuild.hh:6); template_ptrs, t_start, t_end,
 * inds_ptrs, inds_start, ind_lengths are [host] arrays (pointer arrays hold device addresses);
 * synchronises the stream once (the job table is copied from those host arrays) */
int bbhx_InterpTDI(const int64_t *template_ptrs, const double *data_freqs, const double *freqs,
                   const double *y, const double *c1, const double *c2, const double *c3,
                   const double *t_start, const double *t_end, int length, int data_length,
                   int num_bin_all, int num_modes, const int64_t *inds_ptrs,
                   const int *inds_start, const int *ind_lengths, void *stream);

/* fill=True placement of per-binary templates on the data grid (replaces the Python slice
 * additions of src/bbhx/waveformbuild.py:663-693; no C counterpart there); template_ptrs,
 * starts, lengths are [host] arrays (device addresses of [3, len] complex128 templates);
 * combine 0: out [B, 3, N], 1: out [3, N] summed in binary order; out zeroed by the caller;
 * synchronises the stream once (the job table is copied from the host arrays) */
int bbhx_fill_templates(void *out, const int64_t *template_ptrs, const int *starts,
                        const int *lengths, int num_bin_all, int data_length, int combine,
                        void *stream);

/* replaces direct_sum (WaveformBuild.hh:8-10) */
int bbhx_direct_sum(double *templates, const double *buffer, int num_bin_all, int length,
                    int n_channels, int num_modes, const double *t_start, const double *t_end,
                    void *stream);

/* ------------------------------------------------------------------ likelihood */
/* replaces direct_like (src/bbhx/cutils/Likelihood.hh:11); d_h, h_h [host] complex, += ;
 * template_ptrs, inds_start, ind_lengths [host]; blocks until the results are on the host */
int bbhx_direct_like(double *d_h, double *h_h, const double *data, const double *noise,
                     const int64_t *template_ptrs, const int *inds_start, const int *ind_lengths,
                     int data_stream_length, int num_bin_all, void *stream);

/* replaces hdyn (Likelihood.hh:6-9) */
int bbhx_hdyn(double *d_h, double *h_h, const double *residuals, const double *constants,
              const double *freqs, int num_bin_all, int length, int n_channels, void *stream);

/* relative-binning constants of the heterodyned likelihood (replaces the per-bin Python loop
 * of HeterodynedLikelihood.init_heterodyne_info, src/bbhx/likelihood.py:480-530; no C
 * counterpart there): f [n] the narrowed dense grid, d and h0 complex rows of 3 channels with
 * row strides ld_d / ld_h, S PSD rows (stride ld_s), freqs [L] the sparse grid, df the dense
 * bin width.  consts [4, 3, L] complex (A0, A1, B0, B1 summed into slot j + 1, the last dense
 * point excluded), ref [3] = <d|d>, <h0|h0>, Re<d|h0> over the band (device). */
int bbhx_hdyn_constants(void *consts, double *ref, const double *f, const void *d, int ld_d,
                        const void *h0, int ld_h, const double *S, int ld_s, int n,
                        const double *freqs, int L, double df, void *stream);

/* ------------------------------------------------------------------ driver bookkeeping on the
 * device (each replaces elementwise array code of the reference's Python drivers, so a
 * likelihood step runs no framework kernels; no C counterparts in the reference) */
/* front end of a step (phenomhm.py:175-199, waveformbuild.py:477-484): out [6, B] = m1, m2
 * (ordered m1 >= m2, Msun), chi1z, chi2z (swapped with the masses), m1, m2 in kg; t_start, t_end
 * [B] = tSSBfromLframe of the observation limits t_obs_start_L / t_obs_end_L (seconds), may be
 * NULL with lam / beta; tobs_rows [B, M] = t_end - t_start (may be NULL); flags device int
 * [nflags >= 3] cleared, then flags[2] |= 1 (some |chi1z| > 1), |= 2 (some |chi2z| > 1) */
int bbhx_step_front(double *out, double *t_start, double *t_end, double *tobs_rows,
                    const double *m1, const double *m2, const double *chi1z, const double *chi2z,
                    const double *lam, const double *beta, int num_bin_all, int num_modes,
                    double t_obs_start_L, double t_obs_end_L, int *flags, int nflags,
                    void *stream);
/* orbit-table coverage of t(f) (fastfdresponse.py:427-433): *flag = 1 if any tf[0..n) lies
 * outside [tmin, tmax] (only ever set) */
int bbhx_tf_range_check(const double *tf, long long n, double tmin, double tmax, int *flag,
                        void *stream);
/* packed [3 B + nflags] = lnL | Re d_h' | Re h_h | flags, lnL = -(d_d + Re h_h - 2 Re d_h') / 2
 * with d_h' = |d_h| when phase_marginalize (likelihood.py:204-225, :633-648) */
int bbhx_pack_lnl(double *packed, const void *d_h, const void *h_h, double d_d, int num_bin_all,
                  int phase_marginalize, const int *flags, int nflags, void *stream);
/* tSSBfromLframe (inverse 0) / tLfromSSBframe (inverse 1) elementwise (utils/transform.py:75-135),
 * t0 in seconds */
int bbhx_tssb_from_lframe(double *out, const double *t, const double *lam, const double *beta,
                          int n, double t0, int inverse, void *stream);
/* LISA_to_SSB (to_ssb 1) / SSB_to_LISA (to_ssb 0) elementwise (utils/transform.py:136-294),
 * t0 in seconds */
int bbhx_frame_transform(double *t_out, double *lam_out, double *beta_out, double *psi_out,
                         const double *t_in, const double *lam_in, const double *beta_in,
                         const double *psi_in, int n, double t0, int to_ssb, void *stream);
/* mbh_sky_mode_transform (utils/transform.py:296-426) in place on coords [rows, ndim] already
 * tiled by the mode count; kind 0 = both (8), 1 = long (4), 2 = lat (2) */
int bbhx_sky_mode_transform(double *coords, int rows, int ndim, int inc, int lam, int beta,
                            int psi, int kind, int cos_i, void *stream);

/* support [start, start+len) of each binary on the data grid (waveformbuild.py:136-177) */
int bbhx_template_support(int *start, int *len, const double *x, int num_modes, int length,
                          int num_bin_all, const double *data_freqs, int data_length,
                          void *stream);

/* One direct-likelihood problem of a multi-group call: its own data stream (N bins), knots
   x [B, M, L], sparse buffer y and spline coefficients c1..c3 [9, B, M, L], observation
   windows t_start / t_end [B], outputs d_h, h_h [B] complex128.  All pointers are device
   memory. */
typedef struct {
  const double *data_freqs;
  const void *data;
  const double *noise;
  int data_length;
  const double *x, *y, *c1, *c2, *c3;
  const double *t_start, *t_end;
  int num_modes, length, num_bin_all;
  void *d_h, *h_h;
  const void *data32;    /* optional FP32 copies (complex64 [3, N], float [3, N]) used by the */
  const float *noise32;  /* mixed form; null to read the FP64 arrays */
} bbhx_direct_group;

/* Several direct-likelihood problems (uneven grid lengths, mode sets and observation spans) in
   ONE persistent launch of the fused kernel; no reference counterpart.  groups is a HOST array
   of num_groups <= 64 descriptors; tile_bins (multiple of 128, at most 4096) and ctas_per_sm
   are the launch shape (chosen by bbhx_b200.uneven.Autotuner).  Stream-ordered and free of host
   synchronisation, so it can be captured in a CUDA graph. */
int bbhx_direct_like_multi(const bbhx_direct_group *groups, int num_groups, int precision,
                           int tile_bins, int ctas_per_sm, void *stream);

/* One heterodyned (relative-binning) problem of an uneven batch: the arguments of
   bbhx_hdyn_fused for its walkers (orbits handle, records from bbhx_phenomhm_setup, the
   response inputs and t_ref [B], observation limits [B], its own sparse grid freqs [L],
   h0 [3, L] and consts [4, 3, L] complex128); d_h, h_h [B] complex128 are overwritten. */
typedef struct {
  void *orbits;
  void *d_h, *h_h;
  const void *coeffs;
  const int *ells, *mms;
  const double *phi_ref, *inc, *lam, *beta, *psi, *t_ref;
  double t_init;
  const double *t_start, *t_end;
  const double *freqs;
  const void *h0, *consts;
  int TDItag, rescaled, tdi2, num_modes, length, num_bin_all;
} bbhx_hdyn_group;

/* One direct-likelihood problem of an uneven batch given by its binaries' parameters (the
   sparse grids and splines are built inside bbhx_uneven_batch): params [12, B] device
   (m1, m2 [Msun], chi1z, chi2z, distance [m], phi_ref, f_ref, inc, lam, beta, psi, t_ref [s]);
   ells, mms [M] device; the PhenomD ringdown table [8, qnm_n] (y, c1, c2, c3 of the ringdown
   and of the damping spline over the final spin, step dspin); mf_min, mf_max the default
   grid's geometric-frequency bounds; t_init the phase reference time; the L-frame
   observation limits [s]; the orbit table's time coverage [s].  Outputs of the build (device):
   x [B, M, L] knots, y, c1, c2, c3 [9, B, M, L], t_start, t_end [B] and flags [3] (window
   search 1 lower / 2 upper, orbit coverage, |chi| > 1 bits 1 / 2: the flags of
   bbhx_step_front, bbhx_tf_window_regrid and bbhx_tf_range_check).  The data stream and the
   likelihood outputs as in bbhx_direct_group. */
typedef struct {
  void *orbits;
  const double *params;
  const int *ells, *mms;
  const double *qnm_table;
  int qnm_n;
  double dspin, mf_min, mf_max, t_init, t_obs_start_L, t_obs_end_L, orbit_tmin, orbit_tmax;
  int TDItag, rescaled, tdi2, run_phenomd, num_modes, length, num_bin_all;
  double *x, *y, *c1, *c2, *c3, *t_start, *t_end;
  int *flags;
  const double *data_freqs;
  const void *data;
  const double *noise;
  int data_length;
  const void *data32;
  const float *noise32;
  void *d_h, *h_h;
} bbhx_direct_source;

/* Direct and heterodyned problems with uneven grid lengths, mode sets, observation spans and
   sparse grids in ONE persistent launch: the walkers of every heterodyned problem and the
   (data tile, binary) items of every direct problem form one work range from which the warps
   claim items through a queue counter (no reference counterpart).  direct / het: HOST arrays
   of at most 64 descriptors each (either may be empty); precision, tile_bins and ctas_per_sm
   as for bbhx_direct_like_multi (the heterodyned walkers use the same precision).
   Stream-ordered, free of host synchronisation (graph-capturable). */
int bbhx_uneven_like(const bbhx_direct_group *direct, int num_direct, const bbhx_hdyn_group *het,
                     int num_het, int precision, int tile_bins, int ctas_per_sm, void *stream);

/* One heterodyned problem of an uneven batch given by its walkers' parameters: `group` as for
   bbhx_uneven_like, except that group.coeffs ([B, M] PhenomHM records, sized
   bbhx_mode_coeffs_bytes() each), group.t_start and group.t_end are device buffers the batch
   fills from params [12, B] (group.phi_ref .. t_ref may point at params' rows) with the
   PhenomD ringdown table, the L-frame observation limits [s] and run_phenomd as in
   bbhx_direct_source; flags [3] receives the |chi| > 1 bits at flags[2] (cleared first). */
typedef struct bbhx_hdyn_source {
  bbhx_hdyn_group group;
  const double *params;
  const double *qnm_table;
  int qnm_n;
  double dspin, t_obs_start_L, t_obs_end_L;
  int run_phenomd;
  int *flags;
} bbhx_hdyn_source;

/* A whole uneven batch from parameters: one launch makes the records of every row (direct
   rows: PhenomHM and response-mode records and observation limits; heterodyned walkers:
   PhenomHM records and observation limits), one launch builds the sparse grids and splines of
   every direct problem (one CTA per (binary, mode) row: default grid and t(f), window regrid,
   waveform + response, coverage check, spline), then bbhx_uneven_like.  No reference
   counterpart; stream-ordered and graph-capturable. */
int bbhx_uneven_batch(const bbhx_direct_source *direct, int num_direct,
                      const struct bbhx_hdyn_source *het, int num_het, int precision,
                      int tile_bins, int ctas_per_sm, void *stream);

/* fused interpolate + mode sum + noise weighting + <d|h>, <h|h> reduction; no templates are
 * stored (equivalent to InterpTDI followed by direct_like, waveformbuild.py:641-660 +
 * likelihood.py:177-214); d_h, h_h device complex [B], overwritten.
 * precision 0: FP64 throughout (the parity form); 1: mixed -- phase, t(f) and all
 * accumulations in FP64, amplitude / transfer / per-bin products in FP32.
 * data32 / noise32: optional FP32 copies of data (complex64 [3, N]) and noise (float [3, N])
 * read by the mixed form instead of data / noise; both null or both given.  With them the
 * mixed form also forms the per-bin products with data and weights in FP64 (about 20-50x
 * smaller lnL error near the peak of loud sources, ~2 % slower); without them, in FP32. */
int bbhx_direct_like_fused(double *d_h, double *h_h, const double *data_freqs, const double *data,
                           const double *noise, int data_length, const double *x, const double *y,
                           const double *c1, const double *c2, const double *c3,
                           const double *t_start, const double *t_end, int num_modes, int length,
                           int num_bin_all, int precision, const void *data32,
                           const float *noise32, void *stream);

/* fused heterodyned likelihood: PhenomHM + TDI response at the sparse heterodyne grid, mode
   sum, r = h / h0 and the relative-binning bin sums in one kernel (one warp per walker).
   Replaces, as one call, waveform_amp_phase (PhenomHMWaveform.hh:354-371) + LISA_response
   (Response.hh:27-41) + direct_sum (WaveformBuild.hh:8-10) + the host-side ratio
   (likelihood.py:606-616) + hdyn (Likelihood.hh:6-9, GPU form: every bin j >= 1).
   coeffs: records from bbhx_phenomhm_setup [B, M]; freqs [L]; h0 [3, L] complex128;
   consts [4, 3, L] complex128 (A0, A1, B0, B1); d_h, h_h [B] complex128 (device).
   precision: 0 = FP64, 1 = mixed (FP64 phase / t(f) / sums, FP32 amplitude / transfer). */
int bbhx_hdyn_fused(void *orbits, void *d_h, void *h_h, const void *coeffs, const int *ells,
                    const int *mms, const double *phi_ref, const double *inc, const double *lam,
                    const double *beta, const double *psi, const double *t_ref, double t_init,
                    const double *t_start, const double *t_end, const double *freqs,
                    const void *h0, const void *consts, int TDItag, int rescaled, int tdi2,
                    int num_modes, int length, int num_bin_all, int precision, void *stream);

/* Heterodyned lnL terms and the gradient d lnL / d theta of B walkers (no reference
   counterpart).  theta = (m1, m2, chi1z, chi2z, distance, phi_ref, inc, lam, beta, psi,
   t_ref): rows 0-5 and 7-11 of params [12, B] (device, row-major); grad [B, 11] (device).
   Reverse part: adjoint of the relative-binning sums and of r = h / h0 (FP64 forward pass);
   forward part: dual-number tangents of PhenomHM + TDI at every (mode, frequency).
   qnm_table [8, qnm_n]: ringdown / damping spline rows (y, c1, c2, c3 each). */
int bbhx_hdyn_grad(void *orbits, void *d_h, void *h_h, double *grad, const void *coeffs,
                   const double *params, const int *ells, const int *mms, const double *qnm_table,
                   int qnm_n, double dspin, double t_init, const double *t_start,
                   const double *t_end, const double *freqs, const void *h0, const void *consts,
                   int TDItag, int rescaled, int tdi2, int run_phenomd, int num_modes, int length,
                   int num_bin_all, void *stream);

/* Gradient d lnL / d theta [B, 11] of the direct likelihood (no reference counterpart):
   reverse through the <d|h>, <h|h> reduction, the spline interpolation onto the data grid
   and the not-a-knot spline build (transposed tridiagonal solve), forward-mode tangents of
   PhenomHM + TDI at the knots.  x [B, M, L] knots; y, c1, c2, c3 [9, B, M, L] from the forward
   path (bbhx_waveform_response_fused + bbhx_interpolate); data [3, N] complex128 noise-weighted,
   noise [3, N]; params [12, B]; theta as for bbhx_hdyn_grad.  The knots' motion through the
   observation-window regrid (bbhx_tf_window_regrid) is differentiated from f_default, the
   default grid the regrid read (bbhx_default_freqs), and tf_default, its t(f) with t_ref
   (bbhx_phenomhm_tf), both [B, M, L], and the L-frame observation limits t_obs_start_L,
   t_obs_end_L [s]; f_default or tf_default null holds the knots fixed.
   d_h, h_h: device complex128 [B], overwritten with <d|h>, <h|h> of the same evaluation (as
   bbhx_direct_like_fused in FP64, so no separate likelihood call is needed).  Synchronises the
   stream once: the binaries' support lengths are read on the host to batch the adjoint. */
int bbhx_direct_like_grad(void *orbits, void *d_h, void *h_h, double *grad,
                          const double *params, const int *ells,
                          const int *mms, const double *qnm_table, int qnm_n, double dspin,
                          double t_init, const double *data_freqs, const void *data,
                          const double *noise, int data_length, const double *x, const double *y,
                          const double *c1, const double *c2, const double *c3,
                          const double *t_start, const double *t_end, const double *f_default,
                          const double *tf_default, double t_obs_start_L, double t_obs_end_L,
                          int TDItag, int rescaled, int tdi2, int run_phenomd, int num_modes,
                          int length, int num_bin_all, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* BBHX_B200_H */
