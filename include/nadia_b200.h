/*
 * nadia_b200.h -- C ABI of the B200 phase-retrieval library (libnadia_b200.so).
 *
 * One handle (nadia_solver) is one reconstruction: the state of one
 * PlanarCDI / FresnelCDI / PolyCDI object of the reference library
 * (NADIA/include/PlanarCDI.h, FresnelCDI.h, PolyCDI.h over BaseCDI.h),
 * resident on the current CUDA device, with its own CUDA stream.
 *
 * Conventions
 *   - Arrays are host memory.  A real array holds nx*ny doubles, a complex
 *     array nx*ny interleaved (re,im) pairs; element (x,y) is at x*ny+y, the
 *     reference's layout (NADIA/include/Complex_2D.h:179-194,
 *     NADIA/include/Double_2D.h:121-143).
 *   - Every entry point returns NADIA_OK (0) or a nonzero status; none of them
 *     exits the process.  nadia_last_error() gives a message for the calling
 *     thread.  (The reference prints and calls exit(); the IDL binding,
 *     NADIA/interfaces/idl/IDL_interface.c, is the C precedent for this ABI.)
 *   - A handle is used by one host thread at a time.
 *   - Precision: NADIA_FP64 runs the plain double-precision path, which
 *     reproduces the reference's own double build (-DDOUBLE_PRECISION) loop by
 *     loop; NADIA_FP32 runs the fused single-precision path (complex FP32
 *     transforms and projections, FP64 error and support reductions).
 *   - Sizes must be even (the reference's quadrant swap assumes it,
 *     NADIA/src/Complex_2D.c++:327-331), except for PlanarCDI in the FP64
 *     form, which reproduces what the swap does on odd sizes; every prime
 *     factor of a transform length must be at most 1021.
 */
#ifndef NADIA_B200_H
#define NADIA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nadia_solver nadia_solver;

/* status codes */
enum {
    NADIA_OK = 0,
    NADIA_ERR_INVALID = 1,     /* bad argument or size */
    NADIA_ERR_STATE = 2,       /* call not valid in the current state */
    NADIA_ERR_UNSUPPORTED = 3, /* feature not provided on this path */
    NADIA_ERR_CUDA = 4,        /* CUDA runtime error */
    NADIA_ERR_NOMEM = 5,       /* device allocation failed */
    NADIA_ERR_RANGE = 6        /* index out of range (get_best_result) */
};

/* geometries */
enum { NADIA_PLANAR = 0, NADIA_FRESNEL = 1, NADIA_POLY = 2, NADIA_FRESNEL_WF = 3 };

/* arithmetic forms */
enum { NADIA_FP64 = 0, NADIA_FP32 = 1 };

/* algorithms, numbered as the reference's enum (NADIA/include/BaseCDI.h:79) */
enum {
    NADIA_ER = 0, NADIA_BIO = 1, NADIA_BOO = 2, NADIA_HIO = 3, NADIA_DM = 4,
    NADIA_SF = 5, NADIA_ASR = 6, NADIA_HPR = 7, NADIA_RAAR = 8, NADIA_CUSTOM = 9
};

/* Message describing the last failure on the calling thread ("" if none). */
const char *nadia_last_error(void);

/* Library version string. */
const char *nadia_version(void);

/* ---- lifecycle -------------------------------------------------------- */

/* PlanarCDI(Complex_2D&, n_best)  -- NADIA/include/PlanarCDI.h:28-29.
 * The estimate starts at zero; the algorithm starts as ER (BaseCDI.c++:63-64). */
int nadia_planar_create(int nx, int ny, int precision, int n_best, nadia_solver **out);

/* FresnelCDI(initial_guess, white_field, wavelength, focal_detector_length,
 * focal_sample_length, pixel_size, normalisation, n_best)
 * -- NADIA/src/FresnelCDI.c++:20-44.  white_field: complex detector-plane field. */
int nadia_fresnel_create(int nx, int ny, int precision, const double *white_field,
                         double beam_wavelength, double focal_detector_length,
                         double focal_sample_length, double pixel_size,
                         double normalisation, int n_best, nadia_solver **out);

/* PolyCDI(initial_guess, beta, n_best, parallel) -- NADIA/src/PolyCDI.c++:25-35.
 * As in the reference, `beta` is stored but never reaches the algorithm
 * weights (PolyCDI.h:53 shadows BaseCDI's beta); the relaxation parameter is
 * set with nadia_set_relaxation_parameter. */
int nadia_poly_create(int nx, int ny, int precision, double beta, int n_best,
                      nadia_solver **out);

/* FresnelCDI_WF(initial_guess, wavelength, zone_focal_length,
 * focal_detector_length, pixel_size, n_best) -- NADIA/src/FresnelCDI_WF.c++:17-79:
 * recovery of the white field (the detector-plane illumination that
 * FresnelCDI consumes) from a white-field measurement; the estimate is the
 * detector-plane field.  Both forms; NADIA_FP32 on grids of 256 ... 4096 per
 * axis (one column and one row pass per iteration; NADIA_ERR_UNSUPPORTED on
 * other sizes).  Its algorithm is fixed (FresnelCDI_WF.c++:155-162):
 * set_algorithm, set_custom_algorithm and set_relaxation_parameter return
 * NADIA_ERR_UNSUPPORTED, where the reference prints a warning. */
int nadia_fresnel_wf_create(int nx, int ny, int precision, double beam_wavelength,
                            double zone_focal_length, double focal_detector_length,
                            double pixel_size, int n_best, nadia_solver **out);

/* FresnelCDI_WF::set_support(z_diameter, size) -- FresnelCDI_WF.c++:184-203:
 * the disk the zone plate of diameter z_diameter projects (scaled by size,
 * the reference's default 1.01) set to 1, then the support blurred (sigma 3,
 * 5-pixel cut-off). */
int nadia_fresnel_wf_set_support(nadia_solver *s, double z_diameter, double size);

/* Releases the device memory and stream of a handle (NULL is accepted). */
int nadia_destroy(nadia_solver *s);

/* Grid size and kind of a handle. */
int nadia_get_size(const nadia_solver *s, int *nx, int *ny);

/* ---- inputs ------------------------------------------------------------ */

/* BaseCDI::set_support(const Double_2D&, bool soften) -- BaseCDI.c++:95-108:
 * support = obj / max(obj), optionally blurred (sigma 3, 5-pixel cut-off). */
int nadia_set_support(nadia_solver *s, const double *support, int soften);

/* BaseCDI::set_intensity -- BaseCDI.c++:118-124 (stores sqrt(I)). */
int nadia_set_intensity(nadia_solver *s, const double *intensity);

/* BaseCDI::set_beam_stop -- BaseCDI.c++:112-116: 0 = unmeasured pixel,
 * left free by the modulus projection; >0 = measured. */
int nadia_set_beam_stop(nadia_solver *s, const double *mask);

/* PolyCDI::set_spectrum(Double_2D) -- PolyCDI.c++:66-89.  wl_weight holds
 * nlambda rows of (wavelength, weight); list the longest wavelength first
 * (the padding is derived from row 0 and must not be negative). */
int nadia_poly_set_spectrum(nadia_solver *s, const double *wl_weight, int nlambda);

/* PolyCDI::set_spectrum(string) -- PolyCDI.c++:38-63 reading the file with
 * read_spec (NADIA/src/io_spec.c:61-133: tab-separated "energy weight" lines,
 * energy stored as its reciprocal, values pass through float). */
int nadia_poly_set_spectrum_file(nadia_solver *s, const char *path);

/* read_spec (NADIA/src/io_spec.c:61-133) on its own: parses the file into
 * rows of (1/energy, weight), writes min(*nrows, capacity) of them to rows
 * (2 doubles each; rows may be NULL when capacity is 0) and sets *nrows to
 * the number in the file.  Needs no GPU. */
int nadia_read_spec(const char *path, double *rows, int capacity, int *nrows);

/* Moves an FP32 reconstruction to the FP64 form in place (no-op on FP64):
 * estimate, support, intensity, beam stop, Fresnel illumination and geometry,
 * spectrum, algorithm, error history and n-best results carry over, FP32
 * values widened.  Needed before complex-constraint regions or a custom
 * constraint function (FP64 only), or any constraint or phase-diverse
 * position on an FP32 PolyCDI. */
int nadia_convert_to_fp64(nadia_solver *s);

/* NADIA_FP32 or NADIA_FP64. */
int nadia_get_precision(const nadia_solver *s, int *precision);

/* The padding PolyCDI derived from its spectrum (PolyCDI.c++:86-87). */
int nadia_poly_get_padding(const nadia_solver *s, int *px, int *py);

/* ---- transmission constraint ------------------------------------------------ */

/* BaseCDI::set_complex_constraint (NADIA/include/BaseCDI.h:471-473) with a
 * TransmissionConstraint (NADIA/include/TransmissionConstraint.h:200-375):
 * applied after every support projection (BaseCDI::apply_support,
 * BaseCDI.c++:130-134) -- to the estimate, or for FresnelCDI to its
 * transmission function (FresnelCDI.c++:203-215, and in get_transmission).
 * enforce_unity: magnitudes above 1 set to 1; charge_flip with flip_sign
 * (+1 or -1): imaginary parts with flip_sign*imag > 0 negated; nregions (at
 * most 16) ComplexConstraint regions, given as nregions masks of nx*ny
 * (a pixel belongs to the first region whose mask is > 0 there), alpha as
 * nregions pairs (alpha1, alpha2), fixed_c as nregions values (NaN = c_mean
 * measured each time; NULL = all measured).  The FP32 form runs the
 * per-pixel part (unit magnitude, charge flipping) inside its fused row pass
 * and returns NADIA_ERR_UNSUPPORTED for regions and for PolyCDI: convert the
 * handle first (nadia_convert_to_fp64). */
int nadia_set_transmission_constraint(nadia_solver *s, int enforce_unity, int charge_flip,
                                      int flip_sign, int nregions, const double *regions,
                                      const double *alpha, const double *fixed_c);

/* TransmissionConstraint::set_custom_constraint (TransmissionConstraint.h:
 * 357-359): fn is called on the host with the constrained transmission
 * (interleaved complex, x*ny+y) after the built-in steps and may change it;
 * NULL removes it.  Needs a constraint set first; FP64 form only
 * (NADIA_ERR_UNSUPPORTED on FP32 unless fn is NULL). */
int nadia_set_transmission_custom(nadia_solver *s,
                                  void (*fn)(double *transmission, int nx, int ny, void *user),
                                  void *user);

/* Removes the transmission constraint (BaseCDI without one). */
int nadia_clear_transmission_constraint(nadia_solver *s);

/* ---- algorithm ---------------------------------------------------------- */

/* BaseCDI::set_algorithm -- BaseCDI.c++:192-237.  Returns early when the
 * algorithm is unchanged, as the reference does. */
int nadia_set_algorithm(nadia_solver *s, int algorithm);

/* BaseCDI::set_custom_algorithm(m1..m10) -- BaseCDI.c++:240-255. */
int nadia_set_custom_algorithm(nadia_solver *s, const double m[10]);

/* BaseCDI::set_relaxation_parameter -- NADIA/include/BaseCDI.h:264-267.  As in
 * the reference, the new beta takes effect at the next change of algorithm. */
int nadia_set_relaxation_parameter(nadia_solver *s, double beta);

/* The five operator weights [PsPf, PfPs, Ps, Pf, I] in use (BaseCDI.c++:245-249). */
int nadia_get_algorithm_structure(const nadia_solver *s, double w[5], int *algorithm);

/* Host-only helper, no handle or GPU needed: the weights that
 * set_custom_algorithm(m1..m10) produces (BaseCDI.c++:245-249). */
void nadia_custom_weights(const double m[10], double w[5]);

/* ---- estimate ----------------------------------------------------------- */

/* initialise_estimate(seed): PlanarCDI.c++:39-62, FresnelCDI.c++:152-201,
 * PolyCDI.c++:102-126.  Draws the C library's srand(seed)/rand() sequence on
 * the host, as the reference does, from a private generator state (the
 * process's own rand() state is left alone, so handles can initialise from
 * several threads), then uploads the estimate. */
int nadia_initialise_estimate(nadia_solver *s, int seed);

/* BaseCDI::set_exit_surface_wave / get_exit_surface_wave -- NADIA/include/BaseCDI.h:285-291. */
int nadia_set_exit_surface_wave(nadia_solver *s, const double *esw);
int nadia_get_exit_surface_wave(nadia_solver *s, double *esw);

/* Single-precision variants for callers holding float buffers (the
 * reference's default Complex_2D is ComplexR_2D<float>, Complex_2D.h:511-512). */
int nadia_set_exit_surface_wave_f32(nadia_solver *s, const float *esw);
int nadia_get_exit_surface_wave_f32(nadia_solver *s, float *esw);

/* ---- run ---------------------------------------------------------------- */

/* `iterations` calls of BaseCDI::iterate (BaseCDI.c++:297-387) or
 * PolyCDI::iterate (PolyCDI.c++:130-250). */
int nadia_iterate(nadia_solver *s, int iterations);

/* BaseCDI::get_error -- BaseCDI.c++:126-128: the error metric computed by the
 * last modulus projection (that is, of the estimate before the last update). */
int nadia_get_error(nadia_solver *s, double *error);

/* The error metric of each of the last `count` iterations, oldest first
 * (count <= the number of iterations run since the handle was created and
 * <= 65536).  Returns NADIA_ERR_RANGE if fewer are available. */
int nadia_get_error_history(nadia_solver *s, double *errors, int count);

/* BaseCDI::apply_shrinkwrap(gauss_width, threshold) -- BaseCDI.c++:416-429. */
int nadia_apply_shrinkwrap(nadia_solver *s, double gauss_width, double threshold);

/* BaseCDI::get_support -- NADIA/include/BaseCDI.h:408-410 (copy into `support`). */
int nadia_get_support(nadia_solver *s, double *support);

/* BaseCDI::get_best_result(error, index) -- BaseCDI.c++:82-91.
 * Returns NADIA_ERR_RANGE for an index outside [0, n_best). */
int nadia_get_best_result(nadia_solver *s, int index, double *error, double *esw);

/* BaseCDI::reset_best -- NADIA/include/BaseCDI.h:476-479. */
int nadia_reset_best(nadia_solver *s);

/* get_transmission: FresnelCDI::get_transmission_function (FresnelCDI.c++:298-355)
 * for FRESNEL; the exit-surface wave for PLANAR and POLY (PolyCDI.h:210
 * declares get_transmission without a definition). */
int nadia_get_transmission(nadia_solver *s, double *transmission);

/* FresnelCDI::set_transmission_function (FresnelCDI.c++:253-283) for FRESNEL;
 * set_exit_surface_wave for the others. */
int nadia_set_transmission(nadia_solver *s, const double *transmission);

/* FresnelCDI::auto_set_norm / set_norm / get_illumination_at_sample
 * (FresnelCDI.c++:129-148, 293-296; FresnelCDI.h:216). */
int nadia_fresnel_auto_set_norm(nadia_solver *s);
int nadia_fresnel_set_norm(nadia_solver *s, double normalisation);
int nadia_fresnel_get_illumination_at_sample(nadia_solver *s, double *illumination);

/* FresnelCDI::set_experimental_parameters (FresnelCDI.c++:57-95) and
 * FresnelCDI::set_normalisation (FresnelCDI.h:187-189: records the
 * normalisation without rescaling, so the next set_norm scales relative to it). */
int nadia_fresnel_set_experimental_parameters(nadia_solver *s, double beam_wavelength,
                                              double focal_detector_length,
                                              double focal_sample_length, double pixel_size);
int nadia_fresnel_set_normalisation(nadia_solver *s, double normalisation);

/* The single operators, as the IDL binding exposes them
 * (IDL_interface.c:947-985): each transforms the complex array in place
 * on an nx*ny grid (PLANAR and FRESNEL). */
int nadia_propagate_to_detector(nadia_solver *s, double *field);
int nadia_propagate_from_detector(nadia_solver *s, double *field);
int nadia_scale_intensity(nadia_solver *s, double *field);
int nadia_apply_support(nadia_solver *s, double *field);
int nadia_project_intensity(nadia_solver *s, double *field);

/* PlanarCDI::get_intensity_autocorrelation -- PlanarCDI.c++:13-36. */
int nadia_get_intensity_autocorrelation(nadia_solver *s, double *autoc);

/* Complex_2D::perform_forward_fft / perform_backward_fft (Complex_2D.c++:487-503)
 * on a host array: in-place unnormalised 2-D DFT (forward = sign -1), FP64,
 * computed on the current device with the canonical transform schedule. */
int nadia_fft2d(double *field, int nx, int ny, int forward);

/* Waits for the handle's queued device work. */
int nadia_synchronize(nadia_solver *s);

/* ---- batching ------------------------------------------------------------ */

/* Steps `count` independent reconstructions `iterations` times together:
 * handles of the FP32 form with the same grid size run as one batched
 * launch per pass, the groups of different sizes run concurrently, and the
 * whole step is replayed from a CUDA graph.  Each handle ends in the state
 * that `iterations` calls of nadia_iterate would have left it in.  No
 * counterpart in the reference, which runs one reconstruction per process. */
int nadia_iterate_many(nadia_solver *const *solvers, int count, int iterations);

/* ---- serving (no counterpart in the reference) ----------------------------
 *
 * A request loop on the current GPU: diffraction patterns are submitted at
 * any time from any thread, admitted in arrival order while at most
 * `max_active` reconstructions are on the device and the admission charge of
 * the active ones (nadia_estimate_device_bytes) stays within `budget_bytes`,
 * and all active reconstructions step together (as nadia_iterate_many) in
 * steps of up to `chunk` iterations, shortened so that no request passes its
 * next shrinkwrap or its last iteration.  Each request's estimate, support
 * and intensity stay on the device until it finishes; its result then waits
 * on the host until nadia_server_result collects it.  A request's result is
 * the same whether it ran alone or among others.  A request runs the calls
 * of a reference driver loop (CDI_reconstruction.c:377-439):
 *   create -> [FRESNEL: auto_set_norm if asked] -> set_support ->
 *   set_intensity -> [set_beam_stop] -> [POLY: set_spectrum] ->
 *   initialise_estimate(seed) -> set_relaxation_parameter(beta) ->
 *   set_algorithm(algorithm) -> iterations x (iterate, and apply_shrinkwrap
 *   after every `shrinkwrap_every`-th iteration). */
typedef struct nadia_server nadia_server;

typedef struct nadia_request {
    int kind;                    /* NADIA_PLANAR, NADIA_FRESNEL or NADIA_POLY */
    int nx, ny;
    int precision;               /* NADIA_FP32 or NADIA_FP64 */
    const double *intensity;     /* nx*ny, copied at submit */
    const double *support;       /* nx*ny, copied at submit */
    const double *beam_stop;     /* nx*ny or NULL */
    const double *spectrum;      /* POLY: nlambda rows of (wavelength, weight) */
    int nlambda;
    const double *white_field;   /* FRESNEL: nx*ny interleaved complex */
    double wavelength, focal_detector_length, focal_sample_length, pixel_size;
    double normalisation;        /* FRESNEL */
    int fresnel_auto_norm;       /* FRESNEL: call auto_set_norm before initialising */
    int algorithm;               /* NADIA_ER, NADIA_HIO, NADIA_RAAR, ... */
    double beta;                 /* relaxation parameter */
    int iterations;
    int shrinkwrap_every;        /* 0 = no shrinkwrap */
    double shrinkwrap_sigma, shrinkwrap_threshold;
    int seed;                    /* initialise_estimate(seed) */
} nadia_request;

int nadia_server_create(unsigned long long budget_bytes, int max_active, int chunk,
                        nadia_server **out);

/* Copies the request's arrays and queues it; *id identifies it.  Returns
 * NADIA_ERR_NOMEM if its admission charge exceeds the whole budget. */
int nadia_server_submit(nadia_server *srv, const nadia_request *req, long long *id);

/* Waits up to timeout_s seconds (negative = no limit) for a request to
 * finish; *done = 1 when it has finished or failed. */
int nadia_server_wait(nadia_server *srv, long long id, double timeout_s, int *done);

/* Collects a finished request and forgets it: esw (2*nx*ny doubles),
 * support (nx*ny) and the final error metric, each optional (NULL), and
 * times[3] = {queued, on the device, arrival to result} in seconds.
 * Returns the request's own status if it failed. */
int nadia_server_result(nadia_server *srv, long long id, double *esw, double *support,
                        double *final_error, double times[3]);

/* out[12] = {queued, active, completed, failed, bytes charged now, peak bytes
 * charged, steps run, requests admitted, then host microseconds spent by the
 * stepping thread stepping and waiting for work, and by the worker threads
 * preparing requests and reading them back}. */
int nadia_server_stats(nadia_server *srv, long long out[12]);

/* Stops the loop (queued and unfinished requests fail) and frees the server. */
int nadia_server_destroy(nadia_server *srv);

/* The admission charge: device bytes one reconstruction holds once all its
 * buffers exist.  poly_pad_x/poly_pad_y: PolyCDI's padding (else 0). */
int nadia_estimate_device_bytes(int kind, int nx, int ny, int precision, int n_best,
                                int poly_pad_x, int poly_pad_y, int nlambda,
                                unsigned long long *bytes);

/* Bytes of device memory the library's reconstructions hold now. */
long long nadia_device_bytes(void);

/* ---- diagnostics (no counterpart in the reference) ----------------------- */

/* The CUDA stream (cudaStream_t) a handle's device work is queued on, so a
 * caller can time it with events on that stream.  nadia_iterate_many queues
 * on the stream of its first handle. */
int nadia_get_stream(nadia_solver *s, void **stream);

/* Mean device time in microseconds of each pass of the fused FP32 iteration
 * for `count` handles of one size and geometry run as a batch (CUDA events
 * around `reps` launches of each pass): out_us = {column pass, second column
 * pass (PolyCDI's modulus and inverse column transform; 0 otherwise), row
 * pass}.  The passes run for real: each handle advances by 1 + reps
 * iterations. */
int nadia_pass_times(nadia_solver *const *solvers, int count, int reps, double out_us[3]);

/* Kernels this library has launched in this process (graph replays count
 * every kernel they contain). */
long long nadia_launch_count(void);

/* The tile variants the autotuner picked for FP32 grids of nx x ny (tuning
 * them now, on the current GPU, if this process has not yet): one line
 * naming the column- and row-pass variants and their timed microseconds
 * (0 when the choice came from NADIA_TUNE=0 or a tune file).  batched != 0:
 * the choice nadia_iterate_many uses. */
int nadia_tuned_tiles(int nx, int ny, int fresnel, int batched, char *buf, int len);

/* ---- shrinkwrap without device allocation (no counterpart in the reference)
 *
 * For callers that cannot allocate device memory when they need a support
 * update: a server stepping many reconstructions on concurrent streams,
 * where cudaMalloc/cudaFree would synchronise the device and stall the other
 * streams, or a process whose device memory is already committed to an
 * admission budget or another allocator.  Same computation as
 * BaseCDI::apply_shrinkwrap (BaseCDI.c++:416-429) in single precision, on
 * caller-owned device buffers: esw_dev holds nx*ny interleaved complex
 * floats, support_dev receives nx*ny floats (element (x,y) at x*ny+y).  Work
 * is queued on `stream` (a cudaStream_t; NULL = the default stream) and the
 * call returns without waiting.  It allocates nothing: its working memory is
 * a 128 KB array built into the library that every GPU using this entry point
 * keeps until the process exits, which limits the grid to 4096 x 4096
 * (larger grids return NADIA_ERR_INVALID).  All calls on a device share that
 * array, so calls whose work overlaps on the GPU race: serialise them.  The
 * first call on a device looks the array up; make it before capturing a
 * stream on that device. */
int nadia_shrinkwrap_noalloc_f32(const float *esw_dev, float *support_dev, int nx, int ny,
                                 double gauss_width, double threshold, void *stream);

/* ---- PhaseDiverseCDI (phase-diverse / ptychographic reconstruction) -------- */

/* PhaseDiverseCDI (NADIA/include/PhaseDiverseCDI.h, NADIA/src/PhaseDiverseCDI.c++):
 * reconstructions ("frames": FP64 handles, or FP32 ones other than PolyCDI;
 * Fresnel frames exchange their
 * transmission function, others their exit-surface wave) placed at (x, y) on
 * one global object.  Series mode updates the object after each frame;
 * parallel mode iterates every frame (concurrently on the GPU) and then
 * blends them all.  granularity > 1 places frames with sub-pixel resolution
 * (bilinear).  A frame handle can not be destroyed while it belongs to one of
 * these objects.  Arrays are as elsewhere: element (x, y) at x*ny + y,
 * complex interleaved. */
typedef struct nadia_phase_diverse nadia_phase_diverse;

/* PhaseDiverseCDI(beta, gamma, parallel, granularity) -- PhaseDiverseCDI.c++:17-33 */
int nadia_pd_create(double beta, double gamma, int parallel, int granularity,
                    nadia_phase_diverse **out);
int nadia_pd_destroy(nadia_phase_diverse *pd);

/* add_new_position(local, x, y, alpha) -- PhaseDiverseCDI.c++:104-160; grows
 * the object to cover the frame */
int nadia_pd_add_position(nadia_phase_diverse *pd, nadia_solver *frame, double x, double y,
                          double alpha);

/* remove_positions -- PhaseDiverseCDI.c++:60-66: forgets the frames only;
 * frames added afterwards take over the earlier positions by index */
int nadia_pd_remove_positions(nadia_phase_diverse *pd);

/* initialise_estimate -- PhaseDiverseCDI.c++:163-177: object = 1, then every
 * frame's current result blended in */
int nadia_pd_initialise_estimate(nadia_phase_diverse *pd);

/* `cycles` calls of iterate -- PhaseDiverseCDI.c++:180-230 */
int nadia_pd_iterate(nadia_phase_diverse *pd, int cycles);

/* set_iterations_per_cycle / set_feedback_parameter / set_amplification_factor
 * / set_probe_scaling -- PhaseDiverseCDI.h:190-226 (NADIA_ERR_RANGE when the
 * probe number is not that of an added position) */
int nadia_pd_set_iterations_per_cycle(nadia_phase_diverse *pd, int iterations);
int nadia_pd_set_feedback_parameter(nadia_phase_diverse *pd, double beta);
int nadia_pd_set_amplification_factor(nadia_phase_diverse *pd, double gamma);
int nadia_pd_set_probe_scaling(nadia_phase_diverse *pd, int n_probe, double alpha);

/* the object's size (0 x 0 before the first position) */
int nadia_pd_get_size(const nadia_phase_diverse *pd, int *nx, int *ny);

/* get_transmission / set_transmission -- PhaseDiverseCDI.c++:77-101
 * (set: NADIA_ERR_INVALID when the size differs from the current object's) */
int nadia_pd_get_transmission(nadia_phase_diverse *pd, double *out);
int nadia_pd_set_transmission(nadia_phase_diverse *pd, int nx, int ny, const double *t);

/* adjust_positions(type, forwards, x_min, x_max, y_min, y_max, step_size) --
 * PhaseDiverseCDI.c++:232-392: type 0 = CROSS_CORRELATION (image alignment,
 * NADIA/src/utils.c:1151-1300), 1 = MINIMUM_ERROR (search of the frame error,
 * PhaseDiverseCDI.c++:395-447) */
int nadia_pd_adjust_positions(nadia_phase_diverse *pd, int type, int forward, int min_x,
                              int max_x, int min_y, int max_y, double step_size);

/* get_final_x_position / get_final_y_position -- PhaseDiverseCDI.h:255-262 */
int nadia_pd_get_position(const nadia_phase_diverse *pd, int n_probe, double *x, double *y);

#ifdef __cplusplus
}
#endif
#endif /* NADIA_B200_H */
