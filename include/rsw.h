/*
 * rsw.h -- C ABI of the B200 split-step wavefront propagation engine.
 *
 * Plain C types only (pointers, sizes, doubles); CUDA streams are passed as
 * `void*` (a cudaStream_t, NULL = the legacy default stream). Every entry point
 * returns an rsw_status and never exits the process; the message of the last
 * failure on the calling thread is available from rsw_last_error().
 *
 * Field buffers are device memory owned by the caller, interleaved complex
 * (complex128 = {double re, im}, complex64 = {float re, im}), contiguous,
 * sample i at x = (i - N/2) * dx. Calls are asynchronous on the given stream
 * unless stated otherwise. A plan or simulation object may be used by one host
 * thread at a time.
 *
 * Semantics follow the reference's FP64 implementation (rave-sim big-wave):
 * grating mask coordinates (big-wave/optical_element.py:341-377), the frequency
 * cutoff index range (big-wave/propagation.py:74-97), the Fresnel transfer
 * function (big-wave/propagation.py:124-128) and np.histogram detector binning
 * (big-wave/propagation.py:279-320).
 */
#ifndef RSW_H
#define RSW_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RSW_ABI_VERSION 1

typedef enum {
    RSW_OK = 0,
    RSW_ERR_INVALID = 1,      /* bad argument, size or configuration            */
    RSW_ERR_UNSUPPORTED = 2,  /* valid but not implemented (e.g. N not 2^k)     */
    RSW_ERR_CUDA = 3,         /* CUDA runtime error (message has the details)   */
    RSW_ERR_NOMEM = 4,        /* device or host allocation failed               */
    RSW_ERR_TIMEOUT = 5       /* a bounded device wait expired                  */
} rsw_status;

typedef enum {
    RSW_C128 = 0,       /* complex128 field, all arithmetic FP64 ("c16")                  */
    RSW_C64 = 1,        /* complex64 field, FP32 FFT, FP64 phases and intensity ("c8")    */
} rsw_dtype;

typedef struct rsw_plan_s *rsw_plan;
typedef struct rsw_sim_s *rsw_sim;

/* ---------------------------------------------------------------- errors */
const char *rsw_last_error(void);
int rsw_abi_version(void);
/* Number of kernels this library launched since load (all threads). */
uint64_t rsw_launch_count(void);
/* sizeof of the ABI structs, for bindings to verify their layouts:
 * 0 rsw_element, 1 rsw_sim_desc, 2 rsw_source, 3 rsw_source_run, 4 rsw_tuning. */
size_t rsw_struct_size(int which);

/* Photon wavelength in metres for an energy in eV, evaluated exactly as the
 * reference's convert_energy_wavelength (big-wave/propagation.py:26-28, :69-71). */
double rsw_energy_to_wavelength(double energy_ev);

/* ------------------------------------------------------------ FFT plans
 * Replaces fast-wave's FFT<S> (fast-wave/src/fft.hpp:9-24, src/fft.cpp:6-48):
 * a 1-D complex FFT of length N, forward unnormalised, inverse scaled by 1/N
 * (the reference's inverse + scale kernel, fft.cpp:34-44). 64-bit length.
 * Powers of two from 16 to 2^38 (C64) / 2^35 (C128) run the fused passes: up
 * to 2^26 (C64) / 2^25 (C128) a split step costs two passes over the field,
 * beyond that four (three-level plans); log_rows + log_cols = log2 N. Other
 * lengths from 1 to 2^31 (cufftPlan1d's int range) use Bluestein's algorithm
 * on a power-of-two plan of length M >= 2N - 1 (a transform costs three of
 * length M; log_rows = log_cols = 0), as do powers of two below 16. The
 * length-M plan takes the tuning registered for M, if any.
 * The plan owns its twiddle tables and scratch; it is bound to the device that
 * is current at creation. */
rsw_status rsw_plan_create(rsw_plan *out, int64_t n, int dtype);
rsw_status rsw_plan_destroy(rsw_plan plan);
rsw_status rsw_plan_info(rsw_plan plan, int64_t *n, int *dtype, int *log_rows,
                         int *log_cols, int64_t *scratch_bytes);

/* ------------------------------------------------------------ tuning
 * The choices cuFFT makes inside cufftPlan1d (fast-wave/src/fft.cpp:8) are
 * explicit here: the level split and the samples per thread of each kernel.
 * levels: 0 = the default choice, 1 = one row pass, 2 = columns of 2^log_rows
 * samples and rows of the rest, 3 = columns of 2^log_rows, a middle level of
 * 2^log_mid and rows of the rest. row_e, col_e, mid_e: samples per thread of
 * the row, column and middle kernels (8, 16 or 32 where a kernel exists;
 * 0 = default). An unavailable choice returns RSW_ERR_INVALID. */
typedef struct {
    int levels;
    int log_rows;
    int log_mid;
    int row_e, col_e, mid_e;
} rsw_tuning;
rsw_status rsw_plan_create_tuned(rsw_plan *out, int64_t n, int dtype, const rsw_tuning *tuning);
/* The plan's effective choices (of its length-M plan for Bluestein lengths). */
rsw_status rsw_plan_tuning(rsw_plan plan, rsw_tuning *tuning);
/* Register the tuning that later rsw_plan_create / rsw_sim_create calls use
 * for this n and dtype (process-wide; tuning == NULL removes it). The
 * RSW_SPLIT, RSW_SPLIT3, RSW_ROW_E and RSW_COL_E environment variables take
 * precedence over registered tunings. */
rsw_status rsw_set_tuning(int64_t n, int dtype, const rsw_tuning *tuning);
/* No counterpart in the reference (cuFFT tunes inside its plan call): time
 * every available tuning of (n, dtype) on one steady-state split step of a
 * simulation (reps timed steps each, after two untimed ones, on `stream`,
 * over a field of n samples allocated here) and return the fastest in *best
 * and its milliseconds per split step in *best_ms. tried / tried_ms (may be
 * NULL) receive up to max_tried candidates and their times, *n_tried the
 * number timed. Synchronises `stream`. */
rsw_status rsw_autotune(int64_t n, int dtype, int reps, rsw_tuning *best, double *best_ms,
                        rsw_tuning *tried, double *tried_ms, int max_tried, int *n_tried, void *stream);
/* No counterpart in the reference: rsw_autotune with each split step timed
 * over `fields` transforms of length n in one launch per pass, the launch
 * shape in which rsw_sim_run_batch runs the sources of one field length
 * (the plain pass kernels over the fields; the batched kernels add only the
 * per-source table reads). A field buffer of fields * n samples is
 * allocated here. *best_ms and tried_ms are per split step of all fields.
 * fields = 1 is rsw_autotune. The fastest choice for a
 * batch can differ from the fastest for one field: 2^24 complex128 in
 * batches of 32 runs 2 % faster with 16 samples per thread in both passes,
 * one field with 8. */
rsw_status rsw_autotune_batch(int64_t n, int dtype, int64_t fields, int reps, rsw_tuning *best,
                              double *best_ms, rsw_tuning *tried, double *tried_ms, int max_tried,
                              int *n_tried, void *stream);

/* fast-wave FFT<S>::forward / inverse (src/fft.cpp:28-44); natural order in and
 * out; in == out allowed. */
rsw_status rsw_fft_forward(rsw_plan plan, const void *d_in, void *d_out, void *stream);
rsw_status rsw_fft_inverse(rsw_plan plan, const void *d_in, void *d_out, void *stream);

/* No counterpart in the reference. The natural-order forward FFT of
 * rsw_fft_forward (same result) for callers that cannot allocate device
 * memory where they need it: a process whose free device memory is owned by
 * another allocator (a framework's caching allocator, so a raw cudaMalloc
 * fails or fragments it), or a latency-sensitive loop that must not pay the
 * device-wide synchronisation of cudaFree. It needs no plan and allocates
 * nothing: its scratch is a fixed 1.5 MiB array in the library's device
 * image (held by every GPU that loads the library until exit), so n is
 * limited to RSW_NOALLOC_MAX_N samples; larger n returns RSW_ERR_INVALID.
 * The first call on each device (with that device current) looks up the
 * array's device address, and the first call for each n and dtype on a
 * device builds that length's twiddle tables in its own part of the array
 * (never rebuilt afterwards); make those calls before any stream capture: a
 * first call for an n and dtype made while the stream is capturing returns
 * RSW_ERR_INVALID. A CUDA error left pending by earlier work is reported
 * (RSW_ERR_CUDA) and not cleared. All calls share the array's intermediate
 * spectrum and it keeps the last call's contents; calls that overlap on the
 * GPU race and must be serialised by the caller. in == out is allowed. */
#define RSW_NOALLOC_MAX_N 65536
rsw_status rsw_fft_forward_noalloc(const void *d_in, void *d_out, int64_t n, int dtype, void *stream);

/* Out-of-core FFT of a field held in HOST memory (pinned or pageable), for
 * fields larger than the device's memory. Replaces big-fourier's fft / ifft
 * (big-fourier/src/bfft.rs:27-100; Python bfpy.fft_c16 / ifft_c16 / fft_c8 /
 * ifft_c8, big-fourier/src/lib.rs:65-126, called by big-wave/vector.py:134-146)
 * with the same four-step split and NumPy convention (inverse scaled by 1/N).
 * The field streams through two pipelines of three device slabs within
 * device_bytes (at least 6 * 2^ceil(log2(N)/2) samples), on `stream` and a
 * second stream, so that uploads, transforms and downloads overlap; the GPU
 * runs every transform pass.
 * h_scratch holds N samples of intermediate results; NULL uses h_out.
 * h_out may equal h_in when a separate scratch is given; the scratch must not
 * be h_in. N is a power of two >= 256. Synchronises `stream` before returning. */
rsw_status rsw_fft_host(const void *h_in, void *h_out, void *h_scratch, int64_t n, int dtype, int inverse,
                        int64_t device_bytes, void *stream);

/* Transfer function of rsw_propagate and of simulations. RSW_PROP_FRESNEL is
 * the reference's (big-wave/propagation.py:124-128, fast-wave
 * fwcuda/kernels.cu:52) and the default. RSW_PROP_EXACT has no counterpart in
 * the reference: the exact angular-spectrum kernel exp(-i 2 pi dz
 * sqrt(1/wl^2 - f^2)), the constant -2 pi dz / wl taken out as for the
 * Fresnel kernel and the rest, 2 pi dz f^2 / (1/wl + sqrt(1/wl^2 - f^2)),
 * evaluated per sample in FP64; evanescent components (f^2 >= 1/wl^2) are
 * set to zero. Slower than the Fresnel kernel (no chirp factorisation). */
typedef enum { RSW_PROP_FRESNEL = 0, RSW_PROP_EXACT = 1 } rsw_propagator;
rsw_status rsw_plan_set_propagator(rsw_plan plan, int mode);

/* big-wave propagation.propagate (big-wave/propagation.py:100-138) and
 * fast-wave propagate<S> (fast-wave/src/simulation.cpp:34-40): u <- iFFT(H * FFT(u))
 * with H the Fresnel transfer function of distance dz and the big-wave frequency
 * cutoff; on return d_U holds FFT(u_new) in natural order (the reference's
 * postcondition). With skip_fft != 0, d_U must hold FFT(u) on entry and d_u is
 * only written. d_U may be NULL when skip_fft == 0: then the spectrum is not
 * stored (faster). */
rsw_status rsw_propagate(rsw_plan plan, void *d_u, void *d_U, double dx, double wl,
                         double dz, double cutoff_freq, int skip_fft, void *stream);

/* ------------------------------------------------------- transmission
 * The reference's per-element kernels (fast-wave/fwcuda/wrappers.hpp:9-39) with
 * big-wave's discrete semantics. x of sample i is built per chunk of
 * `chunk_size` samples exactly as big-wave's np.linspace does
 * (optical_element.py:352-354); chunk_size <= 0 means one chunk.
 * factor_a/factor_b are {re, im} pairs (the material factors of one sub-step). */
rsw_status rsw_apply_grating_factors(rsw_plan plan, void *d_u, double dx, int64_t chunk_size,
                                     double pitch, double dc, double x_position,
                                     const double factor_a[2], const double factor_b[2],
                                     void *stream);
rsw_status rsw_apply_dba_grating_factors(rsw_plan plan, void *d_u, double dx,
                                         int64_t chunk_size, double pitch0, double pitch1,
                                         double dc0, double dc1, double x_position,
                                         const double factor_a[2], const double factor_b[2],
                                         void *stream);
/* One z-row of a pixelised sample (big-wave/optical_element.py:432-476):
 * u *= exp(i 2 pi dz / wl * interp(x, row_x, row_db, left=0, right=0)).
 * h_row_db: host array of x_len {re, im} pairs (delta, beta) of the row. */
rsw_status rsw_apply_sample_row(rsw_plan plan, void *d_u, double dx, double wl, double dz,
                                double pixel_size_x, double x_position, int64_t x_len,
                                const double *h_row_db, void *stream);
/* u *= factor (fast-wave scale kernel, fwcuda/kernels.cu:160-172). */
rsw_status rsw_scale(rsw_plan plan, void *d_u, const double factor[2], void *stream);
/* Point-source field exp(-2 pi i r / wl)/sqrt(r) (big-wave/propagation.py:141-151). */
rsw_status rsw_point_source(rsw_plan plan, void *d_u, double dx, double wl, double z,
                            double x_source, void *stream);

/* --------------------------------------------------------- detection
 * square_and_downsample (big-wave/propagation.py:279-320): |u|^2 binned with
 * np.histogram semantics into n_pix = int(detector_size // pixel_size_x) pixels,
 * then scaled by cos(atan(x/z)) * dx * pixel_size_y / sqrt(x^2 + z^2).
 * d_out: device array of n_pix doubles. Returns n_pix through *n_pix_out when
 * non-NULL (d_out may then be NULL to query the size only). */
rsw_status rsw_square_and_downsample(rsw_plan plan, const void *d_u, double dx,
                                     double detector_size, double pixel_size_x,
                                     double pixel_size_y, double z, double *d_out,
                                     int64_t *n_pix_out, void *stream);

/* Host-only helper (no GPU needed): the detector geometry used by
 * rsw_square_and_downsample. bounds[j]..bounds[j+1] is the sample-index range
 * binned into pixel j (np.histogram semantics), cosv/rv the per-pixel
 * cos(atan(x/z)) and sqrt(x^2+z^2). Call with bounds == NULL to get n_pix. */
rsw_status rsw_detector_geometry(int64_t n, double dx, double detector_size,
                                 double pixel_size_x, double z, int64_t *n_pix,
                                 int64_t *bounds, double *cosv, double *rv);

/* ------------------------------------------------------ signal retrieval
 * Phase-stepping signal retrieval on the device: signal_retrieval_least_squares
 * of the reference's crack-simulation notebook (notebooks/Crack_simulation.ipynb,
 * cell 4), applied to detector output. d_data: [nsteps][n_pix] FP64, the layout
 * of detected.npy and rsw_sim_read. Phase steps phi_k = k * (2 pi nsteps /
 * period) / nsteps (np.linspace(0, 2 pi nsteps / period, nsteps, endpoint=False));
 * period = nsteps covers one fringe period. Per pixel, the least-squares fit
 * I_k = a sin(phi_k) + b cos(phi_k) + c gives
 *   d_abs = nsteps * c, d_phase = -atan2(a, b), d_vis = sqrt(a^2 + b^2) / c,
 *   d_chi2 = sum_k (I_k - fit_k)^2 (the notebook returns the mean over pixels).
 * Any output may be NULL. 3 <= nsteps <= 64; allocates nothing. */
rsw_status rsw_signal_retrieval(const double *d_data, int64_t n_pix, int nsteps, double period,
                                double *d_abs, double *d_phase, double *d_vis, double *d_chi2,
                                void *stream);

/* ---------------------------------------------------------- simulations
 * A whole per-source schedule (big-wave/wavesim.py:84-298, fast-wave
 * run_simulation_inner, src/simulation.cpp:375-549) run on the fused engine:
 * two HBM sweeps per split step, phase steps restarted from an in-HBM snapshot,
 * detector output accumulated in FP64 on the device.
 *
 * Elements are given as a flat description (rsw_element). Energy-dependent
 * inputs (wavelength, deltabeta values) are given per run. */
typedef enum { RSW_EL_GRATING = 0, RSW_EL_DBA_GRATING = 1, RSW_EL_SAMPLE = 2 } rsw_element_type;

typedef struct {
    int type;                    /* rsw_element_type                                   */
    double z_start;
    double thickness;            /* grating: height of the structure (no substrate)    */
    double substrate_thickness;
    int nr_steps;                /* grating sub-steps                                  */
    double pitch, pitch1;        /* grating pitch; DBA: pitch0, pitch1                 */
    double dc[2], dc1[2];        /* duty cycle (start, end); DBA: dc0, dc1             */
    int n_x_positions;
    const double *x_positions;   /* phase-step shifts (host memory, copied)           */
    /* sample */
    double pixel_size_x, pixel_size_z;
    int64_t grid_z, grid_x;      /* grid shape [z_len, x_len]                           */
    const int8_t *grid;          /* host int8 material indices (copied), 0 = vacuum    */
    int n_materials;             /* materials 1..n_materials                           */
} rsw_element;

typedef struct {
    int64_t n;
    int dtype;                   /* rsw_dtype */
    double dx;
    double z_detector;
    double detector_size;
    double pixel_size_x, pixel_size_y;
    int64_t chunk_size;          /* big-wave chunk_size (grating coordinates)            */
    int n_elements;
    const rsw_element *elements;
    const double *cutoff_angles; /* n_elements + 1                                       */
} rsw_sim_desc;

typedef enum { RSW_SRC_PLANE = 0, RSW_SRC_POINT = 1, RSW_SRC_VECTOR = 2 } rsw_source_type;

typedef struct {
    int type;                    /* rsw_source_type                                       */
    double x, z;                 /* point: position; plane/vector: z of the input field  */
    const void *h_field;         /* vector: host field (N complex of the sim dtype)       */
    const void *d_field;         /* vector: or a device field                             */
} rsw_source;

typedef struct {
    double energy_ev;            /* photon energy; wavelength = h c / (E e)               */
    /* deltabeta of every material as {delta, beta}, per element:
     * gratings: [a, b, substrate] (zeros for absent materials);
     * samples: [material 1 .. n_materials]. Concatenated in element order. */
    const double *deltabeta;
    int64_t n_deltabeta;         /* number of {delta, beta} pairs                       */
    double weight;               /* accumulation weight of this source's detector output */
    double wavelength_m;         /* > 0: use this wavelength instead of deriving it from energy_ev */
} rsw_source_run;

rsw_status rsw_sim_create(rsw_sim *out, const rsw_sim_desc *desc);
rsw_status rsw_sim_destroy(rsw_sim sim);
/* Shape of the detector output: nr_phase_steps x n_pix. */
rsw_status rsw_sim_shape(rsw_sim sim, int64_t *nr_phase_steps, int64_t *n_pix,
                         int64_t *split_steps_per_source);
/* Run one source and add weight * detected[phase][pix] to the device
 * accumulator. Asynchronous on `stream`. */
rsw_status rsw_sim_run(rsw_sim sim, const rsw_source *src, const rsw_source_run *run,
                       void *stream);
/* Run `count` sources (runs[0 .. count-1]: energies, deltabeta, weights) in
 * lockstep. srcs holds n_sources = 1 source description shared by all runs,
 * or one per run (n_sources = count); sources of one lockstep batch share
 * their type and z, and point positions and vector fields may differ (an
 * extended source spot). Replaces the reference's one run per
 * source (big-wave/wavesim.py:84-298 called once per energy by
 * big-wave/multisim.py:50-150; fast-wave's one invocation per source index,
 * fast-wave/Readme.md:22-26): every split step of all sources is one launch
 * per pass over count * N samples, each source an instance with its own
 * wavelength-dependent factors, transfer function and chirp table, and the
 * detector values are added in source order, as count rsw_sim_run calls would
 * add them. The sim keeps batch buffers of count * N samples (two with phase
 * stepping), sized for the largest batch run so far; where they would not fit
 * in four fifths of the device memory that is free or already held by them,
 * the sources run in consecutive lockstep chunks that do, with the same order
 * of accumulation. Lockstep needs a plan
 * of two or three levels, the Fresnel propagator, no history, no keypoints,
 * at least one element and a detector of at least one pixel, no final
 * fields (rsw_sim_set_final_fields) and sources of one type and z;
 * otherwise the sources run one after the other through rsw_sim_run. A batch keeps no
 * final field (rsw_sim_final_field). count <= RSW_BATCH_MAX.
 * d_each (device memory, may be NULL) receives each source's own detector
 * values as well, unweighted, source b's [phase][pix] at
 * d_each + b * nr_phase_steps * n_pix: the detected.npy of one source that
 * big-wave's run_single_simulation writes (big-wave/multisim.py:118-143). */
#define RSW_BATCH_MAX 4096
rsw_status rsw_sim_run_batch(rsw_sim sim, const rsw_source *srcs, int64_t n_sources,
                             const rsw_source_run *runs, int64_t count, double *d_each,
                             void *stream);
/* Zero the accumulator. */
rsw_status rsw_sim_reset(rsw_sim sim, void *stream);
/* Copy the accumulator (nr_phase_steps * n_pix doubles) to host memory;
 * synchronises `stream`. */
rsw_status rsw_sim_read(rsw_sim sim, double *h_out, void *stream);
/* Copy the accumulator to device memory (asynchronous on `stream`). */
rsw_status rsw_sim_read_device(rsw_sim sim, double *d_out, void *stream);
/* Device pointer of the accumulator (for peers / collectives). */
rsw_status rsw_sim_accumulator(rsw_sim sim, double **d_acc);
/* Copy the final field of the last phase step of the last run (natural order,
 * N complex of the sim dtype) to device memory. */
rsw_status rsw_sim_final_field(rsw_sim sim, void *d_dst, void *stream);

/* Per-kernel-kind device timing of the next rsw_sim_run calls (CUDA events on
 * the run's stream). kind: 0 = row pass, 1 = column pass, 2 = detection (the
 * last inverse column pass of each phase step, with the |u|^2 binning fused
 * in; the binning kernel alone for single-level plans), 3 = middle pass
 * (three-level plans, N above the two-level limit).
 * rsw_sim_timing returns the summed milliseconds and launch counts since
 * enabling; it synchronises. */
rsw_status rsw_sim_set_timing(rsw_sim sim, int enable);
rsw_status rsw_sim_timing(rsw_sim sim, int kind, double *ms, int64_t *launches);

/* History recording (big-wave/history.py:43-135, the reference's --history_dz):
 * with history_dz > 0, each following rsw_sim_run records detector images
 * (square_and_downsample at the image's z) on its first phase-step pass:
 * the analytic point-source intensity at np.arange(0, z_first, history_dz)[1:],
 * free-space gaps sampled every history_dz (each point propagated from the
 * gap's start, the last moved to the gap end when closer than history_dz/2),
 * after every grating sub-step and before every sample row. 0 disables.
 * rsw_sim_history copies the images of the last run as [n_pix][n_entries]
 * (np.stack(entries, axis=-1)) and their z to host memory; NULL outputs are
 * skipped; it synchronises. */
rsw_status rsw_sim_set_history(rsw_sim sim, double history_dz);
/* The transfer function of the following runs (rsw_propagator; default
 * RSW_PROP_FRESNEL, the reference's). */
rsw_status rsw_sim_set_propagator(rsw_sim sim, int mode);
rsw_status rsw_sim_history(rsw_sim sim, double *h_history, double *h_z, int64_t *n_entries,
                           void *stream);
/* Keypoints (replaces big-wave's save_keypoints_path, wavesim.py:35-55,
 * :186, :196): during the first phase-step pass of each following run, the
 * field in natural order right before element i is written to dst[2 i] and
 * right after it (grating sub-steps or sample slices done) to dst[2 i + 1].
 * dst holds n_dst = 2 * n_elements device buffers of N samples of the
 * simulation's dtype on its device (NULL entries are skipped); the pointers
 * are kept until the next call, and n_dst = 0 turns keypoints off. Each
 * keypoint costs one copy, or one inverse column pass where the field is held
 * in the passes' intermediate order. */
rsw_status rsw_sim_set_keypoints(rsw_sim sim, void *const *dst, int64_t n_dst);
/* Final fields of every phase step (replaces big-wave's save_u with
 * save_final_u_vectors, wavesim.py:58-82, called after each phase step at
 * :221-227 and :288-294): during each following run, the field at the
 * detector plane of phase step p is written in natural order to dst[p]. dst
 * holds n_dst = nr_phase_steps device buffers of N samples of the
 * simulation's dtype on its device (NULL entries are skipped); the pointers
 * are kept until the next call, and n_dst = 0 turns it off. The field is
 * written by the phase step's last pass, which then stores it instead of only
 * binning it. */
rsw_status rsw_sim_set_final_fields(rsw_sim sim, void *const *dst, int64_t n_dst);

#ifdef __cplusplus
}
#endif

#endif /* RSW_H */
