/*
 * zinq_qd.h -- C-ABI of the B200-native split-operator wavepacket propagator.
 *
 * Drop-in for Zinq's grid quantum-dynamics path (tjira/zinq).  Every entry
 * point below names the reference interface it replaces.  Plain C99: no CUDA,
 * torch or C++ types cross this boundary; device memory is owned by the
 * library.  A Zig host imports it the way src/cimport.zig:3-8 imports FFTW
 * and ExprTk: `@cImport(@cInclude("zinq_qd.h"))`.
 *
 * Status codes: 0 is success, negative values mirror the reference's Zig
 * error set (error.InvalidInput, error.OutOfMemory, error.PlanCreationFailed,
 * error.LapackError, ExprTk's null return) plus device-side conditions.
 */
#ifndef ZINQ_QD_H
#define ZINQ_QD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZQD_ABI_VERSION 1
#define ZQD_MAX_NDIM 3
#define ZQD_MAX_NSTATE 4

typedef enum {
    ZQD_OK = 0,
    ZQD_ERR_INVALID_INPUT = -1, /* error.InvalidInput, src/quantum_dynamics.zig:606-710 */
    ZQD_ERR_OUT_OF_MEMORY = -2, /* error.OutOfMemory (host allocation) */
    ZQD_ERR_DEVICE_OOM = -3,    /* device allocation refused / not enough free HBM */
    ZQD_ERR_PLAN_FAILED = -4,   /* error.PlanCreationFailed, src/fourier_transform.zig:22 */
    ZQD_ERR_EIGEN_FAILED = -5,  /* error.LapackError, src/linear_algebra.zig:69 */
    ZQD_ERR_EXPRESSION = -6,    /* exprtk_init returned null, src/exprtk.cpp:21-23 */
    ZQD_ERR_UNSUPPORTED = -7,   /* valid for the reference, outside this build's limits */
    ZQD_ERR_DEVICE = -8,        /* CUDA runtime error */
    ZQD_ERR_TIMEOUT = -9,       /* a bounded device or host wait ran out */
    ZQD_ERR_CANCELLED = -10,    /* job cancelled through the server */
    ZQD_ERR_NOT_FOUND = -11,    /* unknown job id or result index */
    ZQD_ERR_NO_DEVICE = -12,    /* no CUDA device with sm_100 */
    ZQD_ERR_NUMERIC = -13       /* a served job's norm or populations became NaN or Inf */
} zqd_status;

/* Human-readable text of a status code; the last failing call's detail
   (e.g. "MASS MUST BE GREATER THAN 0") is available from zqd_last_error(). */
const char* zqd_status_string(int status);
const char* zqd_last_error(void);

/* ------------------------------------------------------------------ options
 * zqd_options mirrors `Options` (src/quantum_dynamics.zig:25-67),
 * `InitialConditions` (src/wavepacket.zig:16-23) and the potential `Options`
 * union (src/potential.zig:19-60).  Arrays are pointer + implied length
 * (ndim, nstate); the library deep-copies everything it keeps.
 */
typedef enum {
    ZQD_POT_HARMONIC = 0,    /* src/potential.zig:143-175 */
    ZQD_POT_TIME_LINEAR = 1, /* :178-215 */
    ZQD_POT_TULLY_1 = 2,     /* :218-261 */
    ZQD_POT_TULLY_2 = 3,     /* :264-314 */
    ZQD_POT_TULLY_3 = 4,     /* :317-361 */
    ZQD_POT_CUSTOM = 5,      /* :364-451, expressions as in src/exprtk.cpp:10-40 */
    ZQD_POT_LVC = 6,         /* :493-575 */
    ZQD_POT_FILE = 7         /* :454-490, table as read by src/read_write.zig:24-56 */
} zqd_potential_kind;

typedef struct {
    zqd_potential_kind kind;
    /* harmonic: k[ndim] (default {1}) */
    const double* harmonic_k;
    uint32_t harmonic_ndim;
    /* time_linear: a (10), g (2); tully_1: A B C D; tully_2: A B C D E0; tully_3: A B C */
    double p[5];
    /* custom: nstate x nstate NUL-terminated expressions, row-major */
    const char* const* custom_matrix;
    uint32_t custom_nstate;
    uint32_t custom_ndim;
    int custom_time_dependent;
    /* lvc: frequencies[nmode] cm^-1, excitation_energies[nstate] eV,
       kappa[nstate][nmode], lambda[nstate][nstate][nmode] */
    const double* lvc_frequencies;
    uint32_t lvc_nmode;
    const double* lvc_excitation_energies;
    uint32_t lvc_nstate;
    const double* lvc_kappa;
    const double* lvc_lambda;
    /* file: nrow x ncol row-major table; the first file_ndim columns are coordinates */
    const double* file_table;
    uint32_t file_nrow;
    uint32_t file_ncol;
    uint32_t file_ndim;
} zqd_potential;

/* bits of zqd_options.write_mask: which time series are recorded (Write, src/quantum_dynamics.zig:86-96) */
enum {
    ZQD_WRITE_ACF = 1u << 0,
    ZQD_WRITE_KINETIC_ENERGY = 1u << 1,
    ZQD_WRITE_MOMENTUM = 1u << 2,
    ZQD_WRITE_NORM = 1u << 3,
    ZQD_WRITE_POPULATION = 1u << 4,
    ZQD_WRITE_POSITION = 1u << 5,
    ZQD_WRITE_POTENTIAL_ENERGY = 1u << 6,
    ZQD_WRITE_TOTAL_ENERGY = 1u << 7,
    ZQD_WRITE_WAVEFUNCTION = 1u << 8
};

typedef enum {
    ZQD_FP64 = 0,       /* plain form: complex FP64 throughout */
    ZQD_FP32_MIXED = 1, /* FP32 state, butterflies and phases; FP64 tables, eigh and reductions */
    ZQD_PRECISION_AUTO = 2 /* per job at creation: ZQD_FP32_MIXED, or ZQD_FP64 when the smallest gap
                              between adiabatic surfaces on the grid (at t = 0) is below
                              ZQD_AUTO_GAP_THRESHOLD, where FP32 rounding of the state accumulates
                              in the population transfer of a near-degenerate crossing.  Not valid
                              for zqd_fft_* */
} zqd_precision;

/* Smallest adiabatic gap (Hartree) that ZQD_PRECISION_AUTO propagates in FP32. */
#define ZQD_AUTO_GAP_THRESHOLD 1e-3

typedef struct {
    uint32_t struct_size; /* sizeof(zqd_options); set by zqd_options_init */
    /* grid */
    uint32_t ndim;
    uint32_t npoint;
    const double* grid_bounds; /* [ndim][2] */
    /* initial_conditions */
    const double* ic_position; /* [ndim] */
    const double* ic_momentum; /* [ndim] */
    const double* ic_gamma;    /* [ndim] */
    uint32_t ic_state;
    int ic_adiabatic;
    /* potential */
    zqd_potential potential;
    /* propagation */
    double time_step;
    uint32_t iterations;
    const double* mass; /* [ndim] */
    uint32_t write_mask;
    int adiabatic;
    uint32_t log_interval;
    /* absorbing_potential (optional) */
    int has_absorbing_potential;
    int cap_track_population;
    const double* cap_bounds; /* [ndim][2] */
    double cap_exponent;      /* default 0.001 */
    int cap_has_stop_norm;
    double cap_stop_norm;
    /* fft.plan: accepted for schema compatibility; planning effort has no effect here */
    int fft_plan;
    /* imaginary (optional): number of relaxed states, 0 for real-time propagation */
    uint32_t imaginary_nstate;
    /* spectrum (optional) */
    int has_spectrum;
    uint32_t spectrum_padding;
    double spectrum_threshold; /* default 1e-6 */
    /* this build */
    zqd_precision precision;
    int log; /* compute every observable on log steps, like run(..., log=true) */
    /* Initial wavefunction (this build; the reference has no such input, its solve always starts
       from setGaussian, src/quantum_dynamics.zig:867).  NULL: the Gaussian of initial_conditions.
       Otherwise nstate x npoint^ndim complex values (re, im interleaved, state-major, last axis
       fastest) that replace the Gaussian; the solve then normalises them and applies toDia when
       ic_adiabatic, as after setGaussian.  Chains an imaginary-time relaxation into real time. */
    const double* ic_wavefunction;
} zqd_options;

/* Fills the reference's field defaults (log_interval 1, cap exponent 0.001,
   spectrum threshold 1e-6, fft.plan measure, FP64, harmonic potential). */
void zqd_options_init(zqd_options* opt);
/* Sets a potential's kind and the reference's default constants for it
   (src/potential.zig:24-48: harmonic k {1}; time_linear a 10 g 2; Tully 1/2/3). */
void zqd_potential_init(zqd_potential* pot, zqd_potential_kind kind);

/* ------------------------------------------------------------------ results
 * zqd_result mirrors Result(T) (src/quantum_dynamics.zig:70-83): one
 * Observables entry per imaginary-time state (or one for real time), plus the
 * recorded time series (History, :99-279).  Owned by the library until
 * zqd_result_destroy (the reference's Result.deinit).
 */
typedef struct zqd_result zqd_result;

typedef enum {
    ZQD_SERIES_POSITION = 0, /* rows x ndim */
    ZQD_SERIES_MOMENTUM = 1, /* rows x ndim */
    ZQD_SERIES_POPULATION = 2,
    ZQD_SERIES_POTENTIAL_ENERGY = 3,
    ZQD_SERIES_KINETIC_ENERGY = 4,
    ZQD_SERIES_TOTAL_ENERGY = 5,
    ZQD_SERIES_NORM = 6,
    ZQD_SERIES_ACF = 7 /* rows x 2 (re, im) */
} zqd_series;

typedef struct {
    uint32_t ndim, nstate;
    double pos[ZQD_MAX_NDIM];
    double mom[ZQD_MAX_NDIM];
    double pop[ZQD_MAX_NSTATE];
    double epot, ekin, norm;
    double acf_re, acf_im; /* NaN unless the autocorrelation is recorded */
} zqd_observables;

uint32_t zqd_result_nsolve(const zqd_result* res);
/* final Observables of solve s (Observables.init with log=true, src/quantum_dynamics.zig:949) */
int zqd_result_final(const zqd_result* res, uint32_t solve, zqd_observables* out);
/* one recorded time series; *rows = iterations+1 unless stop_norm ended the solve early */
int zqd_result_series(const zqd_result* res, uint32_t solve, zqd_series which, const double** data, size_t* rows,
                      size_t* cols);
/* final wavefunction of solve s, nstate x npoint^ndim complex (re, im interleaved), state-major */
int zqd_result_wavefunction(const zqd_result* res, uint32_t solve, double* host_out, size_t capacity_doubles);
/* spectrum of solve s (calcSpectrum, src/spectral_analysis.zig:13-44) */
int zqd_result_spectrum(const zqd_result* res, uint32_t solve, const double** acf_padded, size_t* nacf,
                        const double** sigma, size_t* nsigma);
/* GPU time of the propagation kernels of the whole run, milliseconds (CUDA events) */
double zqd_result_device_ms(const zqd_result* res);
/* The precision the job ran in (ZQD_FP64 or ZQD_FP32_MIXED; ZQD_PRECISION_AUTO resolved), -1 for NULL. */
int zqd_result_precision(const zqd_result* res);

/* History.exportWrite (src/quantum_dynamics.zig:218-277): the recorded time series of solve
   `solve` written as the reference's .mat text (writeMatrixLspace, src/read_write.zig:115-136:
   a "rows cols" line, then per row the time 0 .. dt (rows - 1) and the values, each "%20.14f",
   space-separated), and with the spectrum option the padded autocorrelation (time 0 .. dt
   (rows - 1 + padding)) and the spectrum (frequency -pi/dt .. pi/dt (M - 2)/M).  A NULL path
   skips that file; a series that was not recorded returns ZQD_ERR_NOT_FOUND. */
typedef struct {
    const char* acf;
    const char* position;
    const char* momentum;
    const char* population;
    const char* potential_energy;
    const char* kinetic_energy;
    const char* norm;
    const char* total_energy;
    const char* spectrum_acf;
    const char* spectrum;
    const char* wavefunction; /* writeMatrixHjoin(grid.r, History.wfn): per grid point its coordinates, then
                                 re, im of every state at every recorded step */
} zqd_write_paths;
int zqd_result_export(const zqd_result* res, uint32_t solve, const zqd_write_paths* paths);
/* write.wavefunction history of solve `solve` (History.append, src/quantum_dynamics.zig:176-180; in
   the adiabatic basis when `adiabatic`): rows x nstate x npoint_total complex values (re, im),
   copied into out when capacity (doubles) suffices; out may be NULL to query the shape. */
int zqd_result_wavefunction_series(const zqd_result* res, uint32_t solve, double* out, size_t capacity, size_t* rows,
                                   size_t* npoint_total);
void zqd_result_destroy(zqd_result* res);

/* --------------------------------------------------------------- method API
 * zqd_run replaces `quantum_dynamics.run(comptime T, io, opt, log, gpa)`
 * (src/quantum_dynamics.zig:567-603): validation identical to
 * checkInvalidInput (:606-710), setup (:713-749), one solve per
 * imaginary-time state (:582-598) on the GPU.
 */
int zqd_run(const zqd_options* opt, zqd_result** out);

/* Staged form of zqd_run: create (validate, upload, build the potential and
   phase tables on the device), solve, fetch.  A job handle is used by one
   host thread at a time. */
typedef struct zqd_job zqd_job;
int zqd_job_create(const zqd_options* opt, zqd_job** out);
int zqd_job_run(zqd_job* job);                           /* every solve, device-resident, no host copies */
int zqd_job_result(zqd_job* job, zqd_result** out);      /* device -> host copy of observables */
int zqd_job_info(const zqd_job* job, uint32_t* ndim, uint32_t* nstate, uint64_t* npoint_total,
                 uint32_t* cluster_ctas, size_t* device_bytes);
/* Launch shapes of a 2-D or 3-D job's axis passes (no counterpart in the reference: the reference
   has no device passes; for tests and tuning).  tma_row_*: the TMA-staged persistent row pass (rows
   per block, CTAs, threads), all 0 when the per-block kernel takes every row launch; tma_tile_*: the
   TMA-staged persistent tile pass (lines per tile, CTAs, threads), all 0 when the per-block kernel
   runs; rows_per_cta, tile_lines: the per-block kernels' shapes (the launches the TMA-staged forms do
   not take).  ZQD_ERR_UNSUPPORTED for a 1-D job. */
typedef struct {
    uint32_t tma_row_block, tma_row_ctas, tma_row_threads;
    uint32_t tma_tile_lines, tma_tile_ctas, tma_tile_threads;
    uint32_t rows_per_cta, tile_lines;
} zqd_nd_shape;
int zqd_job_nd_shape(const zqd_job* job, zqd_nd_shape* out);
/* device time (ms, CUDA events on the job's stream) of the last zqd_job_run (or of every
   zqd_job_step call of the current step-wise run) */
double zqd_job_device_ms(const zqd_job* job);
void zqd_job_destroy(zqd_job* job);

/* Step-wise form of zqd_job_run, the solve loop of src/quantum_dynamics.zig:860-950 cut into
   pieces.  The first call of a run records row 0 (the initial state, after setGaussian and
   toDia) and then propagates nsteps steps; every later call propagates up to nsteps more.  A call
   ends at the end of a solve (iterations reached, or stop_norm, :933-944) and runs the solve's
   final Observables.init (:949); with imaginary.nstate > 1 the next call starts the next solve.
   The wavefunction stays on the device between calls.  zqd_job_run restarts from the beginning. */
int zqd_job_step(zqd_job* job, uint32_t nsteps);
/* the solve in progress (the last one once finished), its rows recorded so far, and whether every
   solve has ended (zqd_job_result needs that) */
int zqd_job_progress(const zqd_job* job, uint32_t* solve, uint32_t* rows, int* finished);

/* One observables row per recorded step, as History.append records them
   (src/quantum_dynamics.zig:174-215): width = 5 + 2 ndim + nstate doubles,
     [0] norm, [1 .. ndim] position, [1 + ndim .. 2 ndim] momentum,
     [1 + 2 ndim .. 2 ndim + nstate] population,
     [1 + 2 ndim + nstate] potential energy, [2 + 2 ndim + nstate] kinetic energy,
     [3 + 2 ndim + nstate] acf re, [4 + 2 ndim + nstate] acf im,
   NaN where the option set does not record the value (total energy = potential + kinetic). */
typedef struct {
    uint32_t solve;       /* solve (imaginary-time state) of these rows */
    uint32_t first_row;   /* step index of rows[0] */
    uint32_t nrows;       /* 0: nothing new */
    uint32_t width;       /* doubles per row */
    const double* rows;   /* nrows x width, owned by the job, valid until its next call */
    int solve_finished;   /* the solve's last row is among these (or was returned earlier) */
} zqd_obs_rows;
/* The rows recorded since the previous call (of one solve; call again for the next solve).
   Works after zqd_job_step and after zqd_job_run. */
int zqd_job_observables(zqd_job* job, zqd_obs_rows* out);

/* ------------------------------------------------------------ autotuner
 * (no counterpart in the reference, whose FFTW planner is the nearest thing: fft.plan,
 * src/fourier_transform.zig:15-23).  Launch shapes per key (dims, points per axis, states,
 * precision): the 1-D resident kernel's CTAs per cluster and largest local radix, the N-D
 * passes' rows per row-pass CTA and lines per tile-pass CTA.  zqd_autotune times every shape the
 * kernels accept for the key on the current device (a synthetic job of that size, CUDA events)
 * and records the fastest in the process's table, which job creation consults; the file named by
 * the environment variable ZQD_TUNE_FILE is loaded before the first job.  A tuned shape only
 * refactors the transforms, so results stay within the parity bars of the default shape.
 */
typedef struct {
    uint32_t ndim, npoint, nstate; /* the key (in) */
    zqd_precision precision;       /* ZQD_FP64 or ZQD_FP32_MIXED (in) */
    /* out: the chosen shape (0: the built-in rules' choice was fastest), its time per step and the
       rules' time per step, and how many candidate shapes the kernels accepted */
    uint32_t cluster_ctas, radix_log2, rows_per_cta, tile_lines;
    double us_per_step, default_us_per_step;
    uint32_t candidates;
    /* out, N-D: the TMA-staged persistent passes' shapes, rows per row block and lines per tile
       (0: the rules' choice, -1: the per-block kernel instead) */
    int32_t tma_row_block, tma_tile_lines;
} zqd_tune_entry;
int zqd_autotune(zqd_tune_entry* entry);
int zqd_tune_save(const char* path); /* text: one "ndim npoint nstate fp32 C radix_log2 rows tile" line per key */
int zqd_tune_load(const char* path); /* merges a saved table into the process's table */
void zqd_tune_clear(void);
uint32_t zqd_tune_size(void);

/* Several independent jobs advanced together on the device (the batched
   form): one launch per group of jobs with equal kernel shape and precision,
   cluster i of the grid running job i.  results[i] receives the result of
   opts[i].  Replaces a loop of quantum_dynamics.run calls. */
int zqd_run_batch(const zqd_options* const* opts, uint32_t njobs, zqd_result** results);

/* Staged form of zqd_run_batch: tables of every job built once at create;
   each zqd_batch_run propagates all jobs again from their initial state with
   no host copies.  zqd_batch_launches reports the kernel launches of the last
   run. */
typedef struct zqd_batch zqd_batch;
int zqd_batch_create(const zqd_options* const* opts, uint32_t njobs, zqd_batch** out);
int zqd_batch_run(zqd_batch* batch);
int zqd_batch_result(zqd_batch* batch, uint32_t index, zqd_result** out);
double zqd_batch_device_ms(const zqd_batch* batch);
uint32_t zqd_batch_launches(const zqd_batch* batch);
void zqd_batch_destroy(zqd_batch* batch);

/* Bytes the library copied host->device and device->host for this result
   (options, tables and descriptors in; observables and wavefunctions out). */
int zqd_result_transfer_bytes(const zqd_result* res, uint64_t* h2d, uint64_t* d2h);

/* ------------------------------------------------------------ FFT seam
 * Replaces FftPlan(T) (src/fourier_transform.zig:8-49: fftw_plan_dft,
 * fftw_execute_dft, fftw_destroy_plan): in-place N-D complex transform of a
 * device buffer, sign -1 unnormalised forward, +1 inverse followed by 1/N.
 * Square grids n^ndim with n a power of two from 2 to 8192.
 */
typedef struct zqd_fft zqd_fft;
int zqd_fft_plan_create(uint32_t ndim, const int* shape, int sign, zqd_precision precision, zqd_fft** out);
int zqd_fft_execute(zqd_fft* plan, void* device_inout, void* cuda_stream);
void zqd_fft_destroy(zqd_fft* plan);

/* No counterpart in the reference: the same transform as a plan's
   zqd_fft_execute for callers that must not allocate device memory (code
   running inside a framework's memory pool, or a host that owns one fixed
   arena and forbids cudaMalloc/cudaFree).  The twiddle table lives in a
   static 128 KiB device array of the library (held on every GPU that loads
   it until exit), so n is at most 8192; larger n returns ZQD_ERR_UNSUPPORTED.
   The first call on a device looks the array's address up once
   (cudaGetSymbolAddress); make that first call before any stream capture.
   That address is kept for the life of the process: the entry point assumes
   the CUDA runtime's primary context of the device and no cudaDeviceReset
   between calls (after one, the kept address is stale).  Every call rewrites
   the shared table on `cuda_stream`, so calls that overlap on the GPU race with
   one another.  Allocates nothing. */
int zqd_fft_execute_noalloc(uint32_t ndim, const int* shape, int sign, zqd_precision precision, void* device_inout,
                            void* cuda_stream);

/* --------------------------------------------------------- expression seam
 * Replaces exprtk_init / exprtk_evaluate_d0 / exprtk_deinit
 * (src/exprtk.h:1-10, src/exprtk.cpp:10-40): compiles an expression over
 * r1..r<nvar> and t into device bytecode.  A parse error returns
 * ZQD_ERR_EXPRESSION where ExprTk returned null.
 */
typedef struct zqd_expr zqd_expr;
int zqd_expr_compile(const char* text, size_t len, size_t nvar, zqd_expr** out);
/* evaluates on the device for npts coordinate rows (host arrays r[npts][nvar]) */
int zqd_expr_eval_points(const zqd_expr* e, const double* host_r, size_t npts, double t, double* host_out);
void zqd_expr_destroy(zqd_expr* e);

/* ------------------------------------------------------------ eigen seam
 * Replaces eighBatch (src/linear_algebra.zig:28-42, LAPACKE_dsyevd row-major
 * 'V','U' at :67) with the device FP64 solver; exposed for parity tests.
 * W ascending, U[k*n+m] = component k of eigenvector m.
 */
int zqd_eigh_batch(uint32_t n, size_t count, const double* host_V, double* host_W, double* host_U);

/* ------------------------------------------------------------ potential plot
 * potential_plot.run (src/potential_plot.zig:48-106) on the device: V(r, time) at every point of
 * the grid of opt (grid_bounds, npoint, potential; `adiabatic` puts the eigenvalues on the
 * diagonal and zeros elsewhere).  host_U: npoint^ndim x nstate^2 values (may be NULL);
 * write_path: the reference's .mat file (coordinates, then the matrix, "%20.14f"), or NULL.
 * Only the grid, potential and adiabatic fields of opt are read.
 */
int zqd_potential_plot(const zqd_options* opt, double time, double* host_U, size_t capacity, const char* write_path);

/* ------------------------------------------------------------------ server
 * A request loop around quantum_dynamics.run for streams of independent jobs
 * (the reference runs one job per process and has no counterpart).
 * Submission validates and copies the options (errors come back at once, with
 * the reference's messages).  Worker threads admit requests in arrival order
 * while their estimated device memory fits the budget and the device's free
 * memory (measured with cudaMemGetInfo plus the blocks the library's memory pool
 * keeps).  A worker advances its jobs in launches of stream_steps steps:
 * 1-D single-solve requests of the same precision, state count and grid size
 * share each launch of the resident line kernel, every job at its own step;
 * between launches finished or cancelled jobs leave and waiting requests of the
 * same shape join (continuous batching).  After every launch each job's new
 * observable rows are posted as an event; zqd_server_poll pulls events (nothing
 * is called back).  1-D single-solve requests whose line fits one CTA run instead
 * on the persistent line-service kernel: resident CTAs claim requests from a job
 * table in pinned memory as they are posted, keep each wavefunction in shared
 * memory for its whole solve and publish every observable row as it is written
 * (a cancelled request there finishes its solve and is then reported cancelled).
 * Results equal those of zqd_run on the same options, within the parity bars of
 * the launch shape (bit for bit where the shapes agree).
 */
typedef struct zqd_server zqd_server;
typedef struct {
    uint32_t struct_size;         /* sizeof(zqd_server_config); set by zqd_server_config_init */
    uint32_t workers;             /* host threads, each advancing one job or group at a time on its own stream (default 8) */
    uint32_t max_batch;           /* jobs per grouped launch (default 16) */
    uint64_t device_budget_bytes; /* 0: 90% of the device memory free at creation */
    uint32_t stream_steps;        /* steps per launch between event posts (default 256; 0: whole jobs) */
    int stream_rows;              /* post ZQD_EVENT_ROWS events with the observable rows (default 1) */
    uint32_t max_events;          /* events kept for zqd_server_poll (default 65536); beyond it the oldest
                                     row events are dropped and counted, completion events never */
    int persistent_lines;         /* 1-D single-solve requests whose line fits one CTA (npoint <= 2048 FP32,
                                     1024 FP64) run on the persistent line-service kernel (default 1) */
    uint32_t service_ctas;        /* CTAs alive per service table (default 64, 0: one per SM); a table
                                     per (precision, states, CTA size): small lines share an SM */
    double service_idle_us;       /* a service CTA without work exits after this wait (default 200) */
    int fetch_wavefunction;       /* results carry the final wavefunction (default 1; 0 saves its download,
                                     zqd_result_wavefunction then returns ZQD_ERR_NOT_FOUND) */
} zqd_server_config;
typedef struct {
    uint64_t submitted, completed, failed, cancelled, queued;
    uint64_t grouped_launches, grouped_jobs, joined_jobs; /* joined: admitted into a group already on the GPU */
    uint64_t device_budget_bytes, device_bytes_in_use, peak_device_bytes;
    uint64_t pending_events, dropped_events;
    uint64_t service_jobs, service_launches; /* requests run by the persistent kernel; its launches */
} zqd_server_stats;
typedef enum {
    ZQD_EVENT_ROWS = 0,     /* new observable rows of a running job (zqd_obs_rows layout) */
    ZQD_EVENT_DONE = 1,     /* finished; zqd_server_wait returns the result */
    ZQD_EVENT_FAILED = 2,   /* status says why; zqd_server_wait returns it */
    ZQD_EVENT_CANCELLED = 3 /* cancelled before it finished */
} zqd_event_kind;
typedef struct {
    uint64_t ticket;
    int kind;   /* zqd_event_kind */
    int status; /* 0, or the failure's status code */
    uint32_t solve, first_row, nrows, width;
    int solve_finished;
    const double* rows; /* nrows x width (ZQD_EVENT_ROWS), valid until the next zqd_server_poll */
} zqd_event;
void zqd_server_config_init(zqd_server_config* cfg);
int zqd_server_create(const zqd_server_config* cfg, zqd_server** out);
int zqd_server_submit(zqd_server* server, const zqd_options* opt, uint64_t* ticket);
/* Blocks until the request is done; returns its result (owned by the caller) and its latency
   from submission to completion.  A ticket is waited for once. */
int zqd_server_wait(zqd_server* server, uint64_t ticket, zqd_result** out, double* latency_ms);
/* The same, giving up with ZQD_ERR_TIMEOUT after timeout_ms (the request stays waitable). */
int zqd_server_wait_timeout(zqd_server* server, uint64_t ticket, uint32_t timeout_ms, zqd_result** out,
                            double* latency_ms);
/* A queued request is dropped at once; a running one leaves before its next launch.  Its
   zqd_server_wait then returns ZQD_ERR_CANCELLED (a request already done keeps its result). */
int zqd_server_cancel(zqd_server* server, uint64_t ticket);
/* Moves up to max_events pending events into events[], oldest first; *count receives how many. */
int zqd_server_poll(zqd_server* server, zqd_event* events, uint32_t max_events, uint32_t* count);
int zqd_server_stats_get(zqd_server* server, zqd_server_stats* out);
/* waits for every submitted request, then frees the server */
void zqd_server_destroy(zqd_server* server);

/* Fault injection for tests of the failure paths (no effect unless called): after `after` more
   successful device allocations, the next `count` ones fail as if the device were out of memory. */
void zqd_testing_fail_device_allocations(uint64_t after, uint64_t count);
/* Launches the server's persistent line-service kernel with `ctas` CTAs and posts nothing: every
   CTA's wait for work runs out of its clock64 budget (idle_us) and it exits.  *idle_exits receives
   the CTAs that left that way, *wall_ms the host time until the kernel had ended. */
int zqd_testing_service_idle(zqd_precision precision, uint32_t nstate, uint32_t ctas, double idle_us,
                             uint32_t* idle_exits, double* wall_ms);
/* The next `launches` launches of the 2-D / 3-D TMA-staged axis passes issue no first tile load in
   any CTA and bound their mbarrier waits by wait_us: every CTA's first wait runs out, the kernel
   records it in the job's error word and returns, and the run fails with ZQD_ERR_DEVICE (the
   context stays usable).  Tests the failure path of the waits without a device fault. */
int zqd_testing_tma_withhold_load(uint32_t launches, double wait_us);

/* ------------------------------------------------------------------ device */
int zqd_device_count(void);
int zqd_set_device(int device);

/* On-chip denominators for the roofline of the resident 1-D kernel, whose wavefunction stays in
   shared memory (no counterpart in the reference): the shared-memory bandwidth of one SM with every
   SM busy (128-bit loads and stores, no bank conflicts), and the latency of __syncthreads in a
   256-thread CTA and of a barrier across a 16-CTA cluster, measured on the current device. */
typedef struct {
    double smem_bytes_per_cycle_per_sm, smem_gbs_per_sm;
    double syncthreads_cycles, cluster_barrier_cycles;
    double sm_clock_mhz; /* the device's maximum SM clock */
    uint32_t sms;
} zqd_onchip;
int zqd_measure_onchip(zqd_onchip* out);

#ifdef __cplusplus
}
#endif
#endif /* ZINQ_QD_H */
