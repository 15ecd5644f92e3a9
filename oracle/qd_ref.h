/*
 * qd_ref.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Plain C interface of the CPU restatement of Zinq's grid split-operator
 * quantum-dynamics path (src/quantum_dynamics.zig, src/wavepacket.zig,
 * src/potential.zig, src/fourier_transform.zig, src/spectral_analysis.zig of
 * tjira/zinq).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs may load this library: it is the checker, never the product.
 *
 * Parity is pinned against the ten known-answer tests of
 * test/quantum_dynamics.zig:8-282 (final observables at 1e-8 absolute).
 */
#ifndef QD_REF_H
#define QD_REF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    QR_POT_HARMONIC = 0,
    QR_POT_TIME_LINEAR = 1,
    QR_POT_TULLY_1 = 2,
    QR_POT_TULLY_2 = 3,
    QR_POT_TULLY_3 = 4,
    QR_POT_CUSTOM = 5,
    QR_POT_LVC = 6,
    QR_POT_FILE = 7,
};

/* write-flag bits: which time series are recorded (Write, quantum_dynamics.zig:86-96) */
enum {
    QR_W_ACF = 1u << 0,
    QR_W_EKIN = 1u << 1,
    QR_W_MOM = 1u << 2,
    QR_W_NORM = 1u << 3,
    QR_W_POP = 1u << 4,
    QR_W_POS = 1u << 5,
    QR_W_EPOT = 1u << 6,
    QR_W_ETOT = 1u << 7,
    QR_W_WFN = 1u << 8,
};

typedef struct {
    int kind;
    /* harmonic: k[ndim]; time_linear: a, g; tully_1: A B C D; tully_2: A B C D E0; tully_3: A B C */
    const double* params;
    int nparams;
    /* custom: nstate*nstate expression strings, row-major */
    int custom_ndim;
    int custom_nstate;
    const char* const* exprs;
    int time_dependent;
    /* lvc */
    int lvc_nmode, lvc_nstate;
    const double* lvc_freq;   /* [nmode] cm^-1 */
    const double* lvc_exc;    /* [nstate] eV */
    const double* lvc_kappa;  /* [nstate][nmode] */
    const double* lvc_lambda; /* [nstate][nstate][nmode] */
    /* file: a readMatrix table, nrow x ncol row-major; first file_ndim columns are coordinates */
    int file_ndim;
    int file_nrow, file_ncol;
    const double* file_data;
} qr_potential;

typedef struct {
    int ndim;
    uint32_t npoint;
    const double* bounds; /* [ndim][2] */
    const double* mass;   /* [ndim] */
    double time_step;
    uint32_t iterations;
    uint32_t log_interval;
    const double* ic_position; /* [ndim] */
    const double* ic_momentum;
    const double* ic_gamma;
    uint32_t ic_state;
    int ic_adiabatic;
    int adiabatic;
    int has_cap;
    int cap_track_population;
    const double* cap_bounds; /* [ndim][2] */
    double cap_exponent;
    int cap_has_stop_norm;
    double cap_stop_norm;
    uint32_t imag_nstate; /* 0: real-time propagation */
    int has_spectrum;
    uint32_t spectrum_padding;
    double spectrum_threshold;
    uint32_t write_mask;
    int nthreads; /* OpenMP threads for per-point loops and FFT lines (results do not depend on it) */
    qr_potential pot;
    /* Chaining extension (no reference counterpart: its solve always starts from setGaussian):
       NULL, or nstate x npoint^ndim complex values (re, im interleaved, state-major) that
       replace the Gaussian; they are normalised like setGaussian's result. */
    const double* ic_wavefunction;
} qr_options;

typedef struct qr_result qr_result;

/* Runs a whole job; returns 0 on success, -1 for invalid input (error text via qr_last_error). */
int qr_run(const qr_options* opt, qr_result** out);
const char* qr_last_error(void);
void qr_free(qr_result* r);

int qr_nsolve(const qr_result* r);
int qr_nstate(const qr_result* r);
int qr_ndim(const qr_result* r);
size_t qr_npoint_total(const qr_result* r);
/* final observables of solve s (Observables.init with log=true, quantum_dynamics.zig:949) */
void qr_final(const qr_result* r, int s, double* pos, double* mom, double* pop, double* epot, double* ekin,
              double* norm, double* acf /* re,im or NaN */);
/* number of history rows recorded for solve s (iterations+1 unless stop_norm hit) */
size_t qr_hist_rows(const qr_result* r, int s);
/* copy one time series; name in {"pos","mom","pop","epot","ekin","etot","norm","acf"}; returns #cols or -1 */
int qr_hist(const qr_result* r, int s, const char* name, double* out);
/* final wavefunction of solve s: nstate x N complex (interleaved re,im) */
void qr_wavefunction(const qr_result* r, int s, double* out);
/* spectrum of solve s (calcSpectrum, spectral_analysis.zig:13-44): lengths, then data */
size_t qr_spectrum_len(const qr_result* r, int s, size_t* acf_padded_len);
void qr_spectrum(const qr_result* r, int s, double* acf_padded /* complex */, double* sigma);

/* ---- unit-level entry points used by the tests ---- */
/* eigendecomposition of one symmetric n x n matrix (row-major), LAPACK dsyevd('V', 'U')
   restated; W ascending; U[k*n+m] = component k of vector m */
void qr_eigh(int n, const double* V, double* W, double* U);
/* in-place N-D complex DFT (sign -1 forward unnormalised, +1 inverse with 1/N) */
void qr_fft(int ndim, const int* shape, int sign, double* data);
/* compile + evaluate one expression; returns 0 ok, -1 parse error */
int qr_expr_eval(const char* expr, int nvar, const double* vars, double t, double* value);

#ifdef __cplusplus
}
#endif
#endif
