// result.cu -- zqd_result accessors (Result / Observables / History of
// src/quantum_dynamics.zig:70-279) and the FFT, expression and eigen seams.
#include <cmath>
#include <cstring>

#include <cstdio>

#include "internal.h"
#include "line_kernel.cuh"

using namespace zqd;

extern "C" uint32_t zqd_result_nsolve(const zqd_result* r) { return r ? (uint32_t)r->solves.size() : 0; }

extern "C" int zqd_result_final(const zqd_result* r, uint32_t s, zqd_observables* out) {
    if (!r || !out) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (s >= r->solves.size()) return fail(ZQD_ERR_NOT_FOUND, "SOLVE INDEX OUT OF RANGE");
    const RowLayout L{(int)r->ndim, (int)r->nstate};
    const std::vector<double>& f = r->solves[s].fin;
    std::memset(out, 0, sizeof(*out));
    out->ndim = r->ndim;
    out->nstate = r->nstate;
    for (uint32_t i = 0; i < r->ndim; ++i) {
        out->pos[i] = f[L.pos() + i];
        out->mom[i] = f[L.mom() + i];
    }
    for (uint32_t i = 0; i < r->nstate; ++i) out->pop[i] = f[L.pop() + i];
    out->epot = f[L.epot()];
    out->ekin = f[L.ekin()];
    out->norm = f[L.norm()];
    out->acf_re = f[L.acf()];
    out->acf_im = f[L.acf() + 1];
    return ZQD_OK;
}

extern "C" int zqd_result_series(const zqd_result* rc, uint32_t s, zqd_series which, const double** data, size_t* rows,
                                 size_t* cols) {
    zqd_result* r = const_cast<zqd_result*>(rc);
    if (!r || !data || !rows || !cols) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (s >= r->solves.size()) return fail(ZQD_ERR_NOT_FOUND, "SOLVE INDEX OUT OF RANGE");
    const RowLayout L{(int)r->ndim, (int)r->nstate};
    uint32_t need = 0;
    int first = 0, width = 1;
    switch (which) {
    case ZQD_SERIES_POSITION: need = ZQD_WRITE_POSITION; first = L.pos(); width = (int)r->ndim; break;
    case ZQD_SERIES_MOMENTUM: need = ZQD_WRITE_MOMENTUM; first = L.mom(); width = (int)r->ndim; break;
    case ZQD_SERIES_POPULATION: need = ZQD_WRITE_POPULATION; first = L.pop(); width = (int)r->nstate; break;
    case ZQD_SERIES_POTENTIAL_ENERGY: need = ZQD_WRITE_POTENTIAL_ENERGY | ZQD_WRITE_TOTAL_ENERGY; first = L.epot(); break;
    case ZQD_SERIES_KINETIC_ENERGY: need = ZQD_WRITE_KINETIC_ENERGY | ZQD_WRITE_TOTAL_ENERGY; first = L.ekin(); break;
    case ZQD_SERIES_TOTAL_ENERGY: need = ZQD_WRITE_TOTAL_ENERGY; first = -1; break;
    case ZQD_SERIES_NORM: need = ZQD_WRITE_NORM; first = L.norm(); break;
    case ZQD_SERIES_ACF: need = ZQD_WRITE_ACF; first = L.acf(); width = 2; break;
    default: return fail(ZQD_ERR_INVALID_INPUT, "UNKNOWN SERIES");
    }
    if (!(r->write_mask & need)) return fail(ZQD_ERR_NOT_FOUND, "SERIES WAS NOT RECORDED (write option not set)");
    const SolveOut& so = r->solves[s];
    size_t key = (size_t)s * 16 + (size_t)which;
    if (r->series_cache.size() <= key) r->series_cache.resize(key + 1);
    std::vector<double>& v = r->series_cache[key];
    v.assign(so.rows * width, 0.0);
    for (size_t i = 0; i < so.rows; ++i) {
        const double* row = so.hist.data() + i * r->hc;
        if (first < 0) {
            v[i] = row[L.ekin()] + row[L.epot()]; // History.append: etot = ekin + epot (:206-208)
        } else {
            for (int c = 0; c < width; ++c) v[i * width + c] = row[first + c];
        }
    }
    *data = v.data();
    *rows = so.rows;
    *cols = (size_t)width;
    return ZQD_OK;
}

extern "C" int zqd_result_wavefunction(const zqd_result* r, uint32_t s, double* out, size_t capacity) {
    if (!r || !out) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (s >= r->solves.size()) return fail(ZQD_ERR_NOT_FOUND, "SOLVE INDEX OUT OF RANGE");
    const std::vector<double>& p = r->solves[s].psi;
    if (p.empty()) return fail(ZQD_ERR_NOT_FOUND, "THE FINAL WAVEFUNCTION WAS NOT DOWNLOADED (server option)");
    if (capacity < p.size()) return fail(ZQD_ERR_INVALID_INPUT, "OUTPUT BUFFER TOO SMALL");
    std::memcpy(out, p.data(), p.size() * sizeof(double));
    return ZQD_OK;
}

extern "C" int zqd_result_spectrum(const zqd_result* r, uint32_t s, const double** acf_padded, size_t* nacf,
                                   const double** sigma, size_t* nsigma) {
    if (!r) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (s >= r->solves.size()) return fail(ZQD_ERR_NOT_FOUND, "SOLVE INDEX OUT OF RANGE");
    const SolveOut& so = r->solves[s];
    if (so.acfpad.empty()) return fail(ZQD_ERR_NOT_FOUND, "NO SPECTRUM WAS COMPUTED");
    if (acf_padded) *acf_padded = so.acfpad.data();
    if (nacf) *nacf = so.acfpad.size() / 2;
    if (sigma) *sigma = so.sigma.data();
    if (nsigma) *nsigma = so.sigma.size();
    return ZQD_OK;
}

extern "C" double zqd_result_device_ms(const zqd_result* r) { return r ? r->device_ms : 0.0; }
extern "C" int zqd_result_precision(const zqd_result* r) { return r ? (int)r->precision : -1; }

namespace {
// writeMatrixLspace (src/read_write.zig:115-136): "rows cols+1", then per row the grid value
// start + step i (step = (end - start) / (rows - 1), 0 for one row) and the row's values
int write_lspace(const char* path, const double* v, size_t rows, size_t cols, double start, double end) {
    FILE* f = std::fopen(path, "w");
    if (!f) return zqd::fail(ZQD_ERR_INVALID_INPUT, std::string("CANNOT OPEN ") + path);
    std::vector<char> buf(1 << 16);
    std::setvbuf(f, buf.data(), _IOFBF, buf.size());
    std::fprintf(f, "%zu %zu\n", rows, cols + 1);
    const double step = rows > 1 ? (end - start) / (double)(rows - 1) : 0.0;
    for (size_t i = 0; i < rows; ++i) {
        std::fprintf(f, "%20.14f ", start + step * (double)i);
        for (size_t c = 0; c < cols; ++c) std::fprintf(f, "%20.14f%s", v[i * cols + c], c + 1 == cols ? "\n" : " ");
    }
    const bool ok = std::fflush(f) == 0;
    std::fclose(f);
    return ok ? ZQD_OK : zqd::fail(ZQD_ERR_INVALID_INPUT, std::string("WRITE FAILED: ") + path);
}
} // namespace

extern "C" int zqd_result_wavefunction_series(const zqd_result* r, uint32_t s, double* out, size_t capacity, size_t* rows,
                                              size_t* npoint_total) {
    if (!r) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (s >= r->solves.size()) return fail(ZQD_ERR_NOT_FOUND, "SOLVE INDEX OUT OF RANGE");
    const SolveOut& so = r->solves[s];
    if (so.wfn.empty()) return fail(ZQD_ERR_NOT_FOUND, "SERIES WAS NOT RECORDED (write option not set)");
    if (rows) *rows = so.rows;
    if (npoint_total) *npoint_total = r->npoint_total;
    if (out) {
        if (capacity < so.wfn.size()) return fail(ZQD_ERR_INVALID_INPUT, "OUTPUT BUFFER TOO SMALL");
        std::memcpy(out, so.wfn.data(), so.wfn.size() * sizeof(double));
    }
    return ZQD_OK;
}

extern "C" int zqd_result_export(const zqd_result* r, uint32_t s, const zqd_write_paths* paths) {
    if (!r || !paths) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (s >= r->solves.size()) return fail(ZQD_ERR_NOT_FOUND, "SOLVE INDEX OUT OF RANGE");
    const SolveOut& so = r->solves[s];
    const double end = r->time_step * (double)(so.rows > 0 ? so.rows - 1 : 0);
    const struct {
        const char* path;
        zqd_series which;
    } series[] = {{paths->acf, ZQD_SERIES_ACF},
                  {paths->position, ZQD_SERIES_POSITION},
                  {paths->momentum, ZQD_SERIES_MOMENTUM},
                  {paths->population, ZQD_SERIES_POPULATION},
                  {paths->potential_energy, ZQD_SERIES_POTENTIAL_ENERGY},
                  {paths->kinetic_energy, ZQD_SERIES_KINETIC_ENERGY},
                  {paths->norm, ZQD_SERIES_NORM},
                  {paths->total_energy, ZQD_SERIES_TOTAL_ENERGY}};
    int rc;
    for (const auto& e : series) {
        if (!e.path) continue;
        const double* data = nullptr;
        size_t rows = 0, cols = 0;
        if ((rc = zqd_result_series(r, s, e.which, &data, &rows, &cols))) return rc;
        if ((rc = write_lspace(e.path, data, rows, cols, 0.0, end))) return rc;
    }
    if (paths->wavefunction) { // writeMatrixHjoin(grid.r, wfn, 2 nstate index) (quantum_dynamics.zig:253-255)
        if (so.wfn.empty()) return fail(ZQD_ERR_NOT_FOUND, "SERIES WAS NOT RECORDED (write option not set)");
        const size_t N = r->npoint_total, S = r->nstate, d = r->ndim, n = (size_t)r->grid[2 * d];
        FILE* f = std::fopen(paths->wavefunction, "w");
        if (!f) return fail(ZQD_ERR_INVALID_INPUT, std::string("CANNOT OPEN ") + paths->wavefunction);
        std::vector<char> buf(1 << 16);
        std::setvbuf(f, buf.data(), _IOFBF, buf.size());
        std::fprintf(f, "%zu %zu\n", N, d + 2 * S * so.rows);
        for (size_t g = 0; g < N; ++g) {
            size_t q = g;
            double x[3];
            for (size_t l = 0; l < d; ++l) { // Grid.init (wavepacket.zig:55-74)
                const size_t j = d - l - 1;
                const double lo = r->grid[2 * j], hi = r->grid[2 * j + 1];
                x[j] = lo + (double)(q % n) * (hi - lo) / (double)n;
                q /= n;
            }
            for (size_t j = 0; j < d; ++j) std::fprintf(f, "%20.14f ", x[j]);
            for (size_t t = 0; t < so.rows; ++t)
                for (size_t s2 = 0; s2 < S; ++s2) {
                    const size_t e = (t * S + s2) * N + g;
                    const bool last = t + 1 == so.rows && s2 + 1 == S;
                    std::fprintf(f, "%20.14f %20.14f%s", so.wfn[2 * e], so.wfn[2 * e + 1], last ? "\n" : " ");
                }
        }
        const bool ok = std::fflush(f) == 0;
        std::fclose(f);
        if (!ok) return fail(ZQD_ERR_INVALID_INPUT, std::string("WRITE FAILED: ") + paths->wavefunction);
    }
    if (paths->spectrum_acf || paths->spectrum) {
        if (so.acfpad.empty()) return fail(ZQD_ERR_NOT_FOUND, "NO SPECTRUM WAS COMPUTED");
        const size_t lp = so.acfpad.size() / 2;
        if (paths->spectrum_acf) { // time axis extended by the padding (quantum_dynamics.zig:267-270)
            const double pad = r->time_step * (double)(lp - so.rows);
            if ((rc = write_lspace(paths->spectrum_acf, so.acfpad.data(), lp, 2, 0.0, end + pad))) return rc;
        }
        if (paths->spectrum) { // frequency axis from -pi/dt (quantum_dynamics.zig:271-275)
            const double nyquist = 3.14159265358979323846 / r->time_step, nt = (double)so.sigma.size();
            if ((rc = write_lspace(paths->spectrum, so.sigma.data(), so.sigma.size(), 1, -nyquist,
                                   nyquist * (nt - 2) / nt)))
                return rc;
        }
    }
    return ZQD_OK;
}

extern "C" int zqd_result_transfer_bytes(const zqd_result* r, uint64_t* h2d, uint64_t* d2h) {
    if (!r) return fail(ZQD_ERR_INVALID_INPUT, "NULL RESULT");
    if (h2d) *h2d = r->h2d;
    if (d2h) *d2h = r->d2h;
    return ZQD_OK;
}
extern "C" void zqd_result_destroy(zqd_result* r) { delete r; }

// ------------------------------------------------------------ expression seam
struct zqd_expr {
    ExprProgram prog;
    size_t nvar = 0;
};

extern "C" int zqd_expr_compile(const char* text, size_t len, size_t nvar, zqd_expr** out) {
    if (!text || !out) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    *out = nullptr;
    std::unique_ptr<zqd_expr> e(new zqd_expr());
    std::string err;
    if (!compile_expression(std::string(text, len), (int)nvar, e->prog, err)) return fail(ZQD_ERR_EXPRESSION, err);
    e->nvar = nvar;
    *out = e.release();
    return ZQD_OK;
}

__global__ void expr_points_kernel(const uint32_t* code, const double* consts, const double* r, int nvar, size_t npts,
                                   double t, double* out) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= npts) return;
    out[i] = vm_eval(code, consts, r + i * nvar, t);
}

extern "C" int zqd_expr_eval_points(const zqd_expr* e, const double* host_r, size_t npts, double t, double* host_out) {
    if (!e || (!host_r && e->nvar) || !host_out) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (npts == 0) return ZQD_OK;
    uint32_t* dc = nullptr;
    double *dk = nullptr, *dr = nullptr, *dout = nullptr;
    std::vector<double> consts = e->prog.consts;
    if (consts.empty()) consts.push_back(0);
    size_t nr = npts * (e->nvar ? e->nvar : 1);
    int rc = ZQD_OK;
    auto cleanup = [&] {
        cudaFree(dc);
        cudaFree(dk);
        cudaFree(dr);
        cudaFree(dout);
    };
    cudaError_t err = cudaMalloc(&dc, e->prog.code.size() * sizeof(uint32_t));
    if (!err) err = cudaMalloc(&dk, consts.size() * sizeof(double));
    if (!err) err = cudaMalloc(&dr, nr * sizeof(double));
    if (!err) err = cudaMalloc(&dout, npts * sizeof(double));
    if (!err) err = cudaMemcpy(dc, e->prog.code.data(), e->prog.code.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (!err) err = cudaMemcpy(dk, consts.data(), consts.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (!err && e->nvar) err = cudaMemcpy(dr, host_r, nr * sizeof(double), cudaMemcpyHostToDevice);
    if (!err) {
        expr_points_kernel<<<(unsigned)((npts + 127) / 128), 128>>>(dc, dk, dr, (int)e->nvar, npts, t, dout);
        err = cudaGetLastError();
    }
    if (!err) err = cudaMemcpy(host_out, dout, npts * sizeof(double), cudaMemcpyDeviceToHost);
    if (err) rc = fail(ZQD_ERR_DEVICE, cudaGetErrorString(err));
    cleanup();
    return rc;
}

extern "C" void zqd_expr_destroy(zqd_expr* e) { delete e; }

// ------------------------------------------------------------ eigen seam
template <int S> __global__ void eigh_batch_kernel(const double* V, double* W, double* U, size_t count) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= count) return;
    double v[S * S], w[S], u[S * S];
    for (int e = 0; e < S * S; ++e) v[e] = V[i * S * S + e];
    eigh_dev<S>(v, w, u);
    for (int e = 0; e < S; ++e) W[i * S + e] = w[e];
    for (int e = 0; e < S * S; ++e) U[i * S * S + e] = u[e];
}

// potential_plot.run (src/potential_plot.zig:48-106): V(r, t) at every point of Grid.init's grid
// (wavepacket.zig:55-74), or with `adiabatic` the eigenvalues on the diagonal and zeros elsewhere
template <int S>
static __global__ void potential_plot_kernel(const __grid_constant__ PotDev pot, int d, int n, size_t N, double3 lo,
                                             double3 span, double t,
                                             int adiabatic, double* __restrict__ U, double* __restrict__ R) {
    const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (g >= N) return;
    double r[3] = {0, 0, 0};
    const double los[3] = {lo.x, lo.y, lo.z}, sps[3] = {span.x, span.y, span.z};
    size_t q = g;
    for (int l = 0; l < d; ++l) {
        const int j = d - l - 1;
        r[j] = __dadd_rn(los[j], __dmul_rn((double)(q % (size_t)n), sps[j]) / (double)n);
        q /= (size_t)n;
    }
    for (int j = 0; j < d; ++j) R[g * d + j] = r[j];
    double V[S * S];
    pot_eval(pot, r, t, V);
    if (adiabatic) {
        double Vu[S * S], W[S], Uv[S * S];
        for (int a = 0; a < S; ++a)
            for (int b = 0; b < S; ++b) Vu[a * S + b] = V[(a < b ? a : b) * S + (a < b ? b : a)];
        eigh_dev<S>(Vu, W, Uv);
        for (int e = 0; e < S * S; ++e) V[e] = 0.0;
        for (int a = 0; a < S; ++a) V[a * S + a] = W[a];
    }
    for (int e = 0; e < S * S; ++e) U[g * S * S + e] = V[e];
}

extern "C" int zqd_potential_plot(const zqd_options* opt, double time, double* host_U, size_t capacity,
                                  const char* write_path) {
    if (!opt) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    // only the grid and the potential are read; the propagation fields may be left unset
    static const double zeros[3] = {0, 0, 0}, ones[3] = {1, 1, 1};
    zqd_options in = *opt;
    if (!in.ic_position) in.ic_position = zeros;
    if (!in.ic_momentum) in.ic_momentum = zeros;
    if (!in.ic_gamma) in.ic_gamma = ones;
    if (!in.mass) in.mass = ones;
    Opts o;
    int rc = copy_options(&in, o);
    if (rc) return rc;
    if (o.ndim == 0 || o.ndim > ZQD_MAX_NDIM) return fail(ZQD_ERR_UNSUPPORTED, "GRID DIMENSION MUST BE 1..3");
    if (o.npoint == 0) return fail(ZQD_ERR_INVALID_INPUT, "GRID POINT COUNT MUST BE GREATER THAN 0");
    if ((uint32_t)o.pot_nd != o.ndim) return fail(ZQD_ERR_INVALID_INPUT, "POTENTIAL DIMENSION DOES NOT MATCH GRID DIMENSION");
    if (o.pot_ns < 1 || o.pot_ns > ZQD_MAX_NSTATE) return fail(ZQD_ERR_UNSUPPORTED, "MORE THAN 4 ELECTRONIC STATES ARE NOT SUPPORTED");
    const int d = (int)o.ndim, S = o.pot_ns, n = (int)o.npoint;
    size_t N = 1;
    for (int j = 0; j < d; ++j) N *= (size_t)n;
    if (host_U && capacity < N * S * S) return fail(ZQD_ERR_INVALID_INPUT, "OUTPUT BUFFER TOO SMALL");
    PotStore ps;
    if ((rc = build_potential(o, ps))) return rc;
    double3 lo = make_double3(0, 0, 0), span = make_double3(0, 0, 0);
    double* los = &lo.x;
    double* sps = &span.x;
    for (int j = 0; j < d; ++j) {
        los[j] = o.bounds[2 * j];
        sps[j] = o.bounds[2 * j + 1] - o.bounds[2 * j];
    }
    double *dU = nullptr, *dR = nullptr;
    cudaError_t err = dev_alloc((void**)&dU, N * S * S * sizeof(double));
    if (!err) err = dev_alloc((void**)&dR, N * d * sizeof(double));
    std::vector<double> U(N * S * S), R(N * d);
    if (!err) {
        const unsigned b = (unsigned)((N + 127) / 128);
        const int adia = o.adiabatic ? 1 : 0;
        switch (S) {
        case 1: potential_plot_kernel<1><<<b, 128>>>(ps.dev, d, n, N, lo, span, time, adia, dU, dR); break;
        case 2: potential_plot_kernel<2><<<b, 128>>>(ps.dev, d, n, N, lo, span, time, adia, dU, dR); break;
        case 3: potential_plot_kernel<3><<<b, 128>>>(ps.dev, d, n, N, lo, span, time, adia, dU, dR); break;
        default: potential_plot_kernel<4><<<b, 128>>>(ps.dev, d, n, N, lo, span, time, adia, dU, dR); break;
        }
        err = cudaGetLastError();
    }
    if (!err) err = cudaMemcpy(U.data(), dU, U.size() * sizeof(double), cudaMemcpyDeviceToHost);
    if (!err) err = cudaMemcpy(R.data(), dR, R.size() * sizeof(double), cudaMemcpyDeviceToHost);
    dev_free(dU);
    dev_free(dR);
    if (err) return fail(ZQD_ERR_DEVICE, cudaGetErrorString(err));
    if (host_U) std::memcpy(host_U, U.data(), U.size() * sizeof(double));
    if (write_path) { // writeMatrixHjoin(grid.r, U) (src/read_write.zig:79-110)
        FILE* f = std::fopen(write_path, "w");
        if (!f) return fail(ZQD_ERR_INVALID_INPUT, std::string("CANNOT OPEN ") + write_path);
        std::vector<char> buf(1 << 16);
        std::setvbuf(f, buf.data(), _IOFBF, buf.size());
        std::fprintf(f, "%zu %zu\n", N, (size_t)(d + S * S));
        for (size_t g = 0; g < N; ++g) {
            for (int j = 0; j < d; ++j) std::fprintf(f, "%20.14f ", R[g * d + j]);
            for (int e = 0; e < S * S; ++e) std::fprintf(f, "%20.14f%s", U[g * S * S + e], e + 1 == S * S ? "\n" : " ");
        }
        const bool ok = std::fflush(f) == 0;
        std::fclose(f);
        if (!ok) return fail(ZQD_ERR_INVALID_INPUT, std::string("WRITE FAILED: ") + write_path);
    }
    return ZQD_OK;
}

extern "C" int zqd_eigh_batch(uint32_t n, size_t count, const double* hV, double* hW, double* hU) {
    if (n == 0 || n > ZQD_MAX_NSTATE) return fail(ZQD_ERR_UNSUPPORTED, "MATRIX ORDER MUST BE 1..4");
    if (!hV || !hW || !hU) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (count == 0) return ZQD_OK;
    double *dV = nullptr, *dW = nullptr, *dU = nullptr;
    cudaError_t err = cudaMalloc(&dV, count * n * n * sizeof(double));
    if (!err) err = cudaMalloc(&dW, count * n * sizeof(double));
    if (!err) err = cudaMalloc(&dU, count * n * n * sizeof(double));
    if (!err) err = cudaMemcpy(dV, hV, count * n * n * sizeof(double), cudaMemcpyHostToDevice);
    if (!err) {
        unsigned b = (unsigned)((count + 127) / 128);
        switch (n) {
        case 1: eigh_batch_kernel<1><<<b, 128>>>(dV, dW, dU, count); break;
        case 2: eigh_batch_kernel<2><<<b, 128>>>(dV, dW, dU, count); break;
        case 3: eigh_batch_kernel<3><<<b, 128>>>(dV, dW, dU, count); break;
        default: eigh_batch_kernel<4><<<b, 128>>>(dV, dW, dU, count); break;
        }
        err = cudaGetLastError();
    }
    if (!err) err = cudaMemcpy(hW, dW, count * n * sizeof(double), cudaMemcpyDeviceToHost);
    if (!err) err = cudaMemcpy(hU, dU, count * n * n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dV);
    cudaFree(dW);
    cudaFree(dU);
    if (err) return fail(ZQD_ERR_DEVICE, cudaGetErrorString(err));
    return ZQD_OK;
}
