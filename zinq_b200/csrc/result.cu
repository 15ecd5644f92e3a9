// result.cu -- zqd_result accessors (Result / Observables / History of
// src/quantum_dynamics.zig:70-279) and the FFT, expression and eigen seams.
#include <cmath>
#include <cstring>

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
