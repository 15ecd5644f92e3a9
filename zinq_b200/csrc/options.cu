// options.cu -- option deep copy, validation (checkInvalidInput,
// src/quantum_dynamics.zig:606-710), potential upload and twiddle tables.
#include <cmath>
#include <cstring>
#include <memory>
#include <atomic>
#include <mutex>
#include <unordered_map>

#include "internal.h"

namespace zqd {

static thread_local std::string g_error;

void set_error(const std::string& msg) { g_error = msg; }
int fail(int status, const std::string& msg) {
    g_error = msg;
    return status;
}
const char* last_error() { return g_error.c_str(); }

int copy_options(const zqd_options* in, Opts& o) {
    if (!in) return fail(ZQD_ERR_INVALID_INPUT, "NULL OPTIONS");
    if (in->struct_size != 0 && in->struct_size != sizeof(zqd_options))
        return fail(ZQD_ERR_INVALID_INPUT, "zqd_options.struct_size does not match this library (rebuild the caller)");
    o.ndim = in->ndim;
    o.npoint = in->npoint;
    const uint32_t d = in->ndim;
    if (d > 0 && (!in->grid_bounds || !in->ic_position || !in->ic_momentum || !in->ic_gamma || !in->mass))
        return fail(ZQD_ERR_INVALID_INPUT, "GRID BOUNDS, INITIAL CONDITIONS AND MASS ARRAYS MUST NOT BE NULL");
    o.bounds.assign(in->grid_bounds, in->grid_bounds + 2 * d);
    o.pos.assign(in->ic_position, in->ic_position + d);
    o.mom.assign(in->ic_momentum, in->ic_momentum + d);
    o.gamma.assign(in->ic_gamma, in->ic_gamma + d);
    o.mass.assign(in->mass, in->mass + d);
    o.ic_state = in->ic_state;
    o.ic_adiabatic = in->ic_adiabatic != 0;
    o.time_step = in->time_step;
    o.iterations = in->iterations;
    o.write_mask = in->write_mask;
    o.adiabatic = in->adiabatic != 0;
    o.log_interval = in->log_interval;
    o.log = in->log != 0;
    o.has_cap = in->has_absorbing_potential != 0;
    if (o.has_cap) {
        if (!in->cap_bounds) return fail(ZQD_ERR_INVALID_INPUT, "ABSORBING POTENTIAL BOUNDS MUST NOT BE NULL");
        o.cap_bounds.assign(in->cap_bounds, in->cap_bounds + 2 * d);
        o.cap_track = in->cap_track_population != 0;
        o.cap_exponent = in->cap_exponent;
        o.cap_has_stop = in->cap_has_stop_norm != 0;
        o.cap_stop_norm = in->cap_stop_norm;
    }
    o.imag_nstate = in->imaginary_nstate;
    o.has_spectrum = in->has_spectrum != 0;
    o.spectrum_padding = in->spectrum_padding;
    o.spectrum_threshold = in->spectrum_threshold;
    o.precision = in->precision;
    const zqd_potential& p = in->potential;
    o.pkind = (int)p.kind;
    switch (p.kind) {
    case ZQD_POT_HARMONIC:
        if (p.harmonic_ndim == 0 || !p.harmonic_k) o.harmonic_k = {1.0};
        else o.harmonic_k.assign(p.harmonic_k, p.harmonic_k + p.harmonic_ndim);
        o.pot_nd = (int)o.harmonic_k.size();
        o.pot_ns = 1;
        break;
    case ZQD_POT_TIME_LINEAR:
        std::memcpy(o.p, p.p, sizeof(o.p));
        o.pot_nd = 1;
        o.pot_ns = 2;
        o.pot_td = true;
        break;
    case ZQD_POT_TULLY_1:
    case ZQD_POT_TULLY_2:
    case ZQD_POT_TULLY_3:
        std::memcpy(o.p, p.p, sizeof(o.p));
        o.pot_nd = 1;
        o.pot_ns = 2;
        break;
    case ZQD_POT_CUSTOM:
        if (!p.custom_matrix || p.custom_nstate == 0) return fail(ZQD_ERR_INVALID_INPUT, "CUSTOM POTENTIAL MATRIX IS EMPTY");
        for (uint32_t i = 0; i < p.custom_nstate * p.custom_nstate; ++i) {
            if (!p.custom_matrix[i]) return fail(ZQD_ERR_INVALID_INPUT, "CUSTOM POTENTIAL EXPRESSION IS NULL");
            o.custom.emplace_back(p.custom_matrix[i]);
        }
        o.custom_ns = p.custom_nstate;
        o.custom_nd = p.custom_ndim;
        o.custom_td = p.custom_time_dependent != 0;
        o.pot_nd = (int)p.custom_ndim;
        o.pot_ns = (int)p.custom_nstate;
        o.pot_td = o.custom_td;
        break;
    case ZQD_POT_LVC: {
        uint32_t nm = p.lvc_nmode, ns = p.lvc_nstate;
        if (!p.lvc_frequencies || !p.lvc_excitation_energies || !p.lvc_kappa || !p.lvc_lambda || nm == 0 || ns == 0)
            return fail(ZQD_ERR_INVALID_INPUT, "LVC POTENTIAL ARRAYS MUST NOT BE EMPTY");
        o.lvc_freq.assign(p.lvc_frequencies, p.lvc_frequencies + nm);
        o.lvc_exc.assign(p.lvc_excitation_energies, p.lvc_excitation_energies + ns);
        o.lvc_kappa.assign(p.lvc_kappa, p.lvc_kappa + (size_t)ns * nm);
        o.lvc_lambda.assign(p.lvc_lambda, p.lvc_lambda + (size_t)ns * ns * nm);
        o.pot_nd = (int)nm;
        o.pot_ns = (int)ns;
        break;
    }
    case ZQD_POT_FILE: {
        if (!p.file_table || p.file_nrow == 0 || p.file_ncol <= p.file_ndim)
            return fail(ZQD_ERR_INVALID_INPUT, "FILE POTENTIAL TABLE IS EMPTY");
        o.file_table.assign(p.file_table, p.file_table + (size_t)p.file_nrow * p.file_ncol);
        o.file_nrow = p.file_nrow;
        o.file_ncol = p.file_ncol;
        o.file_nd = p.file_ndim;
        o.pot_nd = (int)p.file_ndim;
        double ns = std::sqrt((double)(p.file_ncol - p.file_ndim));
        o.pot_ns = (int)ns;
        if ((uint32_t)(o.pot_ns * o.pot_ns) != p.file_ncol - p.file_ndim)
            return fail(ZQD_ERR_INVALID_INPUT, "FILE POTENTIAL COLUMN COUNT IS NOT NDIM + NSTATE^2");
        break;
    }
    default:
        return fail(ZQD_ERR_INVALID_INPUT, "UNKNOWN POTENTIAL KIND");
    }
    if (in->ic_wavefunction && o.ndim >= 1 && o.ndim <= ZQD_MAX_NDIM && o.pot_ns >= 1 && o.pot_ns <= ZQD_MAX_NSTATE &&
        o.npoint >= 1 && o.npoint <= (1u << 24)) {
        size_t N = 1;
        for (uint32_t i = 0; i < o.ndim; ++i) N *= o.npoint;
        o.ic_wfn.assign(in->ic_wavefunction, in->ic_wavefunction + 2 * (size_t)o.pot_ns * N);
    }
    return ZQD_OK;
}

// The reference's checks, in its order and with its messages; then the
// shape checks the reference leaves to assertions; then this build's limits.
int validate(const Opts& o) {
    auto bad = [](const char* m) { return fail(ZQD_ERR_INVALID_INPUT, m); };
    if (!(o.time_step > 0)) return bad("TIME STEP MUST BE GREATER THAN 0");
    for (double m : o.mass)
        if (!(m > 0)) return bad("MASS MUST BE GREATER THAN 0");
    if (o.mass.size() != o.pos.size()) return bad("MASS VECTOR MUST HAVE THE SAME LENGTH AS POSITION VECTOR");
    if (o.log_interval == 0) return bad("LOG INTERVAL MUST BE GREATER THAN 0");
    if (o.npoint == 0) return bad("GRID POINT COUNT MUST BE GREATER THAN 0");
    if (o.ndim == 0) return bad("GRID BOUNDS MUST NOT BE EMPTY");
    for (uint32_t i = 0; i < o.ndim; ++i)
        if (!(o.bounds[2 * i] < o.bounds[2 * i + 1])) return bad("GRID BOUNDS MIN MUST BE LESS THAN MAX");
    if (o.pos.empty()) return bad("INITIAL POSITION VECTOR MUST NOT BE EMPTY");
    if (o.mom.size() != o.pos.size()) return bad("INITIAL MOMENTUM AND POSITION VECTORS MUST HAVE THE SAME LENGTH");
    if (o.gamma.size() != o.pos.size()) return bad("INITIAL GAMMA VECTOR MUST HAVE THE SAME LENGTH AS POSITION VECTOR");
    if (o.pos.size() != o.ndim) return bad("INITIAL CONDITIONS DIMENSION DOES NOT MATCH GRID DIMENSION");
    if (o.has_cap) {
        if (o.cap_bounds.size() != 2 * (size_t)o.ndim)
            return bad("ABSORBING POTENTIAL BOUNDS DIMENSION DOES NOT MATCH GRID DIMENSION");
        for (uint32_t i = 0; i < o.ndim; ++i) {
            double c0 = o.cap_bounds[2 * i], c1 = o.cap_bounds[2 * i + 1];
            if (c0 < o.bounds[2 * i] || c1 > o.bounds[2 * i + 1] || c0 >= c1)
                return bad("ABSORBING POTENTIAL BOUNDS MUST LIE WITHIN GRID BOUNDS AND CB[0] < CB[1]");
        }
        if (!(o.cap_exponent > 0)) return bad("ABSORBING POTENTIAL EXPONENT MUST BE GREATER THAN 0");
        if (o.cap_has_stop && (o.cap_stop_norm <= 0 || o.cap_stop_norm >= 1))
            return bad("ABSORBING POTENTIAL STOP_NORM MUST BE BETWEEN 0 AND 1");
    }
    if (o.has_spectrum && (o.spectrum_threshold <= 0 || o.spectrum_threshold >= 1))
        return bad("SPECTRUM THRESHOLD MUST BE BETWEEN 0 AND 1");
    // shape consistency the reference asserts (src/potential.zig:99-101, wavepacket.zig:367)
    if ((uint32_t)o.pot_nd != o.ndim) return bad("POTENTIAL DIMENSION DOES NOT MATCH GRID DIMENSION");
    if (o.ic_state >= (uint32_t)o.pot_ns) return bad("INITIAL STATE INDEX OUT OF RANGE");
    // this build's limits
    if (o.ndim > ZQD_MAX_NDIM) return fail(ZQD_ERR_UNSUPPORTED, "MORE THAN 3 GRID DIMENSIONS ARE NOT SUPPORTED");
    if (o.pot_ns > ZQD_MAX_NSTATE) return fail(ZQD_ERR_UNSUPPORTED, "MORE THAN 4 ELECTRONIC STATES ARE NOT SUPPORTED");
    if ((o.npoint & (o.npoint - 1)) != 0 || o.npoint < 4)
        return fail(ZQD_ERR_UNSUPPORTED, "GRID POINT COUNT MUST BE A POWER OF TWO (>= 4)");
    if (o.precision != ZQD_FP64 && o.precision != ZQD_FP32_MIXED && o.precision != ZQD_PRECISION_AUTO)
        return bad("UNKNOWN PRECISION");
    // custom expressions must compile (Custom.init fails like exprtk_init returning null)
    for (size_t e = 0; e < o.custom.size(); ++e) {
        ExprProgram prog;
        std::string err;
        if (!compile_expression(o.custom[e], (int)o.custom_nd, prog, err))
            return fail(ZQD_ERR_EXPRESSION, "EXPRESSION V[" + std::to_string(e / o.custom_ns) + "][" +
                                                 std::to_string(e % o.custom_ns) + "] \"" + o.custom[e] + "\": " + err);
    }
    if (o.write_mask & ZQD_WRITE_WAVEFUNCTION) { // History.wfn: (iterations + 1) x nstate x N complex per solve
        double N = 1;
        for (uint32_t i = 0; i < o.ndim; ++i) N *= (double)o.npoint;
        const double bytes = ((double)o.iterations + 1) * o.pot_ns * N * 16.0 * (o.imag_nstate ? o.imag_nstate : 1);
        if (bytes > 32.0 * 1024 * 1024 * 1024)
            return fail(ZQD_ERR_UNSUPPORTED, "WAVEFUNCTION TIME SERIES LARGER THAN 32 GiB");
    }
    return ZQD_OK;
}

// Host-side fault injection (zqd_testing_fail_device_allocations): after g_alloc_skip more
// successful device allocations, the next g_alloc_fail ones report cudaErrorMemoryAllocation.
static std::atomic<long long> g_alloc_skip{-1}, g_alloc_fail{0};

static bool injected_alloc_failure() {
    if (g_alloc_skip.load(std::memory_order_relaxed) < 0) return false;
    if (g_alloc_skip.fetch_sub(1) > 0) return false;
    g_alloc_skip.store(0);
    if (g_alloc_fail.fetch_sub(1) > 0) return true;
    g_alloc_skip.store(-1); // disarmed
    g_alloc_fail.store(0);
    return false;
}

cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st) {
    if (injected_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    static std::mutex mu;
    static bool configured[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev >= 0 && dev < 64 && !configured[dev]) { // keep freed blocks for reuse instead of releasing them
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                uint64_t keep = UINT64_MAX;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
            configured[dev] = true;
        }
    }
    if (st) return cudaMallocAsync(p, bytes, st);
    e = cudaMallocAsync(p, bytes, cudaStreamPerThread);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread); // usable from any stream after this
    return e;
}

void dev_free(void* p, cudaStream_t st) {
    if (p) cudaFreeAsync(p, st ? st : cudaStreamPerThread);
}

size_t device_free_bytes() {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int dev = 0;
    cudaMemPool_t pool;
    uint64_t reserved = 0, used = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
        free_b += (size_t)(reserved - used); // blocks the pool keeps for reuse
    return free_b;
}

void PotStore::release() {
    dev_free(d_blob, st);
    d_blob = nullptr;
}

// one device block for the potential's data: one allocation and one copy
static int upload_blob(PotStore& ps, const std::vector<double>& blob) {
    if (blob.empty()) return ZQD_OK;
    const size_t b = blob.size() * sizeof(double);
    const cudaStream_t st = ps.st ? ps.st : cudaStreamPerThread;
    ZQD_CUDA(dev_alloc(&ps.d_blob, b, st));
    ZQD_CUDA(cudaMemcpyAsync(ps.d_blob, blob.data(), b, cudaMemcpyHostToDevice, st));
    ZQD_CUDA(cudaStreamSynchronize(st));
    ps.bytes += b;
    return ZQD_OK;
}

int build_potential(const Opts& o, PotStore& ps, cudaStream_t st) {
    ps.release();
    ps.st = st;
    PotDev& P = ps.dev;
    std::memset(&P, 0, sizeof(P));
    P.kind = o.pkind;
    P.nd = o.pot_nd;
    P.ns = o.pot_ns;
    P.td = o.pot_td ? 1 : 0;
    switch (o.pkind) {
    case ZQD_POT_HARMONIC:
        for (size_t i = 0; i < o.harmonic_k.size() && i < 8; ++i) P.prm[i] = o.harmonic_k[i];
        break;
    case ZQD_POT_TIME_LINEAR:
    case ZQD_POT_TULLY_1:
    case ZQD_POT_TULLY_2:
    case ZQD_POT_TULLY_3:
        for (int i = 0; i < 5; ++i) P.prm[i] = o.p[i];
        break;
    case ZQD_POT_CUSTOM: {
        std::vector<uint32_t> code;
        std::vector<double> consts;
        for (size_t e = 0; e < o.custom.size(); ++e) {
            ExprProgram prog;
            std::string err;
            if (!compile_expression(o.custom[e], (int)o.custom_nd, prog, err))
                return fail(ZQD_ERR_EXPRESSION, "EXPRESSION V[" + std::to_string(e / o.custom_ns) + "][" +
                                                     std::to_string(e % o.custom_ns) + "] \"" + o.custom[e] +
                                                     "\": " + err);
            P.code_off[e] = (int)code.size();
            P.const_off[e] = (int)consts.size();
            code.insert(code.end(), prog.code.begin(), prog.code.end());
            consts.insert(consts.end(), prog.consts.begin(), prog.consts.end());
        }
        if (consts.empty()) consts.push_back(0.0);
        // constants first, then the program (two 32-bit words per double slot)
        std::vector<double> blob(consts.size() + (code.size() + 1) / 2, 0.0);
        std::memcpy(blob.data(), consts.data(), consts.size() * sizeof(double));
        std::memcpy(blob.data() + consts.size(), code.data(), code.size() * sizeof(uint32_t));
        int rc;
        if ((rc = upload_blob(ps, blob))) return rc;
        P.consts = static_cast<const double*>(ps.d_blob);
        P.code = reinterpret_cast<const uint32_t*>(static_cast<const double*>(ps.d_blob) + consts.size());
        break;
    }
    case ZQD_POT_LVC: {
        std::vector<double> packed;
        packed.insert(packed.end(), o.lvc_freq.begin(), o.lvc_freq.end());
        packed.insert(packed.end(), o.lvc_exc.begin(), o.lvc_exc.end());
        packed.insert(packed.end(), o.lvc_kappa.begin(), o.lvc_kappa.end());
        packed.insert(packed.end(), o.lvc_lambda.begin(), o.lvc_lambda.end());
        int rc;
        if ((rc = upload_blob(ps, packed))) return rc;
        P.lvc = static_cast<const double*>(ps.d_blob);
        P.lvc_nm = (int)o.lvc_freq.size();
        break;
    }
    case ZQD_POT_FILE: {
        int rc;
        if ((rc = upload_blob(ps, o.file_table))) return rc;
        P.file = static_cast<const double*>(ps.d_blob);
        P.file_nrow = (int)o.file_nrow;
        P.file_ncol = (int)o.file_ncol;
        P.file_size = (int)std::llround(std::pow((double)o.file_nrow, 1.0 / (double)o.file_nd));
        break;
    }
    }
    return ZQD_OK;
}

static std::vector<double> compute_twiddles(int n) {
    // exp(-2 pi i t/n) with the angle reduced to the first octant in exact
    // integer arithmetic, evaluated in long double and rounded once.
    std::vector<double> tw(2 * (size_t)n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int t = 0; t < n; ++t) {
        // angle = 2 pi t / n; use symmetry t -> (t mod n) quadrant decomposition
        long long num = (long long)t * 8; // angle in units of pi/4: 8t/n
        int oct = (int)(num / n);         // 0..7
        long long remn = num - (long long)oct * n;
        long double c, s;
        // base angle within the octant: (oct*n + remn) * pi / (4n)
        long double a = (long double)remn * pi / (4.0L * (long double)n);
        long double ca = cosl(a), sa = sinl(a);
        // rotate by oct * pi/4
        const long double h = 0.707106781186547524400844362104849039L;
        switch (oct) {
        case 0: c = ca; s = sa; break;
        case 1: c = h * (ca - sa); s = h * (ca + sa); break;
        case 2: c = -sa; s = ca; break;
        case 3: c = -h * (ca + sa); s = h * (ca - sa); break;
        case 4: c = -ca; s = -sa; break;
        case 5: c = -h * (ca - sa); s = -h * (ca + sa); break;
        case 6: c = sa; s = -ca; break;
        default: c = h * (ca + sa); s = -h * (ca - sa); break;
        }
        if (remn == 0 && (oct & 1) == 0) { // exact axis values
            c = (oct == 0) ? 1 : (oct == 2) ? 0 : (oct == 4) ? -1 : 0;
            s = (oct == 0) ? 0 : (oct == 2) ? 1 : (oct == 4) ? 0 : -1;
        }
        tw[2 * t] = (double)c;
        tw[2 * t + 1] = (double)-s;
    }
    return tw;
}

// The long-double table costs about a millisecond at 8192 points; jobs of a batch or a
// stream mostly share their lengths, so each length is computed once per process.
std::vector<double> twiddles_f64(int n) {
    static std::mutex mu;
    static std::unordered_map<int, std::shared_ptr<const std::vector<double>>> cache;
    std::shared_ptr<const std::vector<double>> t;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(n);
        if (it != cache.end()) t = it->second;
    }
    if (!t) {
        t = std::make_shared<const std::vector<double>>(compute_twiddles(n));
        std::lock_guard<std::mutex> lk(mu);
        cache.emplace(n, t);
    }
    return *t;
}

} // namespace zqd

extern "C" const char* zqd_last_error(void) { return zqd::last_error(); }

extern "C" const char* zqd_status_string(int status) {
    switch (status) {
    case ZQD_OK: return "ok";
    case ZQD_ERR_INVALID_INPUT: return "invalid input";
    case ZQD_ERR_OUT_OF_MEMORY: return "out of host memory";
    case ZQD_ERR_DEVICE_OOM: return "out of device memory";
    case ZQD_ERR_PLAN_FAILED: return "FFT plan creation failed";
    case ZQD_ERR_EIGEN_FAILED: return "eigendecomposition failed";
    case ZQD_ERR_EXPRESSION: return "expression compilation failed";
    case ZQD_ERR_UNSUPPORTED: return "unsupported by this build";
    case ZQD_ERR_DEVICE: return "CUDA device error";
    case ZQD_ERR_TIMEOUT: return "timed out";
    case ZQD_ERR_CANCELLED: return "cancelled";
    case ZQD_ERR_NOT_FOUND: return "not found";
    case ZQD_ERR_NO_DEVICE: return "no CUDA device";
    case ZQD_ERR_NUMERIC: return "non-finite observable";
    default: return "unknown status";
    }
}

extern "C" void zqd_options_init(zqd_options* o) {
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(zqd_options);
    o->log_interval = 1;
    o->cap_exponent = 0.001;
    o->spectrum_threshold = 1e-6;
    o->fft_plan = 1; /* measure */
    o->precision = ZQD_FP64;
    o->potential.kind = ZQD_POT_HARMONIC;
}

extern "C" void zqd_potential_init(zqd_potential* p, zqd_potential_kind kind) {
    std::memset(p, 0, sizeof(*p));
    p->kind = kind;
    switch (kind) {
    case ZQD_POT_TIME_LINEAR: p->p[0] = 10; p->p[1] = 2; break;
    case ZQD_POT_TULLY_1: p->p[0] = 0.010; p->p[1] = 1.600; p->p[2] = 0.005; p->p[3] = 1.000; break;
    case ZQD_POT_TULLY_2: p->p[0] = 0.10; p->p[1] = 0.28; p->p[2] = 0.015; p->p[3] = 0.06; p->p[4] = 0.05; break;
    case ZQD_POT_TULLY_3: p->p[0] = 6.0e-4; p->p[1] = 0.10; p->p[2] = 0.90; break;
    default: break;
    }
}

namespace zqd {
// Host-side arming of the TMA-wait failure path (zqd_testing_tma_withhold_load): the next
// g_tma_withhold launches of the N-D TMA-staged passes issue no first load and wait at most
// g_tma_wait_cycles.
static std::atomic<long long> g_tma_withhold{0}, g_tma_wait_cycles{0};

long long tma_wait_budget(long long default_cycles, bool* withhold) {
    *withhold = false;
    if (g_tma_withhold.load(std::memory_order_relaxed) <= 0) return default_cycles;
    if (g_tma_withhold.fetch_sub(1) <= 0) return default_cycles;
    *withhold = true;
    return g_tma_wait_cycles.load();
}
} // namespace zqd

extern "C" void zqd_testing_fail_device_allocations(uint64_t after, uint64_t count) {
    zqd::g_alloc_fail.store((long long)count);
    zqd::g_alloc_skip.store(count ? (long long)after : -1);
}

extern "C" int zqd_testing_tma_withhold_load(uint32_t launches, double wait_us) {
    if (!(wait_us > 0)) return zqd::fail(ZQD_ERR_INVALID_INPUT, "WAIT BUDGET MUST BE POSITIVE");
    int dev = 0, khz = 0;
    ZQD_CUDA(cudaGetDevice(&dev));
    ZQD_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev));
    zqd::g_tma_wait_cycles.store((long long)(wait_us * 1e-3 * (double)khz));
    zqd::g_tma_withhold.store((long long)launches);
    return ZQD_OK;
}
