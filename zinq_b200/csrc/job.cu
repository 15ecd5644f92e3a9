// job.cu -- job lifecycle behind the C-ABI: create (init, src/quantum_dynamics.zig:713-749),
// run (run/solve, :567-603 and :860-950) and result download.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "internal.h"
#include "job.h"
#include "line_solve.cuh"

namespace zqd {

// ------------------------------------------------------------------ setup
template <typename T> struct LineTablesArgs {
    int n, m, C, q;
    double lo, hi, mass, dt_re, dt_im;
    int has_cap;
    double cap_lo, cap_hi, cap_exp;
    PotDev pot;
    Tab<T>* R;
    double* V;
    double* U;
    double* capw;
    Tab<T>* expk;
};

// Smallest gap between adiabatic surfaces over the grid at t = 0 (ZQD_PRECISION_AUTO): the
// eigenvalues of V at every point (eigh as in Hamiltonian.init, wavepacket.zig:96-143), the
// smallest |W_i - W_k| per block, then an integer atomicMin on the bits (non-negative doubles
// order like their bit patterns).
struct GapArgs {
    PotDev pot;
    int d, n;
    size_t N;
    double lo[3], span[3];
    unsigned long long* out;
};
template <int S> __global__ void min_gap_kernel(const __grid_constant__ GapArgs a) {
    double best = INFINITY;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < a.N; g += (size_t)gridDim.x * blockDim.x) {
        double r[3];
        size_t t = g;
        for (int l = 0; l < a.d; ++l) { // last axis fastest (Grid.init, wavepacket.zig:55-74)
            const int j = a.d - 1 - l;
            r[j] = __dadd_rn(a.lo[j], __dmul_rn((double)(t % (size_t)a.n), a.span[j]) / (double)a.n);
            t /= (size_t)a.n;
        }
        double V[S * S], Vu[S * S], W[S], U[S * S];
        pot_eval(a.pot, r, 0.0, V);
        for (int i = 0; i < S; ++i)
            for (int k = 0; k < S; ++k) Vu[i * S + k] = V[(i < k ? i : k) * S + (i < k ? k : i)];
        eigh_dev<S>(Vu, W, U);
        for (int i = 0; i < S; ++i)
            for (int k = i + 1; k < S; ++k) best = fmin(best, fabs(W[i] - W[k]));
    }
    for (int off = 16; off > 0; off >>= 1) best = fmin(best, __shfl_down_sync(0xffffffffu, best, off));
    __shared__ double wmin[32];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = fmin(best, wmin[w]);
        atomicMin(a.out, (unsigned long long)__double_as_longlong(best));
    }
}

// ZQD_PRECISION_AUTO -> ZQD_FP32_MIXED, or ZQD_FP64 below the gap threshold (one launch and
// one synchronisation on the job's stream; one-state potentials have no gap and take FP32)
static int resolve_auto_precision(zqd_job* J) {
    if (J->o.precision != ZQD_PRECISION_AUTO) return ZQD_OK;
    J->o.precision = ZQD_FP32_MIXED;
    if (J->S == 1) return ZQD_OK;
    GapArgs a{};
    a.pot = J->pot.dev;
    a.d = J->d;
    a.n = J->n;
    a.N = J->N;
    for (int j = 0; j < J->d; ++j) {
        a.lo[j] = J->o.bounds[2 * j];
        a.span[j] = J->o.bounds[2 * j + 1] - J->o.bounds[2 * j];
    }
    DevBuf out;
    int rc;
    if ((rc = out.alloc(sizeof(unsigned long long), J->stream))) return rc;
    a.out = out.as<unsigned long long>();
    ZQD_CUDA(cudaMemsetAsync(out.p, 0xff, sizeof(unsigned long long), J->stream)); // above every double's bits
    const unsigned blocks = (unsigned)std::min<size_t>(1024, (J->N + 255) / 256);
    switch (J->S) {
    case 2: min_gap_kernel<2><<<blocks, 256, 0, J->stream>>>(a); break;
    case 3: min_gap_kernel<3><<<blocks, 256, 0, J->stream>>>(a); break;
    default: min_gap_kernel<4><<<blocks, 256, 0, J->stream>>>(a); break;
    }
    ZQD_CUDA(cudaGetLastError());
    ZQD_CUDA(cudaStreamSynchronize(J->stream)); // the kernel, then the copy into pageable memory
    unsigned long long bits = 0;
    ZQD_CUDA(cudaMemcpyAsync(&bits, out.p, sizeof(bits), cudaMemcpyDeviceToHost, J->stream));
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    double gap;
    std::memcpy(&gap, &bits, sizeof(gap));
    J->min_gap = gap;
    if (!(gap >= ZQD_AUTO_GAP_THRESHOLD)) J->o.precision = ZQD_FP64; // NaN (no point evaluated) included
    return ZQD_OK;
}

// Hamiltonian.init/update at t = 0 (wavepacket.zig:96-143) and Propagator.init/update
// (quantum_dynamics.zig:387-468) for every grid point, written in the cluster-permuted layout.
template <typename T, int S> __global__ void line_tables_kernel(const __grid_constant__ LineTablesArgs<T> a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const int c = p / a.m, j = p - c * a.m;
    const int x = c + a.C * j;
    double r = __dadd_rn(a.lo, __dmul_rn((double)x, a.hi - a.lo) / (double)a.n);
    double V[S * S], Vu[S * S], W[S], U[S * S];
    pot_eval(a.pot, &r, 0.0, V);
    for (int i = 0; i < S; ++i)
        for (int k = 0; k < S; ++k) Vu[i * S + k] = V[(i < k ? i : k) * S + (i < k ? k : i)];
    eigh_dev<S>(Vu, W, U);
    for (int e = 0; e < S * S; ++e) a.V[(size_t)e * a.n + p] = V[e];
    if (S > 1)
        for (int e = 0; e < S * S; ++e) a.U[(size_t)e * a.n + p] = U[e];
    double cap_sum = 0;
    if (a.has_cap) {
        double dist = fmax(0.0, fmax(a.cap_lo - r, r - a.cap_hi));
        if (dist > 0) cap_sum = __dadd_rn(cap_sum, exp(__dmul_rn(a.cap_exp, dist)) - 1);
    }
    double decay = exp(__dmul_rn(__dmul_rn(-0.5, cap_sum), hypot(a.dt_re, a.dt_im)));
    if (a.capw) a.capw[p] = 1 - decay * decay;
    int idx = 0;
    for (int k = 0; k < S; ++k)
        for (int jj = k; jj < S; ++jj) {
            double re, im;
            propagator_entry<S>(W, U, a.dt_re, a.dt_im, decay, k, jj, re, im);
            a.R[(size_t)idx * a.n + p] = mktab<T>(re, im);
            ++idx;
        }
    // kinetic phase exp(-i K dt) at the wavenumber this slot holds after the forward transform
    {
        const int e = j, k2 = e / a.q, u = e - k2 * a.q;
        const int kidx = c * a.q + u + a.m * k2;
        double nn = (double)kidx;
        double kv = __dmul_rn(kidx < a.n / 2 ? nn : __dsub_rn(nn, (double)a.n), 6.283185307179586476925286766559 / (a.hi - a.lo));
        double K = __dmul_rn(__dmul_rn(0.5, kv), kv) / a.mass;
        // Complex(0, -K) * dt
        double zre = __dsub_rn(__dmul_rn(0.0, a.dt_re), __dmul_rn(-K, a.dt_im));
        double zim = __dadd_rn(__dmul_rn(0.0, a.dt_im), __dmul_rn(-K, a.dt_re));
        double ore, oim;
        cexp_dev(zre, zim, ore, oim);
        a.expk[p] = mktab<T>(ore, oim);
    }
}

// 1-D eigenvector sign continuity (wavepacket.zig:145-155): eigenvector j at
// point x is flipped when its overlap with the (already fixed) vector at x-1
// is negative.  s_x = s_{x-1} for a positive raw overlap, -s_{x-1} for a
// negative one, +1 for zero; a single CTA scans these maps in grid order.
template <int S> __global__ void sign_scan_kernel(double* U, int n, int m, int C, signed char* code) {
    __shared__ int sm_m[1024], sm_c[1024];
    const int nt = blockDim.x, t = threadIdx.x;
    const int chunk = (n + nt - 1) / nt;
    auto pos = [&](int x) { return (x % C) * m + x / C; };
    for (int jcol = 0; jcol < S; ++jcol) {
        // phase 1: per-point maps from raw overlaps, and this thread's composed map
        int M = 1, Cc = 0; // s -> M*s + Cc
        int x0 = t * chunk, x1 = min(n, x0 + chunk);
        for (int x = max(x0, 1); x < x1; ++x) {
            double ov = 0;
            for (int k = 0; k < S; ++k)
                ov = __dadd_rn(ov, __dmul_rn(U[(size_t)(k * S + jcol) * n + pos(x)], U[(size_t)(k * S + jcol) * n + pos(x - 1)]));
            int cd = ov > 0 ? 0 : (ov < 0 ? 1 : 2);
            code[x] = (signed char)cd;
            if (cd == 1) {
                M = -M;
                Cc = -Cc;
            } else if (cd == 2) {
                M = 0;
                Cc = 1;
            }
        }
        sm_m[t] = M;
        sm_c[t] = Cc;
        __syncthreads();
        if (t == 0) { // sequential exclusive scan of the per-thread maps applied to s_0 = +1
            int s = 1;
            for (int i = 0; i < nt; ++i) {
                int mi = sm_m[i], ci = sm_c[i];
                sm_m[i] = s; // sign entering chunk i
                s = mi * s + ci;
            }
        }
        __syncthreads();
        int s = sm_m[t];
        // phase 2: walk the chunk and flip
        for (int x = x0; x < x1; ++x) {
            if (x > 0) {
                int cd = code[x];
                s = cd == 0 ? s : (cd == 1 ? -s : 1);
            }
            if (s < 0)
                for (int k = 0; k < S; ++k) {
                    double* u = &U[(size_t)(k * S + jcol) * n + pos(x)];
                    *u = -*u;
                }
        }
        __syncthreads();
    }
}

} // namespace zqd


using namespace zqd;


namespace zqd {

template <typename T> static size_t cxsize() { return sizeof(cx<T>); }

// Cluster shape of a 1-D job: C CTAs of m = n/C points each, radix-4 local passes (radix 8
// where m/4 threads exceed the kernel's limit) and S m/4 threads per CTA, capped at the
// limit: a pass whose hooks mix the states runs one butterfly of every state per thread on
// the first m/4 threads, the other passes one (butterfly, state) pair per thread.  The default is the smallest C whose CTA fits in shared memory
// and holds at most `target` points (256; measured per step: 8192 points on 16 CTAs 18 %
// faster than on 8, 1024 points on 4 CTAs 15 % faster than on 2); ZQD_LINE_CLUSTER forces C
// (tuning sweeps).  Radix-8 kernels exist for 16-CTA clusters only (lines above 16384 points in
// FP64, 32768 in FP32); radix-4-only kernels keep the instruction footprint small.
static int choose_line_shape(zqd_job* J) {
    const size_t budget = 205 * 1024; // dynamic shared memory per CTA
    int forced = 0, forced_lr = 0;
    ShapeOverride ov;
    if (lookup_shape(1, J->n, J->S, J->fp32, ov)) { // autotuned (or being measured by the autotuner)
        forced = ov.C;
        forced_lr = ov.lrmax;
    }
    if (const char* env = std::getenv("ZQD_LINE_CLUSTER")) forced = std::atoi(env), forced_lr = 0;
    const int target = 256;
    // pass 0: the smallest C with at most `target` points per CTA; 1: the largest C that fits
    // (fewest points per CTA); 2: the same with R read from global memory
    for (int pass = 0; pass < 3; ++pass) {
        const bool rg = pass == 2;
        for (int k = 0; k < 5; ++k) {
            const int C = pass == 0 ? 1 << k : 16 >> k;
            if (forced && C != forced) continue;
            if (J->n % C) continue;
            const int m = J->n / C;
            if (m < 8 || m / C < 1) continue;
            // radix 4 doubles the threads of a CTA (more warps to hide latency) where the limit allows
            int lrmax = 2;
            const int tmax = J->fp32 ? LineMaxThreads<float>::value : LineMaxThreads<double>::value;
            if (((m >> 2) + 31) / 32 * 32 > tmax) lrmax = 3;
            if (forced_lr == 3) lrmax = 3;
            else if (forced_lr == 2 && lrmax != 2) continue;
            if (lrmax == 3 && C != 16) continue; // radix 8 is built for 16-CTA clusters only
            if (std::max(32, ((m >> lrmax) + 31) / 32 * 32) > tmax) continue;
            const size_t smem = J->fp32 ? line_smem_bytes<float>(J->S, C, m, rg, lrmax)
                                        : line_smem_bytes<double>(J->S, C, m, rg, lrmax);
            if (smem > budget) continue;
            // the eigenvectors staged beside the tables where they fit (several states)
            const size_t smem_u = J->fp32 ? line_smem_bytes<float>(J->S, C, m, rg, lrmax, true)
                                          : line_smem_bytes<double>(J->S, C, m, rg, lrmax, true);
            const bool u_smem = J->S > 1 && smem_u <= budget;
            // one thread per butterfly of every state (passes without state-mixing hooks split
            // the states over the threads), within the kernel's thread limit
            const int threads = std::min(tmax, std::max(32, ((m >> lrmax) * J->S + 31) / 32 * 32));
            if (pass == 0 && !forced && m > target) continue;
            J->C = C;
            J->m = m;
            J->q = m / C;
            J->E = 8 * J->S;
            J->threads = threads;
            J->smem = u_smem ? smem_u : smem;
            J->r_global = rg;
            J->lrmax = lrmax;
            J->u_smem = u_smem;
            return ZQD_OK;
        }
    }
    return fail(ZQD_ERR_UNSUPPORTED, "1-D GRID DOES NOT FIT THE RESIDENT CLUSTER KERNEL (at most 16 CTAs of 4096 points)");
}

using LineKernelFn = void (*)(const void*);

// launchers compiled in line_inst.cu, one translation unit per (precision, states)
int launch_line_d1(const LaunchShape*, const void*, int);
int launch_line_d2(const LaunchShape*, const void*, int);
int launch_line_d3(const LaunchShape*, const void*, int);
int launch_line_d4(const LaunchShape*, const void*, int);
int launch_line_f1(const LaunchShape*, const void*, int);
int launch_line_f2(const LaunchShape*, const void*, int);
int launch_line_f3(const LaunchShape*, const void*, int);
int launch_line_f4(const LaunchShape*, const void*, int);

template <typename T> static int launch_line_s(const LaunchShape* J, const void* dj, int nj) {
    static int (*const dtab[4])(const LaunchShape*, const void*, int) = {launch_line_d1, launch_line_d2, launch_line_d3,
                                                                          launch_line_d4};
    static int (*const ftab[4])(const LaunchShape*, const void*, int) = {launch_line_f1, launch_line_f2, launch_line_f3,
                                                                          launch_line_f4};
    if (J->S < 1 || J->S > 4) return fail(ZQD_ERR_UNSUPPORTED, "STATE COUNT MUST BE 1..4");
    return std::is_same<T, double>::value ? dtab[J->S - 1](J, dj, nj) : ftab[J->S - 1](J, dj, nj);
}

template <typename T, int S> static int run_tables(zqd_job* J) {
    LineTablesArgs<T> a{};
    a.n = J->n;
    a.m = J->m;
    a.C = J->C;
    a.q = J->q;
    a.lo = J->o.bounds[0];
    a.hi = J->o.bounds[1];
    a.mass = J->o.mass[0];
    a.dt_re = J->o.imag_nstate ? 0.0 : J->o.time_step;
    a.dt_im = J->o.imag_nstate ? -J->o.time_step : 0.0;
    a.has_cap = J->o.has_cap;
    if (J->o.has_cap) {
        a.cap_lo = J->o.cap_bounds[0];
        a.cap_hi = J->o.cap_bounds[1];
        a.cap_exp = J->o.cap_exponent;
    }
    a.pot = J->pot.dev;
    a.R = J->R.as<Tab<T>>();
    a.V = J->V.as<double>();
    a.U = J->U.as<double>();
    a.capw = J->capw.as<double>();
    a.expk = J->expk.as<Tab<T>>();
    int threads = 128, blocks = (J->n + threads - 1) / threads;
    line_tables_kernel<T, S><<<blocks, threads, 0, J->stream>>>(a);
    ZQD_CUDA(cudaGetLastError());
    if (S > 1) {
        sign_scan_kernel<S><<<1, 1024, 0, J->stream>>>(J->U.as<double>(), J->n, J->m, J->C, J->scratch.as<signed char>());
        ZQD_CUDA(cudaGetLastError());
    }
    return ZQD_OK;
}

template <typename T> static int run_tables_s(zqd_job* J) {
    switch (J->S) {
    case 1: return run_tables<T, 1>(J);
    case 2: return run_tables<T, 2>(J);
    case 3: return run_tables<T, 3>(J);
    default: return run_tables<T, 4>(J);
    }
}

template <typename T> static int create_line(zqd_job* J) {
    const size_t n = J->n, S = J->S, nsym = S * (S + 1) / 2;
    const size_t c = sizeof(cx<T>);
    int rc;
    const size_t tb = sizeof(Tab<T>);
    // every buffer of the job in one pool block: one allocation (and one synchronisation)
    // instead of one per buffer
    const bool acf = J->o.has_spectrum || (J->o.write_mask & ZQD_WRITE_ACF);
    const size_t rows = (size_t)J->o.iterations + 1;
    const struct {
        DevBuf* b;
        size_t bytes;
    } parts[] = {
        {&J->R, nsym * n * tb},
        {&J->expk, n * tb},
        {&J->V, S * S * n * sizeof(double)},
        {&J->U, S > 1 ? S * S * n * sizeof(double) : 0},
        {&J->capw, J->o.has_cap ? n * sizeof(double) : 0},
        {&J->tw, n * tb},
        {&J->psi_save, S * n * c},
        {&J->psi0, acf ? S * n * c : 0},
        {&J->orth, J->o.imag_nstate > 1 ? (size_t)(J->o.imag_nstate - 1) * S * n * c : 0},
        {&J->hist, (size_t)J->nsolve * rows * J->hc * sizeof(double)},
        {&J->fin, (size_t)J->nsolve * J->hc * sizeof(double)},
        {&J->rows, (size_t)J->nsolve * sizeof(int)},
        {&J->jobs, (size_t)J->nsolve * sizeof(LineJob<T>)},
        {&J->scratch, n + 16},
        {&J->wfn_hist, (J->o.write_mask & ZQD_WRITE_WAVEFUNCTION) ? (size_t)J->nsolve * rows * S * n * c : 0},
        {&J->psi_init, J->o.ic_wfn.empty() ? 0 : S * n * c},
        {&J->sgn, needs_sign_tracking(J->o, J->S, J->nsolve) ? S * n * sizeof(double) : 0},
        {&J->carry, (size_t)J->nsolve * S * sizeof(double)},
        {&J->done, (size_t)J->nsolve * sizeof(int)},
    };
    auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t total = 0;
    for (const auto& pt : parts) total += align(pt.bytes);
    if ((rc = J->arena.alloc(total, J->stream))) return rc;
    size_t off = 0;
    for (const auto& pt : parts) {
        pt.b->view(J->arena.as<char>() + off, pt.bytes);
        off += align(pt.bytes);
    }
    if (!J->o.ic_wfn.empty()) { // initial wavefunction in the cluster-permuted layout
        std::vector<cx<T>> h(S * n);
        for (size_t st = 0; st < S; ++st)
            for (size_t p = 0; p < n; ++p) {
                const size_t cc = p / J->m, j = p - cc * J->m, x = cc + J->C * j;
                h[st * n + p] = mk<T>((T)J->o.ic_wfn[2 * (st * n + x)], (T)J->o.ic_wfn[2 * (st * n + x) + 1]);
            }
        ZQD_CUDA(cudaMemcpyAsync(J->psi_init.p, h.data(), S * n * c, cudaMemcpyHostToDevice, J->stream));
        ZQD_CUDA(cudaStreamSynchronize(J->stream));
        J->h2d += S * n * c;
    }
    J->device_bytes = J->R.bytes + J->expk.bytes + J->V.bytes + J->U.bytes + J->capw.bytes + J->tw.bytes +
                      J->psi_save.bytes + J->psi0.bytes + J->orth.bytes + J->hist.bytes;
    // twiddles
    std::vector<double> tw = twiddles_f64(J->n);
    std::vector<Tab<T>> twt(n);
    for (size_t t = 0; t < n; ++t) twt[t] = mktab<T>(tw[2 * t], tw[2 * t + 1]);
    // (a copy from pageable memory has read the host buffer when the call returns)
    ZQD_CUDA(cudaMemcpyAsync(J->tw.p, twt.data(), n * tb, cudaMemcpyHostToDevice, J->stream));
    J->h2d += n * tb + J->pot.bytes;
    if ((rc = run_tables_s<T>(J))) return rc;
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    return ZQD_OK;
}

template <typename T> static LineJob<T> line_job_desc(const zqd_job* J, int s) {
    LineJob<T> L{};
    const Opts& o = J->o;
    L.n = J->n;
    L.m = J->m;
    L.logm = 0;
    while ((1 << L.logm) < J->m) ++L.logm;
    L.q = J->q;
    L.lo = o.bounds[0];
    L.hi = o.bounds[1];
    L.dr = (o.bounds[1] - o.bounds[0]) / (double)o.npoint;
    L.dk = L.dr / (double)J->N;
    L.mass = o.mass[0];
    L.iters = (int)o.iterations;
    L.dt_re = o.imag_nstate ? 0.0 : o.time_step;
    L.dt_im = o.imag_nstate ? -o.time_step : 0.0;
    L.tstep = o.time_step;
    L.itp = o.imag_nstate > 0;
    L.ic_state = (int)o.ic_state;
    L.ic_adia = o.ic_adiabatic;
    L.x0 = o.pos[0];
    L.p0 = o.mom[0];
    L.gamma = o.gamma[0];
    L.wmask = o.write_mask;
    L.log = o.log;
    L.log_interval = (int)o.log_interval;
    L.adiabatic = o.adiabatic;
    L.calc_acf = o.has_spectrum || (o.write_mask & ZQD_WRITE_ACF);
    L.track = o.has_cap && o.cap_track;
    L.has_stop = o.has_cap && o.cap_has_stop;
    L.stop_norm = o.cap_stop_norm;
    L.td = o.pot_td;
    L.has_cap = o.has_cap;
    if (o.has_cap) {
        L.cap_lo = o.cap_bounds[0];
        L.cap_hi = o.cap_bounds[1];
        L.cap_exp = o.cap_exponent;
    }
    L.R = J->R.as<Tab<T>>();
    L.psi_init = J->psi_init.as<cx<T>>();
    L.r_global = J->r_global ? 1 : 0;
    L.lrmax = J->lrmax;
    L.u_smem = J->u_smem ? 1 : 0;
    L.sign_track = needs_sign_tracking(o, J->S, J->nsolve) ? 1 : 0;
    L.sgn = J->sgn.as<double>();
    L.wfn_hist = J->wfn_hist.p ? J->wfn_hist.as<cx<T>>() + (size_t)s * ((size_t)o.iterations + 1) * J->S * J->n : nullptr;
    L.expk = J->expk.as<Tab<T>>();
    L.V = J->V.as<double>();
    L.U = J->U.as<double>();
    L.capw = J->capw.as<double>();
    L.tw = J->tw.as<Tab<T>>();
    L.psi_save = J->psi_save.as<cx<T>>();
    L.psi0 = J->psi0.as<cx<T>>();
    L.orth = J->orth.as<cx<T>>();
    L.northo = s;
    size_t rows = (size_t)o.iterations + 1;
    L.hist = J->hist.as<double>() + (size_t)s * rows * J->hc;
    L.fin = J->fin.as<double>() + (size_t)s * J->hc;
    L.rows = J->rows.as<int>() + s;
    L.i0 = 0;
    L.i1 = L.iters;
    L.carry = J->carry.as<double>() + (size_t)s * J->S;
    L.done = J->done.as<int>() + s;
    L.pot = J->pot.dev;
    return L;
}

// A time-dependent potential leaves the tables at the last update's time: a later run of the same
// job starts again from the t = 0 tables (Hamiltonian.init, Propagator.init).
template <typename T> static int refresh_line_tables(zqd_job* J) {
    if (!J->o.pot_td || J->runs++ == 0) return ZQD_OK;
    return run_tables_s<T>(J);
}

// the start of a run (whole or step-wise): progress and observable cursors back to zero
static void reset_progress(zqd_job* J) {
    J->step_solve = 0;
    J->solve_rows.assign(J->nsolve, 0);
    J->solve_ended.assign(J->nsolve, 0);
    J->obs_solve = J->obs_row = 0;
    J->stepping = false;
}

// after a whole run: every solve ended, with the row counts the device recorded
static int mark_all_ended(zqd_job* J) {
    std::vector<int> rows(J->nsolve);
    ZQD_CUDA(cudaMemcpyAsync(rows.data(), J->rows.p, rows.size() * sizeof(int), cudaMemcpyDeviceToHost, J->stream));
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    J->solve_rows = rows;
    J->solve_ended.assign(J->nsolve, 1);
    J->step_solve = J->nsolve;
    return ZQD_OK;
}

template <typename T> static int run_line(zqd_job* J) {
    const size_t SN = (size_t)J->S * J->n * sizeof(cx<T>);
    reset_progress(J);
    if (int rc = refresh_line_tables<T>(J)) return rc;
    std::vector<LineJob<T>> descs;
    for (int s = 0; s < J->nsolve; ++s) descs.push_back(line_job_desc<T>(J, s));
    ZQD_CUDA(cudaMemcpyAsync(J->jobs.p, descs.data(), descs.size() * sizeof(LineJob<T>), cudaMemcpyHostToDevice, J->stream));
    J->h2d += descs.size() * sizeof(LineJob<T>);
    ZQD_CUDA(cudaEventRecord(J->ev0, J->stream));
    LaunchShape sh{J->S, J->C, J->E, J->threads, J->smem, J->stream};
    sh.lrmax = J->lrmax;
    for (int s = 0; s < J->nsolve; ++s) {
        int rc = launch_line_s<T>(&sh, J->jobs.as<LineJob<T>>() + s, 1);
        if (rc) return rc;
        if (s + 1 < J->nsolve) // orthw.append (quantum_dynamics.zig:586-591)
            ZQD_CUDA(cudaMemcpyAsync(J->orth.as<char>() + (size_t)s * SN, J->psi_save.p, SN, cudaMemcpyDeviceToDevice, J->stream));
    }
    ZQD_CUDA(cudaEventRecord(J->ev1, J->stream));
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    ZQD_CUDA(cudaEventElapsedTime(&J->last_ms, J->ev0, J->ev1));
    return mark_all_ended(J);
}

// One launch of rows i0..i1 of solve s of a 1-D job (zqd_job_step); *rows and *ended come back
// from the device.
template <typename T> static int step_line(zqd_job* J, int s, int i0, int i1, int* rows, int* ended) {
    LineJob<T> d = line_job_desc<T>(J, s);
    d.i0 = i0;
    d.i1 = i1;
    ZQD_CUDA(cudaMemcpyAsync(J->jobs.as<LineJob<T>>() + s, &d, sizeof(d), cudaMemcpyHostToDevice, J->stream));
    J->h2d += sizeof(d);
    LaunchShape sh{J->S, J->C, J->E, J->threads, J->smem, J->stream};
    sh.lrmax = J->lrmax;
    ZQD_CUDA(cudaEventRecord(J->ev0, J->stream));
    if (int rc = launch_line_s<T>(&sh, J->jobs.as<LineJob<T>>() + s, 1)) return rc;
    ZQD_CUDA(cudaEventRecord(J->ev1, J->stream));
    // wait first: a copy into pageable memory queued behind the launch would wait inside the driver,
    // where it can hold up other threads' copies
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    int flags[2] = {0, 0};
    ZQD_CUDA(cudaMemcpyAsync(&flags[0], J->rows.as<int>() + s, sizeof(int), cudaMemcpyDeviceToHost, J->stream));
    ZQD_CUDA(cudaMemcpyAsync(&flags[1], J->done.as<int>() + s, sizeof(int), cudaMemcpyDeviceToHost, J->stream));
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    float ms = 0;
    ZQD_CUDA(cudaEventElapsedTime(&ms, J->ev0, J->ev1));
    J->last_ms += ms;
    J->d2h += sizeof(flags);
    *rows = flags[0];
    *ended = flags[1];
    return ZQD_OK;
}

// Per-thread pinned staging buffer for result copies (device-to-host copies into pageable
// memory go through the driver's bounce buffer at a fraction of the bandwidth).  Fixed size,
// allocated at a thread's first result and never reallocated: freeing pinned memory
// synchronises the whole device, which would stall other jobs' kernels.  Null for larger
// results (and when pinned memory cannot be had): the caller then copies directly.
static char* pinned_staging(size_t bytes) {
    constexpr size_t kBytes = (size_t)8 << 20;
    struct Buf {
        char* p = nullptr;
        bool tried = false;
        ~Buf() {
            if (p) cudaFreeHost(p);
        }
    };
    thread_local Buf b;
    if (bytes > kBytes) return nullptr;
    if (!b.tried) {
        b.tried = true;
        if (cudaHostAlloc((void**)&b.p, kBytes, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
        }
    }
    return b.p;
}

template <typename T> static int fetch_line(zqd_job* J, zqd_result* R) {
    size_t rows = (size_t)J->o.iterations + 1;
    std::vector<double> hist((size_t)J->nsolve * rows * J->hc), fin((size_t)J->nsolve * J->hc);
    std::vector<int> nrows(J->nsolve);
    const size_t SN = (size_t)J->S * J->N;
    // the final wavefunctions are skipped for callers that do not read them (the server's option)
    const size_t SNw = J->fetch_psi ? SN : 0;
    std::vector<cx<T>> save(SNw), orth((size_t)(J->nsolve - 1) * SNw);
    const struct {
        void* host;
        const void* dev;
        size_t bytes;
    } parts[] = {{hist.data(), J->hist.p, hist.size() * sizeof(double)},
                 {fin.data(), J->fin.p, fin.size() * sizeof(double)},
                 {nrows.data(), J->rows.p, nrows.size() * sizeof(int)},
                 {save.data(), J->psi_save.p, SNw * sizeof(cx<T>)},
                 {orth.data(), J->orth.p, orth.size() * sizeof(cx<T>)}};
    size_t total = 0;
    for (const auto& pt : parts) total += (pt.bytes + 15) & ~(size_t)15;
    char* stage = pinned_staging(total);
    size_t off = 0;
    for (const auto& pt : parts) {
        if (!pt.bytes) continue;
        ZQD_CUDA(cudaMemcpyAsync(stage ? stage + off : pt.host, pt.dev, pt.bytes, cudaMemcpyDeviceToHost, J->stream));
        off += (pt.bytes + 15) & ~(size_t)15;
    }
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    if (stage) {
        off = 0;
        for (const auto& pt : parts) {
            if (!pt.bytes) continue;
            std::memcpy(pt.host, stage + off, pt.bytes);
            off += (pt.bytes + 15) & ~(size_t)15;
        }
    }
    J->d2h += (hist.size() + fin.size()) * sizeof(double) + nrows.size() * sizeof(int) +
              (save.size() + orth.size()) * sizeof(cx<T>);
    R->h2d = J->h2d;
    R->d2h = J->d2h;
    R->ndim = (uint32_t)J->d;
    R->nstate = J->S;
    R->npoint_total = J->N;
    R->hc = J->hc;
    R->write_mask = J->o.write_mask;
    R->time_step = J->o.time_step;
    R->grid = J->o.bounds;
    R->grid.push_back((double)J->o.npoint);
    R->device_ms = J->last_ms;
    R->precision = J->fp32 ? ZQD_FP32_MIXED : ZQD_FP64;
    R->solves.resize(J->nsolve);
    for (int s = 0; s < J->nsolve; ++s) {
        SolveOut& so = R->solves[s];
        so.rows = (size_t)nrows[s];
        so.hist.assign(hist.begin() + (size_t)s * rows * J->hc, hist.begin() + ((size_t)s * rows + so.rows) * J->hc);
        so.fin.assign(fin.begin() + (size_t)s * J->hc, fin.begin() + (size_t)(s + 1) * J->hc);
        if (J->o.has_spectrum) { // exportWrite's calcSpectrum (quantum_dynamics.zig:257-276), on the device
            const int rc = spectrum_device(J->stream, J->hist.as<double>() + (size_t)s * rows * J->hc, J->hc,
                                           RowLayout{J->d, J->S}.acf(), so.rows, J->o, so, J->d2h);
            if (rc) return rc;
            R->d2h = J->d2h;
        }
        if (J->wfn_hist.p && so.rows) { // History.wfn of this solve
            std::vector<cx<T>> w(so.rows * SN);
            ZQD_CUDA(cudaMemcpyAsync(w.data(), J->wfn_hist.as<cx<T>>() + (size_t)s * rows * SN, w.size() * sizeof(cx<T>),
                                     cudaMemcpyDeviceToHost, J->stream));
            ZQD_CUDA(cudaStreamSynchronize(J->stream));
            J->d2h += w.size() * sizeof(cx<T>);
            R->d2h = J->d2h;
            so.wfn.resize(2 * w.size());
            for (size_t st = 0; st < so.rows * J->S; ++st)
                for (size_t p = 0; p < J->N; ++p) {
                    size_t x = p;
                    if (J->d == 1) { // position p = c*m + j holds grid index c + C*j
                        const size_t c = p / J->m, j = p - c * J->m;
                        x = c + (size_t)J->C * j;
                    }
                    so.wfn[2 * (st * J->N + x)] = (double)w[st * J->N + p].x;
                    so.wfn[2 * (st * J->N + x) + 1] = (double)w[st * J->N + p].y;
                }
        }
        if (!J->fetch_psi) continue;
        const cx<T>* src = (s + 1 < J->nsolve) ? orth.data() + (size_t)s * SN : save.data();
        so.psi.resize(2 * SN);
        if (J->d == 1) {
            for (int st = 0; st < J->S; ++st)
                for (int p = 0; p < J->n; ++p) { // un-permute: position p = c*m + j holds grid index c + C*j
                    int c = p / J->m, j = p - c * J->m, x = c + J->C * j;
                    cx<T> z = src[(size_t)st * J->n + p];
                    so.psi[2 * ((size_t)st * J->n + x)] = (double)z.x;
                    so.psi[2 * ((size_t)st * J->n + x) + 1] = (double)z.y;
                }
        } else {
            for (size_t e = 0; e < SN; ++e) {
                so.psi[2 * e] = (double)src[e].x;
                so.psi[2 * e + 1] = (double)src[e].y;
            }
        }
    }
    return ZQD_OK;
}

// N-D drivers compiled in nd_inst.cu, one translation unit per (precision, states)
#define ZQD_ND_DECL(t, s)                                                                                           \
    int nd_create_##t##s(zqd_job*);                                                                                 \
    int nd_run_##t##s(zqd_job*);                                                                                    \
    int nd_step_##t##s(zqd_job*, int, int, int, int*, int*);
ZQD_ND_DECL(d, 1) ZQD_ND_DECL(d, 2) ZQD_ND_DECL(d, 3) ZQD_ND_DECL(d, 4)
ZQD_ND_DECL(f, 1) ZQD_ND_DECL(f, 2) ZQD_ND_DECL(f, 3) ZQD_ND_DECL(f, 4)
#undef ZQD_ND_DECL

static int nd_create(zqd_job* J) {
    static int (*const dt[4])(zqd_job*) = {nd_create_d1, nd_create_d2, nd_create_d3, nd_create_d4};
    static int (*const ft[4])(zqd_job*) = {nd_create_f1, nd_create_f2, nd_create_f3, nd_create_f4};
    return J->fp32 ? ft[J->S - 1](J) : dt[J->S - 1](J);
}
static int nd_run(zqd_job* J) {
    static int (*const dt[4])(zqd_job*) = {nd_run_d1, nd_run_d2, nd_run_d3, nd_run_d4};
    static int (*const ft[4])(zqd_job*) = {nd_run_f1, nd_run_f2, nd_run_f3, nd_run_f4};
    reset_progress(J);
    const int rc = J->fp32 ? ft[J->S - 1](J) : dt[J->S - 1](J);
    return rc ? rc : mark_all_ended(J);
}
static int nd_step(zqd_job* J, int s, int i0, int i1, int* rows, int* ended) {
    using Fn = int (*)(zqd_job*, int, int, int, int*, int*);
    static const Fn dt[4] = {nd_step_d1, nd_step_d2, nd_step_d3, nd_step_d4};
    static const Fn ft[4] = {nd_step_f1, nd_step_f2, nd_step_f3, nd_step_f4};
    return (J->fp32 ? ft : dt)[J->S - 1](J, s, i0, i1, rows, ended);
}

// Advances a job by up to nsteps propagation steps (zqd_job_step).  The first call of a run also
// records row 0 (the initial state); a call never crosses into the next imaginary-time solve.
static int job_step(zqd_job* J, uint32_t nsteps) {
    if (!J->stepping) {
        reset_progress(J);
        J->stepping = true;
        if (J->d == 1) {
            const int rc = J->fp32 ? refresh_line_tables<float>(J) : refresh_line_tables<double>(J);
            if (rc) return rc;
        }
        J->last_ms = 0;
    }
    const int s = J->step_solve;
    if (s >= J->nsolve || nsteps == 0) return ZQD_OK;
    const int iters = (int)J->o.iterations, i0 = J->solve_rows[s];
    const long long want = i0 == 0 ? (long long)nsteps : (long long)i0 + nsteps - 1;
    const int i1 = (int)std::min<long long>(iters, want);
    int rows = 0, ended = 0, rc;
    if (J->d > 1) rc = nd_step(J, s, i0, i1, &rows, &ended);
    else rc = J->fp32 ? step_line<float>(J, s, i0, i1, &rows, &ended) : step_line<double>(J, s, i0, i1, &rows, &ended);
    if (rc) return rc;
    J->solve_rows[s] = rows;
    if (ended) {
        J->solve_ended[s] = 1;
        if (J->d == 1 && s + 1 < J->nsolve) { // orthw.append (quantum_dynamics.zig:586-591)
            const size_t SN = (size_t)J->S * J->n * (J->fp32 ? sizeof(cx<float>) : sizeof(cx<double>));
            ZQD_CUDA(cudaMemcpyAsync(J->orth.as<char>() + (size_t)s * SN, J->psi_save.p, SN, cudaMemcpyDeviceToDevice,
                                     J->stream));
            ZQD_CUDA(cudaStreamSynchronize(J->stream));
        }
        ++J->step_solve;
    }
    return ZQD_OK;
}

} // namespace zqd

// ------------------------------------------------------------------ C-ABI
extern "C" int zqd_job_create(const zqd_options* opt, zqd_job** out) {
    if (!out) return fail(ZQD_ERR_INVALID_INPUT, "NULL OUTPUT HANDLE");
    *out = nullptr;
    Opts o;
    int rc = copy_options(opt, o);
    if (rc) return rc;
    if ((rc = validate(o))) return rc;
    return zqd::job_create_opts(std::move(o), out);
}

// A job from already copied and validated options (zqd_job_create, the server).
int zqd::job_create_opts(Opts&& o, zqd_job** out, cudaStream_t stream) {
    *out = nullptr;
    std::unique_ptr<zqd_job> J(new (std::nothrow) zqd_job());
    if (!J) return fail(ZQD_ERR_OUT_OF_MEMORY, "host allocation failed");
    J->o = std::move(o);
    int rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(ZQD_ERR_NO_DEVICE, "no CUDA device");
    J->S = J->o.pot_ns;
    J->d = (int)J->o.ndim;
    J->n = (int)J->o.npoint;
    J->N = 1;
    for (int i = 0; i < J->d; ++i) J->N *= (size_t)J->n;
    J->nsolve = J->o.imag_nstate ? (int)J->o.imag_nstate : 1;
    J->hc = RowLayout{J->d, J->S}.width();
    if (J->d > 1 && J->n < 8) return fail(ZQD_ERR_UNSUPPORTED, "MULTI-DIMENSIONAL GRIDS NEED AT LEAST 8 POINTS PER AXIS");
    if (stream) {
        J->stream = stream;
        J->own_stream = false;
    } else {
        ZQD_CUDA(cudaStreamCreateWithFlags(&J->stream, cudaStreamNonBlocking));
    }
    ZQD_CUDA(cudaEventCreate(&J->ev0));
    ZQD_CUDA(cudaEventCreate(&J->ev1));
    if ((rc = build_potential(J->o, J->pot, J->stream))) return rc;
    if ((rc = resolve_auto_precision(J.get()))) return rc;
    J->fp32 = J->o.precision == ZQD_FP32_MIXED;
    if (J->d == 1 && (rc = choose_line_shape(J.get()))) return rc;
    if (J->d == 1) rc = J->fp32 ? create_line<float>(J.get()) : create_line<double>(J.get());
    else rc = nd_create(J.get());
    if (rc) return rc;
    *out = J.release();
    return ZQD_OK;
}

extern "C" int zqd_job_run(zqd_job* J) {
    if (!J) return fail(ZQD_ERR_INVALID_INPUT, "NULL JOB");
    if (J->d > 1) return nd_run(J);
    return J->fp32 ? run_line<float>(J) : run_line<double>(J);
}

extern "C" int zqd_job_step(zqd_job* J, uint32_t nsteps) {
    if (!J) return fail(ZQD_ERR_INVALID_INPUT, "NULL JOB");
    return job_step(J, nsteps);
}

extern "C" int zqd_job_progress(const zqd_job* J, uint32_t* solve, uint32_t* rows, int* finished) {
    if (!J) return fail(ZQD_ERR_INVALID_INPUT, "NULL JOB");
    const int s = std::min(J->step_solve, J->nsolve - 1);
    if (solve) *solve = (uint32_t)s;
    if (rows) *rows = J->solve_rows.empty() ? 0u : (uint32_t)J->solve_rows[s];
    if (finished) *finished = J->step_solve >= J->nsolve ? 1 : 0;
    return ZQD_OK;
}

extern "C" int zqd_job_observables(zqd_job* J, zqd_obs_rows* out) {
    if (!J || !out) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    *out = zqd_obs_rows{};
    out->width = (uint32_t)J->hc;
    if (J->solve_rows.empty()) return ZQD_OK; // nothing ran yet
    // the first solve with rows not yet returned
    while (J->obs_solve < J->nsolve && J->obs_row >= J->solve_rows[J->obs_solve] && J->solve_ended[J->obs_solve] &&
           J->obs_solve + 1 < J->nsolve) {
        ++J->obs_solve;
        J->obs_row = 0;
    }
    const int s = J->obs_solve, r0 = J->obs_row, r1 = J->solve_rows[s];
    out->solve = (uint32_t)s;
    out->first_row = (uint32_t)r0;
    if (r1 <= r0) {
        out->solve_finished = J->solve_ended[s];
        return ZQD_OK;
    }
    const size_t rows_per_solve = (size_t)J->o.iterations + 1;
    J->obs_buf.resize((size_t)(r1 - r0) * J->hc);
    ZQD_CUDA(cudaMemcpyAsync(J->obs_buf.data(), J->hist.as<double>() + ((size_t)s * rows_per_solve + r0) * J->hc,
                             J->obs_buf.size() * sizeof(double), cudaMemcpyDeviceToHost, J->stream));
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    J->d2h += J->obs_buf.size() * sizeof(double);
    J->obs_row = r1;
    out->nrows = (uint32_t)(r1 - r0);
    out->rows = J->obs_buf.data();
    out->solve_finished = J->solve_ended[s] && r1 == J->solve_rows[s];
    return ZQD_OK;
}

extern "C" int zqd_job_result(zqd_job* J, zqd_result** out) {
    if (!J || !out) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (J->step_solve < J->nsolve) return fail(ZQD_ERR_INVALID_INPUT, "JOB HAS NOT FINISHED (zqd_job_run or zqd_job_step until finished)");
    std::unique_ptr<zqd_result> R(new (std::nothrow) zqd_result());
    if (!R) return fail(ZQD_ERR_OUT_OF_MEMORY, "host allocation failed");
    int rc = J->fp32 ? fetch_line<float>(J, R.get()) : fetch_line<double>(J, R.get());
    if (rc) return rc;
    *out = R.release();
    return ZQD_OK;
}

extern "C" int zqd_job_info(const zqd_job* J, uint32_t* ndim, uint32_t* nstate, uint64_t* npoint_total,
                            uint32_t* cluster_ctas, size_t* device_bytes) {
    if (!J) return fail(ZQD_ERR_INVALID_INPUT, "NULL JOB");
    if (ndim) *ndim = (uint32_t)J->d;
    if (nstate) *nstate = (uint32_t)J->S;
    if (npoint_total) *npoint_total = J->N;
    if (cluster_ctas) *cluster_ctas = (uint32_t)J->C;
    if (device_bytes) *device_bytes = J->device_bytes;
    return ZQD_OK;
}

extern "C" int zqd_job_nd_shape(const zqd_job* J, zqd_nd_shape* out) {
    if (!J || !out) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (J->d < 2) return fail(ZQD_ERR_UNSUPPORTED, "NOT A 2-D OR 3-D JOB");
    *out = zqd_nd_shape{};
    if (J->nd_row_tma) {
        out->tma_row_block = 1u << J->nd_row_tma_logL;
        out->tma_row_ctas = (uint32_t)J->nd_row_tma_ctas;
        out->tma_row_threads = (uint32_t)((size_t)J->S * J->n * out->tma_row_block / 8);
    }
    if (J->nd_tma) {
        out->tma_tile_lines = 1u << J->nd_tma_logW;
        out->tma_tile_ctas = (uint32_t)J->nd_tma_ctas;
        out->tma_tile_threads = (uint32_t)((size_t)J->n * out->tma_tile_lines / 8);
    }
    out->rows_per_cta = (uint32_t)J->nd_rows;
    out->tile_lines = (uint32_t)J->nd_tile;
    return ZQD_OK;
}

extern "C" double zqd_job_device_ms(const zqd_job* J) { return J ? (double)J->last_ms : 0.0; }

extern "C" void zqd_job_destroy(zqd_job* J) { delete J; }

extern "C" int zqd_run(const zqd_options* opt, zqd_result** out) {
    if (!out) return fail(ZQD_ERR_INVALID_INPUT, "NULL OUTPUT HANDLE");
    *out = nullptr;
    zqd_job* J = nullptr;
    int rc = zqd_job_create(opt, &J);
    if (rc) return rc;
    rc = zqd_job_run(J);
    if (!rc) rc = zqd_job_result(J, out);
    zqd_job_destroy(J);
    return rc;
}

struct zqd_batch {
    std::vector<std::unique_ptr<zqd_job, void (*)(zqd_job*)>> jobs;
    struct Group {
        std::vector<zqd_job*> members;
        LaunchShape shape{};
        DevBuf descs; // LineJob array, one per member (solve 0)
        bool fp32 = false;
    };
    std::vector<std::unique_ptr<Group>> groups;
    std::vector<zqd_job*> solo; // multi-solve (imaginary-time) jobs run on their own
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0;
    uint32_t launches = 0;
    ~zqd_batch() {
        if (stream) cudaStreamSynchronize(stream);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace zqd {
template <typename T> static int upload_group(zqd_batch* B, zqd_batch::Group* g) {
    std::vector<LineJob<T>> descs;
    for (zqd_job* J : g->members) {
        descs.push_back(line_job_desc<T>(J, 0));
        g->shape.threads = std::max(g->shape.threads, J->threads);
        g->shape.smem = std::max(g->shape.smem, J->smem);
        J->h2d += sizeof(LineJob<T>);
    }
    int rc = g->descs.alloc(descs.size() * sizeof(LineJob<T>));
    if (rc) return rc;
    ZQD_CUDA(cudaMemcpyAsync(g->descs.p, descs.data(), descs.size() * sizeof(LineJob<T>), cudaMemcpyHostToDevice, B->stream));
    ZQD_CUDA(cudaStreamSynchronize(B->stream));
    return ZQD_OK;
}
} // namespace zqd

extern "C" int zqd_batch_create(const zqd_options* const* opts, uint32_t njobs, zqd_batch** out) {
    if (!opts || !out) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    *out = nullptr;
    std::unique_ptr<zqd_batch> B(new (std::nothrow) zqd_batch());
    if (!B) return fail(ZQD_ERR_OUT_OF_MEMORY, "host allocation failed");
    for (uint32_t i = 0; i < njobs; ++i) {
        zqd_job* J = nullptr;
        int rc = zqd_job_create(opts[i], &J);
        if (rc) return rc;
        B->jobs.emplace_back(J, zqd_job_destroy);
    }
    ZQD_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    ZQD_CUDA(cudaEventCreate(&B->ev0));
    ZQD_CUDA(cudaEventCreate(&B->ev1));
    // group single-solve jobs by kernel instantiation (precision, states, cluster size)
    std::vector<bool> done(njobs, false);
    for (uint32_t i = 0; i < njobs; ++i) {
        if (done[i]) continue;
        zqd_job* a = B->jobs[i].get();
        done[i] = true;
        if (a->nsolve > 1 || a->d > 1) { // multi-solve and N-D jobs run on their own stream
            B->solo.push_back(a);
            continue;
        }
        std::unique_ptr<zqd_batch::Group> g(new zqd_batch::Group());
        g->members.push_back(a);
        g->fp32 = a->fp32;
        g->shape = LaunchShape{a->S, a->C, a->E, 0, 0, B->stream};
        g->shape.lrmax = a->lrmax;
        for (uint32_t k = i + 1; k < njobs; ++k) {
            zqd_job* b = B->jobs[k].get();
            if (!done[k] && b->d == 1 && b->nsolve == 1 && b->fp32 == a->fp32 && b->S == a->S && b->C == a->C &&
                b->r_global == a->r_global && b->lrmax == a->lrmax && b->u_smem == a->u_smem) {
                g->members.push_back(b);
                done[k] = true;
            }
        }
        int rc = g->fp32 ? upload_group<float>(B.get(), g.get()) : upload_group<double>(B.get(), g.get());
        if (rc) return rc;
        B->groups.push_back(std::move(g));
    }
    *out = B.release();
    return ZQD_OK;
}

extern "C" int zqd_batch_run(zqd_batch* B) {
    if (!B) return fail(ZQD_ERR_INVALID_INPUT, "NULL BATCH");
    B->launches = 0;
    for (auto& g : B->groups)
        for (zqd_job* J : g->members) {
            const int rc = g->fp32 ? refresh_line_tables<float>(J) : refresh_line_tables<double>(J);
            if (rc) return rc;
            if (J->o.pot_td) ZQD_CUDA(cudaStreamSynchronize(J->stream));
        }
    ZQD_CUDA(cudaEventRecord(B->ev0, B->stream));
    for (auto& g : B->groups) {
        int rc = g->fp32 ? launch_line_s<float>(&g->shape, g->descs.p, (int)g->members.size())
                         : launch_line_s<double>(&g->shape, g->descs.p, (int)g->members.size());
        if (rc) return rc;
        ++B->launches;
    }
    ZQD_CUDA(cudaEventRecord(B->ev1, B->stream));
    for (zqd_job* J : B->solo) { // runs on its own stream, overlapping the grouped launches
        int rc = zqd_job_run(J);
        if (rc) return rc;
        B->launches += (uint32_t)J->nsolve;
    }
    ZQD_CUDA(cudaStreamSynchronize(B->stream));
    float ms = 0;
    ZQD_CUDA(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
    for (zqd_job* J : B->solo) ms = std::max(ms, J->last_ms);
    B->last_ms = ms;
    for (auto& g : B->groups)
        for (zqd_job* J : g->members) {
            J->last_ms = ms;
            if (int rc = mark_all_ended(J)) return rc;
        }
    return ZQD_OK;
}

// One grouped launch of 1-D single-solve jobs of the same precision, state count and cluster
// shape (the batch's grouping, for callers that hold the jobs themselves); waits for it.
int zqd::run_line_group(const std::vector<zqd_job*>& jobs, cudaStream_t st, float* ms) {
    if (jobs.empty()) return ZQD_OK;
    const zqd_job* a = jobs[0];
    for (const zqd_job* J : jobs)
        if (J->d != 1 || J->nsolve != 1 || J->fp32 != a->fp32 || J->S != a->S || J->C != a->C || J->r_global != a->r_global ||
            J->lrmax != a->lrmax || J->u_smem != a->u_smem)
            return fail(ZQD_ERR_INVALID_INPUT, "JOBS OF ONE GROUP MUST SHARE PRECISION, STATES AND CLUSTER SHAPE");
    LaunchShape sh{a->S, a->C, a->E, 0, 0, st};
    sh.lrmax = a->lrmax;
    for (const zqd_job* J : jobs) {
        sh.threads = std::max(sh.threads, J->threads);
        sh.smem = std::max(sh.smem, J->smem);
    }
    DevBuf descs;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ZQD_CUDA(cudaEventCreate(&e0));
    ZQD_CUDA(cudaEventCreate(&e1));
    auto go = [&]() -> int {
        int rc;
        if (a->fp32) {
            std::vector<LineJob<float>> d;
            for (zqd_job* J : jobs) d.push_back(line_job_desc<float>(J, 0));
            if ((rc = descs.alloc(d.size() * sizeof(d[0]), st))) return rc;
            ZQD_CUDA(cudaMemcpyAsync(descs.p, d.data(), d.size() * sizeof(d[0]), cudaMemcpyHostToDevice, st));
            ZQD_CUDA(cudaEventRecord(e0, st));
            if ((rc = launch_line_s<float>(&sh, descs.p, (int)jobs.size()))) return rc;
        } else {
            std::vector<LineJob<double>> d;
            for (zqd_job* J : jobs) d.push_back(line_job_desc<double>(J, 0));
            if ((rc = descs.alloc(d.size() * sizeof(d[0]), st))) return rc;
            ZQD_CUDA(cudaMemcpyAsync(descs.p, d.data(), d.size() * sizeof(d[0]), cudaMemcpyHostToDevice, st));
            ZQD_CUDA(cudaEventRecord(e0, st));
            if ((rc = launch_line_s<double>(&sh, descs.p, (int)jobs.size()))) return rc;
        }
        ZQD_CUDA(cudaEventRecord(e1, st));
        ZQD_CUDA(cudaStreamSynchronize(st));
        float t = 0;
        ZQD_CUDA(cudaEventElapsedTime(&t, e0, e1));
        for (zqd_job* J : jobs) {
            J->last_ms = t;
            if ((rc = mark_all_ended(J))) return rc;
        }
        if (ms) *ms = t;
        return ZQD_OK;
    };
    const int rc = go();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// One launch advancing single-solve 1-D jobs of one kernel shape by up to nsteps each, every job
// from its own position (continuous batching: members join and leave between launches).  Like
// zqd_job_step per member; waits for the launch.
int zqd::step_line_group(const std::vector<zqd_job*>& jobs, uint32_t nsteps, cudaStream_t st) {
    if (jobs.empty() || nsteps == 0) return ZQD_OK;
    const zqd_job* a = jobs[0];
    for (const zqd_job* J : jobs)
        if (J->d != 1 || J->nsolve != 1 || J->fp32 != a->fp32 || J->S != a->S || J->C != a->C || J->r_global != a->r_global ||
            J->lrmax != a->lrmax || J->u_smem != a->u_smem)
            return fail(ZQD_ERR_INVALID_INPUT, "JOBS OF ONE GROUP MUST SHARE PRECISION, STATES AND CLUSTER SHAPE");
    LaunchShape sh{a->S, a->C, a->E, 0, 0, st};
    sh.lrmax = a->lrmax;
    std::vector<int> i0(jobs.size()), i1(jobs.size());
    for (size_t k = 0; k < jobs.size(); ++k) {
        zqd_job* J = jobs[k];
        if (!J->stepping) {
            reset_progress(J);
            J->stepping = true;
            J->last_ms = 0;
            const int rc = J->fp32 ? refresh_line_tables<float>(J) : refresh_line_tables<double>(J);
            if (rc) return rc;
            ZQD_CUDA(cudaStreamSynchronize(J->stream));
        }
        if (J->step_solve >= J->nsolve) return fail(ZQD_ERR_INVALID_INPUT, "JOB OF THE GROUP HAS ALREADY FINISHED");
        i0[k] = J->solve_rows[0];
        const long long want = i0[k] == 0 ? (long long)nsteps : (long long)i0[k] + nsteps - 1;
        i1[k] = (int)std::min<long long>((long long)J->o.iterations, want);
        sh.threads = std::max(sh.threads, J->threads);
        sh.smem = std::max(sh.smem, J->smem);
    }
    DevBuf descs;
    std::vector<int> flags(2 * jobs.size());
    auto go = [&](auto tag) -> int {
        using T = decltype(tag);
        std::vector<LineJob<T>> d;
        for (size_t k = 0; k < jobs.size(); ++k) {
            d.push_back(line_job_desc<T>(jobs[k], 0));
            d.back().i0 = i0[k];
            d.back().i1 = i1[k];
            jobs[k]->h2d += sizeof(LineJob<T>);
        }
        int rc;
        if ((rc = descs.alloc(d.size() * sizeof(d[0]), st))) return rc;
        ZQD_CUDA(cudaMemcpyAsync(descs.p, d.data(), d.size() * sizeof(d[0]), cudaMemcpyHostToDevice, st));
        if ((rc = launch_line_s<T>(&sh, descs.p, (int)jobs.size()))) return rc;
        return ZQD_OK;
    };
    int rc = a->fp32 ? go(float{}) : go(double{});
    if (rc) return rc;
    ZQD_CUDA(cudaStreamSynchronize(st)); // the launch first, then the copies into pageable memory
    for (size_t k = 0; k < jobs.size(); ++k) { // rows written and the end flag of every member
        ZQD_CUDA(cudaMemcpyAsync(&flags[2 * k], jobs[k]->rows.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        ZQD_CUDA(cudaMemcpyAsync(&flags[2 * k + 1], jobs[k]->done.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    ZQD_CUDA(cudaStreamSynchronize(st));
    for (size_t k = 0; k < jobs.size(); ++k) {
        zqd_job* J = jobs[k];
        J->d2h += 2 * sizeof(int);
        J->solve_rows[0] = flags[2 * k];
        if (flags[2 * k + 1]) {
            J->solve_ended[0] = 1;
            J->step_solve = 1;
        }
    }
    return ZQD_OK;
}

// Descriptor of a created single-solve 1-D job for the persistent service kernel: the whole solve
// in one claim, rows published through `progress` (a device pointer into pinned host memory).
size_t zqd::line_desc_bytes(bool fp32) { return fp32 ? sizeof(LineJob<float>) : sizeof(LineJob<double>); }

int zqd::service_desc(zqd_job* J, void* out, int* progress) {
    if (J->d != 1 || J->nsolve != 1 || J->C != 1) return fail(ZQD_ERR_INVALID_INPUT, "SERVICE JOBS ARE SINGLE-CTA 1-D SOLVES");
    if (!J->stepping) {
        reset_progress(J);
        J->stepping = true;
        const int rc = J->fp32 ? refresh_line_tables<float>(J) : refresh_line_tables<double>(J);
        if (rc) return rc;
        ZQD_CUDA(cudaStreamSynchronize(J->stream));
    }
    if (J->fp32) {
        LineJob<float> d = line_job_desc<float>(J, 0);
        d.progress = progress;
        std::memcpy(out, &d, sizeof(d));
    } else {
        LineJob<double> d = line_job_desc<double>(J, 0);
        d.progress = progress;
        std::memcpy(out, &d, sizeof(d));
    }
    J->h2d += line_desc_bytes(J->fp32);
    return ZQD_OK;
}

// a service job's solve ended on the device: its progress as after zqd_job_run
int zqd::service_job_ended(zqd_job* J) { return mark_all_ended(J); }

// rows the service kernel has published for the job (zqd_job_observables reads up to here)
void zqd::service_job_rows(zqd_job* J, int rows) {
    if (!J->solve_rows.empty() && rows > J->solve_rows[0]) J->solve_rows[0] = rows;
}

extern "C" int zqd_batch_result(zqd_batch* B, uint32_t i, zqd_result** out) {
    if (!B || !out) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    if (i >= B->jobs.size()) return fail(ZQD_ERR_NOT_FOUND, "JOB INDEX OUT OF RANGE");
    return zqd_job_result(B->jobs[i].get(), out);
}

extern "C" double zqd_batch_device_ms(const zqd_batch* B) { return B ? (double)B->last_ms : 0.0; }
extern "C" uint32_t zqd_batch_launches(const zqd_batch* B) { return B ? B->launches : 0; }
extern "C" void zqd_batch_destroy(zqd_batch* B) { delete B; }

extern "C" int zqd_run_batch(const zqd_options* const* opts, uint32_t njobs, zqd_result** results) {
    if (!opts || !results) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    for (uint32_t i = 0; i < njobs; ++i) results[i] = nullptr;
    zqd_batch* B = nullptr;
    int rc = zqd_batch_create(opts, njobs, &B);
    if (rc) return rc;
    std::unique_ptr<zqd_batch, void (*)(zqd_batch*)> guard(B, zqd_batch_destroy);
    if ((rc = zqd_batch_run(B))) return rc;
    for (uint32_t i = 0; i < njobs; ++i) {
        if ((rc = zqd_batch_result(B, i, &results[i]))) {
            for (uint32_t k = 0; k < i; ++k) {
                zqd_result_destroy(results[k]);
                results[k] = nullptr;
            }
            return rc;
        }
    }
    return ZQD_OK;
}

extern "C" int zqd_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

extern "C" int zqd_set_device(int dev) {
    ZQD_CUDA(cudaSetDevice(dev));
    return ZQD_OK;
}
