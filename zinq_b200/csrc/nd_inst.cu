// nd_inst.cu -- the 2-D / 3-D driver for one (precision, state count) pair.
// Compiled once per pair with -DZQD_T=<double|float> -DZQD_S=<1..4>
// -DZQD_ND_CREATE=<symbol> -DZQD_ND_RUN=<symbol> -DZQD_ND_STEP=<symbol>.
//
// A solve (src/quantum_dynamics.zig:860-950) is a stream-ordered sequence of
// axis passes (nd_kernels.cuh); nothing returns to the host until the end.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "job.h"
#include "nd_kernels.cuh"

#if !defined(ZQD_T) || !defined(ZQD_S) || !defined(ZQD_ND_CREATE) || !defined(ZQD_ND_RUN) || !defined(ZQD_ND_STEP)
#error "nd_inst.cu needs -DZQD_T, -DZQD_S, -DZQD_ND_CREATE, -DZQD_ND_RUN and -DZQD_ND_STEP"
#endif

namespace zqd {
namespace {

using T = ZQD_T;
constexpr int S = ZQD_S;
constexpr int NSYM = S * (S + 1) / 2;

NdJob<T> describe(zqd_job* J) {
    NdJob<T> D{};
    const Opts& o = J->o;
    D.d = J->d;
    D.n = J->n;
    while ((1 << D.logn) < J->n) ++D.logn;
    D.S = S;
    D.N = J->N;
    for (int j = 0; j < D.d; ++j) {
        D.lo[j] = o.bounds[2 * j];
        D.span[j] = o.bounds[2 * j + 1] - o.bounds[2 * j];
        D.mass[j] = o.mass[j];
        D.dkunit[j] = 6.283185307179586476925286766559 / D.span[j];
        D.x0[j] = o.pos[j];
        D.p0[j] = o.mom[j];
        D.gamma[j] = o.gamma[j];
        if (o.has_cap) {
            D.cap_lo[j] = o.cap_bounds[2 * j];
            D.cap_hi[j] = o.cap_bounds[2 * j + 1];
        }
    }
    double dr = 1; // Grid.init (wavepacket.zig:44-53)
    for (int j = 0; j < D.d; ++j) dr *= D.span[j] / (double)J->n;
    D.dr = dr;
    D.dk = dr / (double)J->N;
    D.dt_re = o.imag_nstate ? 0.0 : o.time_step;
    D.dt_im = o.imag_nstate ? -o.time_step : 0.0;
    D.adiabatic = o.adiabatic;
    D.track = o.has_cap && o.cap_track;
    D.has_cap = o.has_cap;
    D.cap_exp = o.cap_exponent;
    D.ic_state = (int)o.ic_state;
    D.ic_adia = o.ic_adiabatic;
    D.psi = J->psi_save.as<cx<T>>();
    D.phi = J->phi.as<cx<T>>();
    D.psi0 = J->psi0.as<cx<T>>();
    D.psi_init = J->psi_init.as<cx<T>>();
    D.orth = J->orth.as<cx<T>>();
    D.R = J->R.as<Tab<T>>();
    D.V = J->V.as<double>();
    D.U = J->U.as<double>();
    D.capw = J->capw.as<double>();
    D.tw = J->tw.as<Tab<T>>();
    D.kphase = J->expk.as<double2>();
    D.axis = reinterpret_cast<const double4*>(J->expk.as<double2>() + (size_t)J->d * J->n);
    D.part = J->part.as<double>();
    D.nparts = J->part.bytes / (NDV * 2 * sizeof(double));
    D.rows_per_cta = J->nd_rows;
    D.tile = J->nd_tile;
    while ((1 << D.logtile) < J->nd_tile) ++D.logtile;
    D.stopped = J->flags.as<int>();
    D.err = J->flags.as<int>() + 2;
    D.nsum = J->book.as<NdBook>()->scal; // where nd_reduce_kernel leaves the norm's sum (device address)
    D.pot = J->pot.dev;
    return D;
}

// Row CTAs of at most 256 threads with several states take the 256-thread kernel form (up
// to 255 registers).  One state keeps the 512-thread form: its sweep fits in 128 registers
// and two 256-thread CTAs per SM hide more latency than extra registers would.
inline bool row_narrow(unsigned threads) { return S > 1 && threads <= 256; }

using RowTmaKernel = void (*)(NdJob<T>, CUtensorMap, CUtensorMap, NdRowTma, size_t, NdFin);
// the momentum-copy form of the TMA row kernel (one state: with several it holds too many registers
// for the per-block kernel's speed, and those launches take that kernel), or null
inline RowTmaKernel row_tma_phi(int d) {
    if constexpr (S == 1)
        return d == 2 ? nd_row_tma_kernel<T, 2, S, true> : nd_row_tma_kernel<T, 3, S, true>;
    else
        return nullptr;
}
// the 512-thread plain form of the TMA row kernel (one or two states), or null
inline RowTmaKernel row_tma_wide(int d) {
    if constexpr (S <= 2)
        return d == 2 ? nd_row_tma_kernel<T, 2, S, false, NDR_THREADS_WIDE> : nd_row_tma_kernel<T, 3, S, false, NDR_THREADS_WIDE>;
    else
        return nullptr;
}

struct Launch {
    zqd_job* J;
    NdJob<T> D;
    size_t nrow_blocks, ntile_blocks, ngrid;
    // partial-sum regions (in blocks)
    size_t R0, R1, R2, K, G;

    int row(uint32_t mode, uint32_t obs, size_t region, bool nostop = false, NdFin f = NdFin{}, cx<T>* wout = nullptr) {
        NdJob<T> d = D;
        d.wfn_out = wout;
        if (nostop) d.stopped = J->flags.as<int>() + 1; // a flag nothing sets
        if (J->nd_row_tma && (!(mode & RM_PHI) || J->nd_row_tma_phi)) {
            NdRowTma P{};
            P.mode = mode;
            P.obs = obs;
            P.logL = J->nd_row_tma_logL;
            P.nitems = (unsigned)(J->N / J->n >> P.logL);
            bool withhold = false;
            P.wait_cycles = tma_wait_budget(NDT_WAIT_CYCLES, &withhold);
            P.withhold = withhold;
            const size_t smem = ndr_smem_bytes<T>(S, 1 << P.logL, J->n);
            const unsigned nt = (unsigned)((S * J->n << P.logL) / 8), nb = (unsigned)J->nd_row_tma_ctas;
            const CUtensorMap* map = reinterpret_cast<const CUtensorMap*>(J->nd_row_map);
            const CUtensorMap* mphi = reinterpret_cast<const CUtensorMap*>(J->nd_row_map_phi);
            RowTmaKernel kern = D.d == 2 ? nd_row_tma_kernel<T, 2, S, false> : nd_row_tma_kernel<T, 3, S, false>;
            if (!(obs & ~(uint32_t)(WM_POP | WM_NORM)) && nt <= (unsigned)NDR_THREADS) // populations and norm only
                kern = D.d == 2 ? nd_row_tma_kernel<T, 2, S, false, NDR_THREADS, true>
                                : nd_row_tma_kernel<T, 3, S, false, NDR_THREADS, true>;
            if (mode & RM_PHI) kern = row_tma_phi(D.d); // only where nd_row_tma_phi (one state)
            if (nt > (unsigned)NDR_THREADS) kern = row_tma_wide(D.d);
            kern<<<nb, nt, smem, J->stream>>>(d, *map, *mphi, P, region, f);
            ZQD_CUDA(cudaGetLastError());
            return ZQD_OK;
        }
        const size_t smem = nd_smem_bytes<T>(2, S * J->nd_rows, J->n);
        const unsigned nb = (unsigned)nrow_blocks, nt = (unsigned)J->nd_row_threads;
        if (row_narrow(nt)) {
            if (D.d == 2) nd_row_kernel<T, 2, S, 256><<<nb, nt, smem, J->stream>>>(d, mode, obs, region, f);
            else nd_row_kernel<T, 3, S, 256><<<nb, nt, smem, J->stream>>>(d, mode, obs, region, f);
        } else {
            if (D.d == 2) nd_row_kernel<T, 2, S, 512><<<nb, nt, smem, J->stream>>>(d, mode, obs, region, f);
            else nd_row_kernel<T, 3, S, 512><<<nb, nt, smem, J->stream>>>(d, mode, obs, region, f);
        }
        ZQD_CUDA(cudaGetLastError());
        return ZQD_OK;
    }
    int tile(int axis, uint32_t mode, size_t region, bool nostop = false, NdFin f = NdFin{}) {
        NdJob<T> d = D;
        if (nostop) d.stopped = J->flags.as<int>() + 1;
        const size_t smem = nd_smem_bytes<T>(2, J->nd_tile, J->n);
        const dim3 grid((unsigned)ntile_blocks, S);
        if (D.d == 2) nd_tile_kernel<T, 2><<<grid, J->nd_tile_threads, smem, J->stream>>>(d, axis, mode, region, f);
        else nd_tile_kernel<T, 3><<<grid, J->nd_tile_threads, smem, J->stream>>>(d, axis, mode, region, f);
        ZQD_CUDA(cudaGetLastError());
        return ZQD_OK;
    }
    // the TMA-staged persistent form of a tile pass: over psi (modes TM_FWD, TM_KPHASE, TM_INV) or
    // over phi (TM_FWD, or TM_FWD | TM_KOBS: the momentum sums into region `region`, finalized by f)
    int tile_tma(int axis, uint32_t mode, bool phi = false, size_t region = 0, bool nostop = false, NdFin f = NdFin{}) {
        NdJob<T> d = D;
        if (nostop) d.stopped = J->flags.as<int>() + 1;
        const CUtensorMap* map = reinterpret_cast<const CUtensorMap*>(phi ? J->nd_maps_phi[axis] : J->nd_maps[axis]);
        NdTma P{};
        P.axis = axis;
        P.mode = mode;
        P.logW = J->nd_tma_logW;
        const int lstride = D.logn * (D.d - 1 - axis);
        int logN = 0;
        while (((size_t)1 << logN) < J->N) ++logN;
        P.logtiles = logN - D.logn - P.logW;
        P.logO = logN - D.logn - lstride;
        P.nitems = (unsigned)S << P.logtiles;
        P.ncols = (unsigned)(S * ntile_blocks); // the momentum region's width
        const size_t smem = ndt_smem_bytes<T>(1 << P.logW, J->n);
        const unsigned threads = (unsigned)((J->n << P.logW) / 8);
        // the momentum sums are grouped per CTA: that launch's grid is the job's own (never the
        // server's cap) and fits the region
        const unsigned grid = (mode & TM_KOBS) ? (unsigned)std::min<size_t>((size_t)J->nd_tma_ctas_full, P.ncols)
                                               : (unsigned)J->nd_tma_ctas;
        bool withhold = false;
        P.wait_cycles = tma_wait_budget(NDT_WAIT_CYCLES, &withhold);
        P.withhold = withhold;
        if (D.d == 2) nd_tile_tma_kernel<T, 2><<<grid, threads, smem, J->stream>>>(d, *map, P, region, f);
        else nd_tile_tma_kernel<T, 3><<<grid, threads, smem, J->stream>>>(d, *map, P, region, f);
        ZQD_CUDA(cudaGetLastError());
        return ZQD_OK;
    }
    int ptile(int axis, uint32_t mode) { return J->nd_tma ? tile_tma(axis, mode) : tile(axis, mode, 0); }
    // forward along axes d-2..1, forward + kinetic phase + inverse along axis 0, inverse along 1..d-2;
    // `first`: mode bits of the first of these launches only (TM_SCALE)
    int step_tiles(uint32_t first = 0) {
        int rc;
        for (int a = D.d - 2; a >= 1; --a, first = 0)
            if ((rc = ptile(a, TM_FWD | first))) return rc;
        if ((rc = ptile(0, TM_FWD | TM_KPHASE | TM_INV | first))) return rc;
        for (int a = 1; a <= D.d - 2; ++a)
            if ((rc = ptile(a, TM_INV))) return rc;
        return ZQD_OK;
    }
    double* scal() const { return J->book.as<NdBook>()->scal; }
    // Hamiltonian.update at time t (with_R: and Propagator.update); with sign tracking, the global
    // eigenvector alignment with the previous update follows (wavepacket.zig:157-167)
    int table(double t, int with_R) {
        if (!needs_sign_tracking(J->o, S, J->nsolve)) {
            nd_table_kernel<T, S><<<(unsigned)((J->N + 127) / 128), 128, 0, J->stream>>>(D, t, with_R);
            ZQD_CUDA(cudaGetLastError());
            return ZQD_OK;
        }
        const unsigned nb = (unsigned)std::min<size_t>(ngrid, (J->N + 127) / 128);
        nd_table_sign_kernel<T, S><<<nb, 128, 0, J->stream>>>(D, t, with_R, G);
        ZQD_CUDA(cudaGetLastError());
        int rc = reduce(G, G + nb, S);
        if (rc) return rc;
        nd_sign_flip_kernel<S><<<(unsigned)ngrid, 256, 0, J->stream>>>(D.U, J->N, scal(), D.stopped);
        ZQD_CUDA(cudaGetLastError());
        return ZQD_OK;
    }
    // scalar sums of slots [0, nv) over partial blocks [b0, b1) into scal()
    int reduce(size_t b0, size_t b1, int nv, bool clear = false) {
        nd_reduce_kernel<<<1, 32 * nv, 0, J->stream>>>(D.part, D.nparts, b0, b1, nv, D.stopped, scal(), clear ? 1 : 0);
        ZQD_CUDA(cudaGetLastError());
        return ZQD_OK;
    }
    // momentum observables of phi (the forward transform along the last axis is already done)
    int kobs(bool nostop, NdFin f) {
        int rc;
        if (J->nd_tma) {
            for (int a = D.d - 2; a >= 1; --a)
                if ((rc = tile_tma(a, TM_FWD, true, 0, nostop))) return rc;
            return tile_tma(0, TM_FWD | TM_KOBS, true, K, nostop, f);
        }
        for (int a = D.d - 2; a >= 1; --a)
            if ((rc = tile(a, TM_FWD | TM_PHI, 0, nostop))) return rc;
        return tile(0, TM_FWD | TM_KOBS | TM_PHI, K, nostop, f);
    }
};

// resident CTAs per SM the tile pass's persistent grid may use: the job server's setting, else
// all that fit (the tile pass reduces nothing, so its grid changes no result)
inline int tma_ctas_per_sm_cap(const zqd_job* J) { return J->o.tma_ctas_per_sm > 0 ? J->o.tma_ctas_per_sm : 1 << 20; }

// The TMA-staged tile pass: lines per tile W (a power of two, W <= n) with rows of W c >= 16
// bytes (an even number of 8-byte words), W n / 8 threads (whole warps, at most 512) and two
// stages within the shared-memory budget; by default the widest W up to 64-byte rows.  w_override
// (the autotuner's candidate or table entry): 0 keeps the default, -1 keeps the earlier tile
// kernel, else W.  ZQD_ND_TMA=0 in the environment also keeps it.
int setup_tma(zqd_job* J, int w_override) {
    constexpr int c = (int)sizeof(cx<T>), E = c / 8;
    const int n = J->n, d = J->d;
    const size_t budget = 200 * 1024;
    J->nd_tma = false;
    const char* env = getenv("ZQD_ND_TMA");
    if ((env && env[0] == '0') || w_override < 0) return ZQD_OK;
    int dev = 0, sms = 148;
    ZQD_CUDA(cudaGetDevice(&dev));
    ZQD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (auto f : {nd_tile_tma_kernel<T, 2>, nd_tile_tma_kernel<T, 3>})
        ZQD_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget));
    auto fits = [&](int W) {
        return W >= 1 && W <= n && (E * W) % 2 == 0 && (size_t)W * n / 8 <= 512 && ((size_t)W * n / 8) % 32 == 0 &&
               ndt_smem_bytes<T>(W, n) <= budget;
    };
    // resident CTAs on the device for a W (the job's own count: the shape, and with it every result,
    // must not depend on the server's cap, which only trims the grid of the passes that sum nothing)
    auto ctas_for = [&](int W, int& ctas) -> int {
        const int threads = W * n / 8;
        int per_sm = 0;
        ZQD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, d == 2 ? (const void*)nd_tile_tma_kernel<T, 2> : (const void*)nd_tile_tma_kernel<T, 3>, threads,
            ndt_smem_bytes<T>(W, n)));
        ctas = std::max(1, per_sm) * sms;
        return ZQD_OK;
    };
    const size_t lines = J->N / (size_t)n; // lines of one state along any axis
    int W = 0;
    if (w_override > 0) W = w_override;
    if (W) {
        if (!fits(W) || lines % (size_t)W) return fail(ZQD_ERR_UNSUPPORTED, "TMA TILE SHAPE OUTSIDE THE KERNEL'S LIMITS");
    } else {
        // measured: 32- to 64-byte rows win; on 2-D FP32 lines of 512 points 32-byte rows (twice the
        // tiles) were 3-5 % faster per step than 64-byte rows with 1 to 3 states
        const int wmax = (c == 8 && d == 2 && n == 512) ? 32 / c : 64 / c;
        for (int w = std::max(1, wmax); w >= 1 && !W; w >>= 1)
            if (fits(w) && lines % (size_t)w == 0) W = w;
        if (!W) return ZQD_OK; // no shape fits: the earlier tile kernel runs
    }
    int logW = 0;
    while ((1 << logW) < W) ++logW;
    int ctas = 0, rc;
    if ((rc = ctas_for(W, ctas))) return rc;
    const size_t items = (size_t)S * (lines / W);
    J->nd_tma_ctas_full = (int)std::min<size_t>(items, (size_t)ctas);
    const int per_sm = ctas / sms;
    J->nd_tma_ctas = (int)std::min<size_t>(items, (size_t)std::min(per_sm, tma_ctas_per_sm_cap(J)) * sms);
    J->nd_tma_logW = logW;
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    for (int a = 0; a + 1 < d; ++a) {
        const int lstride = logn * (d - 1 - a);
        const uint64_t st = (uint64_t)1 << lstride, O = J->N / ((uint64_t)n * st);
        const uint64_t dims[3] = {(uint64_t)E * st, (uint64_t)n, (uint64_t)S * O};
        const uint32_t box[3] = {(uint32_t)(E * W), (uint32_t)std::min(n, 256), 1};
        const int l2 = W * c >= 128 ? 128 : 0; // (promotion measured no faster on narrower rows)
        const int e = encode_map_3d(reinterpret_cast<CUtensorMap*>(J->nd_maps[a]), J->psi_save.p, dims, st * c,
                                    (uint64_t)n * st * c, box, l2) ||
                      encode_map_3d(reinterpret_cast<CUtensorMap*>(J->nd_maps_phi[a]), J->phi.p, dims, st * c,
                                    (uint64_t)n * st * c, box, l2);
        if (e) return fail(ZQD_ERR_DEVICE, "cuTensorMapEncodeTiled failed for the tile pass");
    }
    J->nd_tma = true;
    return ZQD_OK;
}

// The TMA-staged row pass: L rows (a power of two dividing N/n) per block with L n c >= 1024 bytes
// (the stages keep the 128-byte swizzle's 1024-byte alignment), S L n / 8 threads (whole warps, at
// most 256, or 512 for one or two states on lines too long for 256; the momentum copy then takes
// the per-block kernel) and two stages within the budget; by default the largest L of at most 256
// threads (the wide form only where no 256-thread block fits).  The grid takes every resident CTA
// (jobs created by the server too: its observables' sums are grouped per CTA, so a job's results
// depend on its grid, which must not change with where it runs).
// l_override: 0 keeps the default, -1 keeps the earlier row kernel, else L.  ZQD_ND_TMA=0 also
// keeps it.
int choose_row_tma(zqd_job* J, int l_override) {
    constexpr int c = (int)sizeof(cx<T>);
    const int n = J->n, d = J->d;
    const size_t budget = 200 * 1024, lines = J->N / (size_t)n;
    J->nd_row_tma = false;
    const char* env = getenv("ZQD_ND_TMA");
    if ((env && env[0] == '0') || l_override < 0) return ZQD_OK;
    int dev = 0, sms = 148;
    ZQD_CUDA(cudaGetDevice(&dev));
    ZQD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (auto f : {nd_row_tma_kernel<T, 2, S, false>, nd_row_tma_kernel<T, 3, S, false>,
                   nd_row_tma_kernel<T, 2, S, false, NDR_THREADS, true>, nd_row_tma_kernel<T, 3, S, false, NDR_THREADS, true>})
        ZQD_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget));
    for (int dd : {2, 3})
        for (RowTmaKernel f : {row_tma_wide(dd), row_tma_phi(dd)})
            if (f) ZQD_CUDA(cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget));
    auto threads_of = [&](int L) { return (size_t)S * L * n / 8; };
    auto fits = [&](int L) {
        const size_t t = threads_of(L);
        // whole warps: the block reduction's shuffles run on full warps
        return L >= 1 && (size_t)L <= lines && lines % (size_t)L == 0 && (size_t)L * n * c >= 1024 && t % 32 == 0 &&
               (t <= (size_t)NDR_THREADS || (t <= (size_t)NDR_THREADS_WIDE && row_tma_wide(d))) &&
               ndr_smem_bytes<T>(S, L, n) <= budget;
    };
    auto ctas_for = [&](int L, int& ctas) -> int {
        const unsigned nt = (unsigned)threads_of(L);
        const void* f = nt > (unsigned)NDR_THREADS ? (const void*)row_tma_wide(d)
                        : d == 2                   ? (const void*)nd_row_tma_kernel<T, 2, S, false>
                                                   : (const void*)nd_row_tma_kernel<T, 3, S, false>;
        int per_sm = 0;
        ZQD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, (int)nt, ndr_smem_bytes<T>(S, L, n)));
        ctas = std::max(1, per_sm) * sms;
        return ZQD_OK;
    };
    int L = 0;
    if (l_override > 0) L = l_override;
    if (L) {
        if (!fits(L)) return fail(ZQD_ERR_UNSUPPORTED, "TMA ROW-BLOCK SHAPE OUTSIDE THE KERNEL'S LIMITS");
    } else { // the largest block of at most 256 threads (measured: fewer, larger CTAs win), else the wide form
        for (int l = std::max(1, 4096 / (S * n)); l >= 1 && !L; l >>= 1)
            if (fits(l) && (threads_of(l) <= (size_t)NDR_THREADS || !fits(l / 2))) L = l;
        if (!L) return ZQD_OK; // no shape fits: the earlier row kernel runs
    }
    int logL = 0;
    while ((1 << logL) < L) ++logL;
    int ctas = 0, rc;
    if ((rc = ctas_for(L, ctas))) return rc;
    J->nd_row_tma_ctas = (int)std::min<size_t>(lines / L, (size_t)ctas);
    J->nd_row_tma_logL = logL;
    // the momentum-copy form holds the end-of-step state in registers besides the sweep's: with one
    // state it keeps up with the per-block kernel, with several it does not (one CTA per SM)
    J->nd_row_tma_phi = row_tma_phi(d) && threads_of(L) <= (size_t)NDR_THREADS;
    J->nd_row_tma = true;
    return ZQD_OK;
}

// the row pass's tensor maps over psi and phi (after they are allocated)
int encode_row_tma(zqd_job* J) {
    constexpr int c = (int)sizeof(cx<T>);
    const int L = 1 << J->nd_row_tma_logL, n = J->n;
    const uint64_t rows_total = (uint64_t)S * J->N * c / 128;
    const uint64_t dims[3] = {16, rows_total, 1};
    const uint32_t box[3] = {16, (uint32_t)std::min<uint64_t>(256, (uint64_t)L * n * c / 128), 1};
    if (encode_map_3d(reinterpret_cast<CUtensorMap*>(J->nd_row_map), J->psi_save.p, dims, 128, rows_total * 128, box, 256,
                      true) ||
        encode_map_3d(reinterpret_cast<CUtensorMap*>(J->nd_row_map_phi), J->phi.p, dims, 128, rows_total * 128, box, 256,
                      true))
        return fail(ZQD_ERR_DEVICE, "cuTensorMapEncodeTiled failed for the row pass");
    return ZQD_OK;
}

} // namespace

int ZQD_ND_CREATE(zqd_job* J) {
    const size_t N = J->N, c = sizeof(cx<T>), tb = sizeof(Tab<T>);
    const Opts& o = J->o;
    const int n = J->n;
    // Launch shapes.  Row pass: L rows (all S states) per CTA, about 2048 points a CTA, at
    // least two CTAs per SM where the grid allows, within the shared-memory budget (two line
    // buffers; one thread per 8-point group).
    // Tile pass: Tn lines per CTA, rows of Tn * c >= 32 bytes (one sector), shrunk from
    // 128 bytes until the grid has two CTAs per SM.
    const int budget = 200 * 1024, sms2 = 2 * 148;
    const int max_items = 512; // 8-point groups of a CTA, one thread each
    J->nd_row_bufs = 2;
    if (S * n > 8 * max_items) return fail(ZQD_ERR_UNSUPPORTED, "GRID LINE TOO LONG FOR THE ROW PASS (states x npoint at most 4096)");
    static_assert(ND_IPT == 1, "launch shapes assume one 8-point group per thread");
    int L = std::max(1, std::min<int>((int)(N / n), 2048 / (S * n)));
    while (L > 1 && (N / n / L < (size_t)sms2 || nd_smem_bytes<T>(J->nd_row_bufs, S * L, n) > (size_t)budget)) L >>= 1;
    if (nd_smem_bytes<T>(J->nd_row_bufs, S * L, n) > (size_t)budget)
        return fail(ZQD_ERR_UNSUPPORTED, "GRID LINE TOO LONG FOR THE ROW PASS");
    J->nd_rows = L;
    J->nd_row_threads = std::max(32, (S * L * n / 8 + 31) / 32 * 32);
    const int tmin = std::max(1, (int)(32 / c));
    int Tn = std::min(n, (int)(128 / c));
    // at most 256 threads, except that long lines keep one 32-byte sector per row (up to 512 threads)
    while (Tn > 1 && ((Tn * n / 8 > 256 && (Tn > tmin || Tn * n / 8 > max_items)) ||
                      nd_smem_bytes<T>(2, Tn, n) > (size_t)budget || (Tn > tmin && (size_t)S * (N / n / Tn) < (size_t)sms2)))
        Tn >>= 1;
    if (nd_smem_bytes<T>(2, Tn, n) > (size_t)budget || Tn * n / 8 > max_items)
        return fail(ZQD_ERR_UNSUPPORTED, "GRID LINE TOO LONG FOR THE TILE PASS");
    J->nd_tile = Tn;
    ShapeOverride ov; // autotuned shape (or a candidate the autotuner measures), within the same limits
    if (lookup_shape(J->d, n, S, J->fp32, ov)) {
        if (ov.rows) {
            if ((size_t)ov.rows > N / n || (N / n) % (size_t)ov.rows || S * ov.rows * n / 8 > max_items ||
                nd_smem_bytes<T>(J->nd_row_bufs, S * ov.rows, n) > (size_t)budget)
                return fail(ZQD_ERR_UNSUPPORTED, "ROW-PASS SHAPE OUTSIDE THE KERNEL'S LIMITS");
            J->nd_rows = L = ov.rows;
            J->nd_row_threads = std::max(32, (S * L * n / 8 + 31) / 32 * 32);
        }
        if (ov.tile) {
            if (ov.tile > n || (N / n) % (size_t)ov.tile || ov.tile * n / 8 > max_items ||
                nd_smem_bytes<T>(2, ov.tile, n) > (size_t)budget)
                return fail(ZQD_ERR_UNSUPPORTED, "TILE-PASS SHAPE OUTSIDE THE KERNEL'S LIMITS");
            J->nd_tile = Tn = ov.tile;
        }
    }
    J->nd_tile_threads = std::max(32, (Tn * n / 8 + 31) / 32 * 32);
    int rc;
    // The TMA-staged row pass, where a shape fits: the per-block row kernel (the launches the TMA
    // form does not take) uses the same rows per block, so both write every column of a partial-sum
    // region, one column per block.
    if ((rc = choose_row_tma(J, ov.tma_rows))) return rc;
    if (J->nd_row_tma) {
        const int Lt = 1 << J->nd_row_tma_logL;
        if (S * Lt * n / 8 <= max_items && nd_smem_bytes<T>(J->nd_row_bufs, S * Lt, n) <= (size_t)budget) {
            J->nd_rows = L = Lt;
            J->nd_row_threads = std::max(32, (S * L * n / 8 + 31) / 32 * 32);
        } else {
            J->nd_row_tma = false;
        }
    }
    const size_t nrow_blocks = N / n / L, ntile_blocks = N / n / Tn;
    const size_t nparts = 3 * nrow_blocks + S * ntile_blocks + 1024;
    if ((rc = J->psi_save.alloc((size_t)S * N * c, J->stream))) return rc;
    if ((rc = J->phi.alloc((size_t)S * N * c, J->stream))) return rc;
    if ((o.has_spectrum || (o.write_mask & ZQD_WRITE_ACF)) && (rc = J->psi0.alloc((size_t)S * N * c, J->stream))) return rc;
    if (o.imag_nstate > 1 && (rc = J->orth.alloc((size_t)(o.imag_nstate - 1) * S * N * c, J->stream))) return rc;
    if ((rc = J->R.alloc((size_t)NSYM * N * tb, J->stream))) return rc;
    if ((rc = J->V.alloc((size_t)S * S * N * sizeof(double), J->stream))) return rc;
    if (S > 1 && (rc = J->U.alloc((size_t)S * S * N * sizeof(double), J->stream))) return rc;
    if (o.has_cap && (rc = J->capw.alloc(N * sizeof(double), J->stream))) return rc;
    if ((rc = J->tw.alloc((size_t)n * tb, J->stream))) return rc;
    if ((rc = J->expk.alloc((size_t)J->d * n * (sizeof(double2) + sizeof(double4)), J->stream))) return rc; // phases, axis table
    if ((rc = J->part.alloc(nparts * NDV * 2 * sizeof(double), J->stream))) return rc;
    if ((o.write_mask & ZQD_WRITE_WAVEFUNCTION) &&
        (rc = J->wfn_hist.alloc((size_t)J->nsolve * (o.iterations + 1) * S * N * c, J->stream)))
        return rc;
    if (!o.ic_wfn.empty()) { // initial wavefunction, natural order
        if ((rc = J->psi_init.alloc((size_t)S * N * c, J->stream))) return rc;
        std::vector<cx<T>> h((size_t)S * N);
        for (size_t e = 0; e < (size_t)S * N; ++e) h[e] = mk<T>((T)o.ic_wfn[2 * e], (T)o.ic_wfn[2 * e + 1]);
        ZQD_CUDA(cudaMemcpyAsync(J->psi_init.p, h.data(), (size_t)S * N * c, cudaMemcpyHostToDevice, J->stream));
        ZQD_CUDA(cudaStreamSynchronize(J->stream));
        J->h2d += (size_t)S * N * c;
    }
    if ((rc = J->book.alloc(sizeof(NdBook), J->stream))) return rc;
    if ((rc = J->flags.alloc(4 * sizeof(int), J->stream))) return rc; // stopped, never set, TMA error, spare
    const size_t rows = (size_t)o.iterations + 1;
    if ((rc = J->hist.alloc((size_t)J->nsolve * rows * J->hc * sizeof(double), J->stream))) return rc;
    if ((rc = J->fin.alloc((size_t)J->nsolve * J->hc * sizeof(double), J->stream))) return rc;
    if ((rc = J->rows.alloc((size_t)J->nsolve * sizeof(int), J->stream))) return rc;
    J->device_bytes = J->psi_save.bytes + J->phi.bytes + J->psi0.bytes + J->orth.bytes + J->R.bytes + J->V.bytes +
                      J->U.bytes + J->capw.bytes + J->part.bytes + J->hist.bytes;
    std::vector<double> tw = twiddles_f64(n);
    std::vector<Tab<T>> twt(n);
    for (int t = 0; t < n; ++t) twt[t] = mktab<T>(tw[2 * t], tw[2 * t + 1]);
    ZQD_CUDA(cudaMemcpyAsync(J->tw.p, twt.data(), (size_t)n * tb, cudaMemcpyHostToDevice, J->stream));
    ZQD_CUDA(cudaMemsetAsync(J->flags.p, 0, 4 * sizeof(int), J->stream));
    ZQD_CUDA(cudaMemsetAsync(J->hist.p, 0xff, J->hist.bytes, J->stream)); // NaN until written
    J->h2d += (size_t)n * tb + J->pot.bytes;
    NdJob<T> D = describe(J);
    nd_table_kernel<T, S><<<(unsigned)((N + 127) / 128), 128, 0, J->stream>>>(D, 0.0, 1);
    ZQD_CUDA(cudaGetLastError());
    nd_kphase_kernel<T><<<(unsigned)((J->d * n + 127) / 128), 128, 0, J->stream>>>(
        D, J->expk.as<double2>(), const_cast<double4*>(D.axis));
    ZQD_CUDA(cudaGetLastError());
    for (auto f : {nd_row_kernel<T, 2, S, 256>, nd_row_kernel<T, 3, S, 256>, nd_row_kernel<T, 2, S, 512>,
                   nd_row_kernel<T, 3, S, 512>})
        ZQD_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, budget));
    for (auto f : {nd_tile_kernel<T, 2>, nd_tile_kernel<T, 3>})
        ZQD_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, budget));
    if ((rc = setup_tma(J, ov.tma_w))) return rc;
    if (J->nd_row_tma && (rc = encode_row_tma(J))) return rc;
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    return ZQD_OK;
}

namespace {
// The launches of a run, in stream order, in three pieces per solve: the prologue (setGaussian,
// normalise, toDia), the launches of loop index i (step i, then the observables of row i) and the
// epilogue (final observables, orthw.append).  A whole run (enqueue) is every piece in order; a
// step range (ZQD_ND_STEP) is a run of consecutive loop indices.
struct Seq {
    zqd_job* J;
    Launch Lc;
    bool split, acf;
    int iters, HC;
    size_t SN;
    unsigned ng;

    explicit Seq(zqd_job* j) : J(j), Lc{j, describe(j)} {
        const Opts& o = J->o;
        const size_t N = J->N;
        Lc.nrow_blocks = N / J->n / J->nd_rows;
        Lc.ntile_blocks = N / J->n / J->nd_tile;
        Lc.ngrid = std::min<size_t>(1024, (N + 255) / 256);
        Lc.R0 = 0;
        Lc.R1 = Lc.nrow_blocks;
        Lc.R2 = 2 * Lc.nrow_blocks;
        Lc.K = 3 * Lc.nrow_blocks;
        Lc.G = Lc.K + S * Lc.ntile_blocks;
        split = o.imag_nstate > 0 || o.pot_td || (o.has_cap && o.cap_has_stop);
        acf = o.has_spectrum || (o.write_mask & ZQD_WRITE_ACF);
        iters = (int)o.iterations;
        HC = J->hc;
        SN = (size_t)S * N * sizeof(cx<T>);
        ng = (unsigned)Lc.ngrid;
        Lc.D.orth = J->orth.as<cx<T>>();
    }
    double* hist(int s) const { return J->hist.as<double>() + (size_t)s * (iters + 1) * HC; }
    int* rows_out(int s) const { return J->rows.as<int>() + s; }
    // Imaginary time, first state, no absorbing potential, no time-dependent potential and no
    // wavefunction history: the renormalisation of step i (quantum_dynamics.zig:898-906 with no
    // earlier states) is deferred.  Propagation is linear, the norm, populations, energies and
    // positions are quadratic in psi and the autocorrelation is linear, so the step closes and the
    // next one opens in a single row pass over the unnormalised psi, as in real time; its finalize
    // scales the observables row by the renormalisation factor (squared) and keeps the sum of
    // |psi|^2, and the first tile pass of step i+1 (or the final observables' pass) multiplies psi
    // by that factor as it loads it.
    bool deferred(int s) const {
        const Opts& o = J->o;
        return o.imag_nstate && s == 0 && !o.has_cap && !o.pot_td && !J->wfn_hist.p;
    }
    // this solve's wavefunction history entry of step i (write.wavefunction), or null
    cx<T>* whist(int s, int i) const {
        return J->wfn_hist.p ? J->wfn_hist.as<cx<T>>() + ((size_t)s * (iters + 1) + i) * S * J->N : nullptr;
    }
    // finalize descriptors, run by the last CTA of the launch that ends a step
    NdFin fin(int s, int kind, size_t x0, size_t x1, bool k, uint32_t mask, double* row, int i) const {
        const Opts& o = J->o;
        NdFin f{};
        f.row = row;
        f.rows_out = rows_out(s);
        f.book = J->book.as<NdBook>();
        f.x0 = x0;
        f.x1 = x1;
        f.k0 = Lc.K;
        f.k1 = k ? Lc.K + S * Lc.ntile_blocks : Lc.K;
        f.stop_norm = o.cap_stop_norm;
        f.mask = mask;
        f.row_index = i;
        f.kind = kind;
        f.has_stop = kind == 0 && o.has_cap && o.cap_has_stop;
        f.enabled = 1;
        return f;
    }
    int itp_ops(int s) { // quantum_dynamics.zig:898-906
        int rc;
        for (int j = 0; j < s; ++j) {
            nd_dot_kernel<T><<<ng, 256, 0, J->stream>>>(Lc.D, j, Lc.G);
            if ((rc = Lc.reduce(Lc.G, Lc.G + ng, 2))) return rc;
            nd_orth_apply_kernel<T><<<ng, 256, 0, J->stream>>>(Lc.D, j, Lc.scal());
        }
        nd_dot_kernel<T><<<ng, 256, 0, J->stream>>>(Lc.D, -1, Lc.G);
        if ((rc = Lc.reduce(Lc.G, Lc.G + ng, 1))) return rc;
        nd_normalize_kernel<T, S><<<ng, 256, 0, J->stream>>>(Lc.D, Lc.scal(), 0, 0);
        ZQD_CUDA(cudaGetLastError());
        return ZQD_OK;
    }
    int prologue(int s) {
        const Opts& o = J->o;
        ZQD_CUDA(cudaMemsetAsync(J->flags.p, 0, 2 * sizeof(int), J->stream));
        ZQD_CUDA(cudaMemsetAsync(J->book.p, 0, sizeof(NdBook), J->stream));
        if (s == 0 && o.pot_td) { // a later run starts again from the t = 0 tables (Hamiltonian.init, Propagator.init)
            nd_table_kernel<T, S><<<(unsigned)((J->N + 127) / 128), 128, 0, J->stream>>>(Lc.D, 0.0, 1);
            ZQD_CUDA(cudaGetLastError());
        }
        // setGaussian, normalise, toDia, acf reference (quantum_dynamics.zig:867-882)
        nd_gauss_kernel<T><<<ng, 256, 0, J->stream>>>(Lc.D, Lc.G);
        ZQD_CUDA(cudaGetLastError());
        if (int rc = Lc.reduce(Lc.G, Lc.G + ng, 1)) return rc;
        nd_normalize_kernel<T, S><<<ng, 256, 0, J->stream>>>(Lc.D, Lc.scal(), o.ic_adiabatic ? 1 : 0, acf ? 1 : 0);
        ZQD_CUDA(cudaGetLastError());
        return ZQD_OK;
    }
    int step(int s, int i) {
        const Opts& o = J->o;
        int rc;
        const bool logstep = o.log && ((i % o.log_interval == 0) || (i == iters));
        const uint32_t mask = o.write_mask | (logstep ? (uint32_t)WM_ALL_OBS : 0u) | (acf ? (uint32_t)WM_ACF : 0u);
        const bool needk = mask & (WM_MOM | WM_EKIN | WM_ETOT);
        const uint32_t obs = mask | ((o.has_cap && o.cap_has_stop) ? (uint32_t)WM_NORM : 0u);
        double* row = hist(s) + (size_t)i * HC;
        const bool defer = deferred(s);
        if (i > 0 && (rc = Lc.step_tiles(defer ? (uint32_t)TM_SCALE : 0u))) return rc;
        if (!split || defer) {
            uint32_t mode = RM_OBS | RM_STORE | (needk ? RM_PHI : 0u);
            if (i > 0) mode |= RM_INV | RM_REND;
            if (i < iters) mode |= RM_RSTART | RM_FWD;
            NdFin f = fin(s, 0, Lc.R0, Lc.R0 + Lc.nrow_blocks, needk, mask, row, i);
            if (defer) f.nsum_out = Lc.scal();
            const uint32_t o2 = obs | (defer ? (uint32_t)WM_NORM : 0u);
            if ((rc = Lc.row(mode, o2, Lc.R0, false, needk ? NdFin{} : f, whist(s, i)))) return rc;
            if (needk && (rc = Lc.kobs(false, f))) return rc;
            return ZQD_OK;
        }
        // Imaginary time, first state (nothing to orthogonalise against), no absorbing potential, after
        // step 0: the pass that closes step i also sums |psi|^2, and the next pass divides by the norm
        // as it loads psi, in place of the norm and normalisation kernels (quantum_dynamics.zig:898-906
        // with no earlier states); without a time-dependent potential that pass also records the
        // step's observables and opens step i+1.
        const bool fuse = o.imag_nstate && s == 0 && i > 0 && !o.has_cap;
        if (i > 0 && (rc = Lc.row(RM_INV | RM_REND | RM_STORE | (fuse ? (uint32_t)RM_NORM : 0u), 0, Lc.R0))) return rc;
        if (fuse) { // the norm's sum into scal[0], taken out of R0 (the observables row sums R0 too)
            if ((rc = Lc.reduce(Lc.R0, Lc.R0 + Lc.nrow_blocks, 1, true))) return rc;
        } else if (o.imag_nstate && (rc = itp_ops(s))) {
            return rc; // every i, the initial state included
        }
        if (o.pot_td && (rc = Lc.table((double)i * o.time_step, 0))) return rc;
        // R0 holds the end-of-step sums of the row pass that closed step i (none at i = 0)
        const NdFin f = fin(s, 0, i > 0 ? Lc.R0 : Lc.R1, Lc.R1 + Lc.nrow_blocks, needk, mask, row, i);
        if (fuse && !o.pot_td && i < iters) { // normalise, observe, and open step i+1 in one pass
            const uint32_t mode = RM_SCALE | RM_OBS | RM_RSTART | RM_FWD | RM_STORE | (needk ? (uint32_t)RM_PHI : 0u);
            if ((rc = Lc.row(mode, obs, Lc.R1, false, needk ? NdFin{} : f, whist(s, i)))) return rc;
            if (needk && (rc = Lc.kobs(false, f))) return rc;
            return ZQD_OK;
        }
        const uint32_t omode = RM_OBS | (needk ? (uint32_t)RM_PHI : 0u) | (fuse ? (uint32_t)(RM_SCALE | RM_STORE) : 0u);
        if ((rc = Lc.row(omode, obs, Lc.R1, false, needk ? NdFin{} : f, whist(s, i)))) return rc;
        if (needk && (rc = Lc.kobs(false, f))) return rc;
        if (i < iters) {
            if (o.pot_td && (rc = Lc.table(((double)i + 0.5) * o.time_step, 1))) return rc;
            // the absorbed sums of step i+1's first accumAbsorbed
            const NdFin fc = fin(s, 2, Lc.R2, Lc.R2 + Lc.nrow_blocks, false, 0, nullptr, 0);
            if ((rc = Lc.row(RM_RSTART | RM_FWD | RM_STORE, 0, Lc.R2, false, fc))) return rc;
        }
        return ZQD_OK;
    }
    int epilogue(int s) {
        int rc;
        // final Observables.init(..., log = true) (quantum_dynamics.zig:949)
        const uint32_t all = WM_ALL_OBS | (acf ? (uint32_t)WM_ACF : 0u);
        // a deferred renormalisation (the last step's) is applied here, and psi stored normalised
        const uint32_t scale = deferred(s) ? (uint32_t)(RM_SCALE | RM_STORE) : 0u;
        if ((rc = Lc.row(RM_OBS | RM_PHI | scale, all, Lc.R1, true))) return rc;
        if ((rc = Lc.kobs(true, fin(s, 1, Lc.R1, Lc.R1 + Lc.nrow_blocks, true, all, J->fin.as<double>() + (size_t)s * HC, 0))))
            return rc;
        if (s + 1 < J->nsolve) // orthw.append (quantum_dynamics.zig:586-591)
            ZQD_CUDA(cudaMemcpyAsync(J->orth.as<char>() + (size_t)s * SN, J->psi_save.p, SN, cudaMemcpyDeviceToDevice, J->stream));
        return ZQD_OK;
    }
};

// every launch of a run, in stream order (captured into a graph by ZQD_ND_RUN)
int enqueue(zqd_job* J) {
    Seq q(J);
    int rc;
    for (int s = 0; s < J->nsolve; ++s) {
        if ((rc = q.prologue(s))) return rc;
        for (int i = 0; i <= q.iters; ++i)
            if ((rc = q.step(s, i))) return rc;
        if ((rc = q.epilogue(s))) return rc;
    }
    return ZQD_OK;
}
} // namespace

// The TMA-staged passes record a load that never landed in flags[2] (the job's buffers are
// then suspect): report it as a device error.
static int check_tma(zqd_job* J) {
    if (!J->nd_tma && !J->nd_row_tma) return ZQD_OK;
    int e = 0;
    ZQD_CUDA(cudaMemcpyAsync(&e, J->flags.as<int>() + 2, sizeof(int), cudaMemcpyDeviceToHost, J->stream));
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    J->d2h += sizeof(int);
    return e ? fail(ZQD_ERR_DEVICE, "A TMA LOAD OF AN AXIS PASS DID NOT COMPLETE WITHIN ITS WAIT BUDGET") : ZQD_OK;
}

// Rows i0..i1 of solve s (zqd_job_step), launched directly; then, if the solve ended (its last
// step, or stop_norm), its final observables.  *rows: rows of the solve's history written so far.
int ZQD_ND_STEP(zqd_job* J, int s, int i0, int i1, int* rows, int* ended) {
    Seq q(J);
    int rc;
    ZQD_CUDA(cudaEventRecord(J->ev0, J->stream));
    if (i0 == 0 && (rc = q.prologue(s))) return rc;
    for (int i = i0; i <= i1; ++i)
        if ((rc = q.step(s, i))) return rc;
    // the steps first, then the copies into pageable memory (one queued behind the steps would wait
    // inside the driver, where it can hold up other threads' copies)
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    int flags[2] = {0, 0}; // stopped, rows
    ZQD_CUDA(cudaMemcpyAsync(&flags[0], J->flags.p, sizeof(int), cudaMemcpyDeviceToHost, J->stream));
    ZQD_CUDA(cudaMemcpyAsync(&flags[1], q.rows_out(s), sizeof(int), cudaMemcpyDeviceToHost, J->stream));
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    J->d2h += sizeof(flags);
    *rows = flags[1];
    *ended = flags[0] || i1 >= q.iters;
    if ((rc = check_tma(J))) return rc;
    if (*ended && (rc = q.epilogue(s))) return rc;
    ZQD_CUDA(cudaEventRecord(J->ev1, J->stream));
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    float ms = 0;
    ZQD_CUDA(cudaEventElapsedTime(&ms, J->ev0, J->ev1));
    J->last_ms += ms;
    return ZQD_OK;
}

// A run is a fixed sequence of launches: it is captured into a CUDA graph on the
// first call and the graph is replayed by every later call on the job.
int ZQD_ND_RUN(zqd_job* J) {
    if (!J->nd_use_graph) {
        ZQD_CUDA(cudaEventRecord(J->ev0, J->stream));
        const int rc = enqueue(J);
        if (rc) return rc;
        ZQD_CUDA(cudaEventRecord(J->ev1, J->stream));
        ZQD_CUDA(cudaStreamSynchronize(J->stream));
        ZQD_CUDA(cudaEventElapsedTime(&J->last_ms, J->ev0, J->ev1));
        return check_tma(J);
    }
    if (!J->nd_graph) {
        ZQD_CUDA(cudaStreamBeginCapture(J->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue(J);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(J->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        ZQD_CUDA(e);
        const cudaError_t ei = cudaGraphInstantiate(&J->nd_graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) J->nd_graph = nullptr;
        ZQD_CUDA(ei);
    }
    ZQD_CUDA(cudaEventRecord(J->ev0, J->stream));
    ZQD_CUDA(cudaGraphLaunch(J->nd_graph, J->stream));
    ZQD_CUDA(cudaEventRecord(J->ev1, J->stream));
    ZQD_CUDA(cudaStreamSynchronize(J->stream));
    ZQD_CUDA(cudaEventElapsedTime(&J->last_ms, J->ev0, J->ev1));
    return check_tma(J);
}

} // namespace zqd
