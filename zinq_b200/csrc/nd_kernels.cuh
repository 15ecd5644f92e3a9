// nd_kernels.cuh -- split-operator passes for 2-D and 3-D grids.
//
// The wavefunction (S x N complex, state-major, last axis fastest: the
// reference's Matrix(Complex) layout, src/wavepacket.zig:182) stays in global
// memory; a time step is a sequence of axis passes, each staging lines of one
// axis in shared memory, running the Stockham FFT passes there and writing
// them back:
//   row pass   (last axis, contiguous; all S states of a row in one CTA)
//              [inverse FFT, 1/N, accumAbsorbed, R]  ... end of step i
//              [observables of step i]
//              [accumAbsorbed, R, forward FFT]       ... start of step i+1
//   tile pass  (a strided axis; `tile` consecutive lines of one state per CTA)
//              forward FFT | forward FFT, exp(-i K dt), inverse FFT | inverse FFT
// so a 2-D step is one row pass + one tile pass, a 3-D step one row pass and
// three tile passes (Propagator.step, src/quantum_dynamics.zig:417-427).
// Observables are per-CTA compensated partial sums combined in a fixed order.
#pragma once

#include <cuda_runtime.h>

#include "cx.cuh"
#include "line_kernel.cuh"
#include "physics.cuh"
#include "tma.cuh"

namespace zqd {

constexpr int NDV = 24; // reduction slots of the N-D passes

// norm | pos[d] | epot | acf re, im | mom[d] | ekin | pop[S] | absorbed, this step [S] | absorbed, next step [S]
struct NdSlots {
    int d, S;
    __host__ __device__ constexpr int norm() const { return 0; }
    __host__ __device__ constexpr int pos() const { return 1; }
    __host__ __device__ constexpr int epot() const { return 1 + d; }
    __host__ __device__ constexpr int acf() const { return 2 + d; }
    __host__ __device__ constexpr int mom() const { return 4 + d; }
    __host__ __device__ constexpr int ekin() const { return 4 + 2 * d; }
    __host__ __device__ constexpr int pop() const { return 5 + 2 * d; }
    __host__ __device__ constexpr int abs() const { return 5 + 2 * d + S; }
    __host__ __device__ constexpr int absn() const { return 5 + 2 * d + 2 * S; }
    __host__ __device__ constexpr int count() const { return 5 + 2 * d + 3 * S; }
};

template <typename T> struct NdJob {
    int d, n, logn, S;
    size_t N;
    double lo[3], span[3], mass[3];
    double dr, dk, dkunit[3];
    double dt_re, dt_im;
    int adiabatic, track, has_cap, ic_state, ic_adia;
    double cap_lo[3], cap_hi[3], cap_exp, x0[3], p0[3], gamma[3];
    cx<T>* psi;   // [S][N]
    cx<T>* phi;   // [S][N] scratch: the forward transform of the end-of-step psi
    cx<T>* psi0;  // [S][N] autocorrelation reference
    const cx<T>* psi_init; // [S][N] initial wavefunction replacing the Gaussian, or null
    cx<T>* wfn_out;        // [S][N] this launch's entry of the wavefunction history, or null
    const cx<T>* orth; // [northo][S][N] relaxed states (imaginary time)
    Tab<T>* R;    // [NSYM][N]
    double* V;    // [S*S][N]
    double* U;    // [S*S][N]
    double* capw; // [N]
    const Tab<T>* tw; // [n] exp(-2 pi i t / n)
    const double2* kphase; // [D][n] exp(Complex(0, -k^2 / (2 m_j)) * dt) of axis j
    const double4* axis;   // [D][n] per-axis grid values: coordinate r, wavenumber k, 0.5 k^2 / m_j
    double* part;     // per-CTA partial sums, slot-major: [NDV][nparts][2]
    const double* nsum; // RM_SCALE: the reduced sum of |psi|^2 the load divides by (sqrt of dr times it)
    size_t nparts;
    int rows_per_cta; // row pass: rows of the last axis per CTA
    int tile, logtile; // tile pass: lines per CTA (a power of two) and its log2
    int* stopped;     // set by the finalize kernel when stop_norm ends the solve
    int* err;         // set when a TMA load did not land within its wait budget
    PotDev pot;
};

// row-pass modes
enum : uint32_t {
    RM_INV = 1u << 0,    // inverse FFT along the last axis, then 1/N
    RM_REND = 1u << 1,   // accumAbsorbed (if tracking) then R: end of a step
    RM_OBS = 1u << 2,    // position-space observables (after RM_REND)
    RM_PHI = 1u << 3,    // forward FFT of the end-of-step psi into phi (momentum observables)
    RM_RSTART = 1u << 4, // accumAbsorbed (if tracking) then R: start of the next step
    RM_FWD = 1u << 5,    // forward FFT along the last axis
    RM_STORE = 1u << 6,  // write psi back
    RM_NORM = 1u << 7,   // after RM_REND: sum |psi|^2 into the norm slot (imaginary time: the renormalisation's norm)
    RM_SCALE = 1u << 8,  // on load: psi /= sqrt(dr * *nsum), as the normalisation kernel does (imaginary time)
};
// tile-pass modes
enum : uint32_t {
    TM_FWD = 1u << 0,
    TM_KPHASE = 1u << 1, // after the forward FFT along axis 0: psi *= exp(-i K dt)
    TM_INV = 1u << 2,
    TM_KOBS = 1u << 3,   // after the forward FFT along axis 0: momentum observables, no store
    TM_PHI = 1u << 4,    // operate on phi instead of psi
    TM_SCALE = 1u << 5,  // on load: psi *= nd_norm_factor(*nsum, dr) (imaginary time, renormalisation deferred)
};

// The renormalisation factor of psi whose sum of |psi|^2 is `sum`: 1 / sqrt(dr * sum), formed as
// Wavefunction.normalize's division by the real sqrt(norm) is (wavepacket.zig:282-284): sq / sq^2.
__host__ __device__ inline double nd_norm_factor(double sum, double dr) {
    const double sq = sqrt(sum * dr);
    return sq / (sq * sq);
}
// psi times an FP64 factor, rounded once to the state's precision
template <typename T> __device__ __forceinline__ cx<T> nd_scaled(cx<T> v, double f) {
    return mk<T>((T)((double)v.x * f), (T)((double)v.y * f));
}

template <typename T> __host__ __device__ inline int tile_ldp(int n) { return padded_len<T>(n) | 1; }
// dynamic shared memory: nbuf line buffers of `lines` lines, then the twiddle table on a 16-byte boundary
template <typename T> __host__ __device__ inline size_t nd_tw_offset(int nbuf, int lines, int n) {
    return ((size_t)nbuf * lines * tile_ldp<T>(n) * sizeof(cx<T>) + 15) & ~(size_t)15;
}
// entries of one direction's middle-pass twiddle tables: the middle passes take the span p
// from 8 (after the first radix-8 pass) to n/8 (before a last radix-8 pass, n >= 64) or n
// (n = 16, 32), and a pass of span p and radix R holds (R - 1) p entries: p_end - 8 in all
__host__ __device__ inline int nd_mid_tw(int n) { return n < 16 ? 0 : (n >= 64 ? n / 8 : n) - 8; }
// after the buffers: W_n^t (t < n) for the register-resident last pass, then the forward
// and the inverse middle-pass tables
template <typename T> __host__ __device__ inline size_t nd_smem_bytes(int nbuf, int lines, int n) {
    return nd_tw_offset<T>(nbuf, lines, n) + (size_t)(n + 2 * nd_mid_tw(n)) * sizeof(Tab<T>);
}

template <typename T> __device__ __forceinline__ void grid_coords(const NdJob<T>& J, size_t gidx, double* r) {
    // Grid.init (wavepacket.zig:55-74): last axis fastest
    size_t t = gidx;
    for (int l = 0; l < J.d; ++l) {
        const int j = J.d - l - 1;
        r[j] = __dadd_rn(J.lo[j], __dmul_rn((double)(t % (size_t)J.n), J.span[j]) / (double)J.n);
        t /= (size_t)J.n;
    }
}
template <typename T> __device__ __forceinline__ void grid_wavenumbers(const NdJob<T>& J, size_t gidx, double* k) {
    size_t t = gidx;
    for (int l = 0; l < J.d; ++l) {
        const int j = J.d - l - 1;
        const int idx = (int)(t % (size_t)J.n);
        k[j] = __dmul_rn(idx < J.n / 2 ? (double)idx : __dsub_rn((double)idx, (double)J.n), J.dkunit[j]);
        t /= (size_t)J.n;
    }
}

// Radix-R Stockham pass over `ngroups` groups of G lines of n = 2^logn points
// (line (g, s) at index s * ngroups + g, stride ldp).  A thread handles butterfly
// i of all G lines of a group, so the G states of a grid point meet in one thread.
// twp: this pass's twiddles W_n^(r kk n/(p R)) at [(r - 1) p + kk] (contiguous for a warp).
template <typename T, int G, int R, int SIGN, bool FIRST, bool LAST, typename H>
__device__ __forceinline__ void tpass(const cx<T>* __restrict__ in, cx<T>* __restrict__ out, int ldp, int logn, int p,
                                      const Tab<T>* __restrict__ twp, int ngroups, H& h) {
    constexpr int LR = R == 2 ? 1 : R == 4 ? 2 : 3;
    const int logmr = logn - LR, mr = 1 << logmr;
    const int items = ngroups << logmr;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int g = it >> logmr, i = it & (mr - 1);
        cx<T> v[G][R];
#pragma unroll
        for (int s = 0; s < G; ++s)
#pragma unroll
            for (int r = 0; r < R; ++r) v[s][r] = in[(s * ngroups + g) * ldp + padx<T>(i + r * mr)];
        if constexpr (FIRST) h.template first<R>(g, i, mr, v);
        const int kk = i & (p - 1);
        if (p > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const Tab<T> w = twp[(r - 1) * p + kk];
#pragma unroll
                for (int s = 0; s < G; ++s) v[s][r] = tmul<SIGN>(v[s][r], w);
            }
        }
#pragma unroll
        for (int s = 0; s < G; ++s) dft<R, SIGN, T>(v[s]);
        const int o0 = ((i - kk) << LR) + kk;
        if constexpr (LAST) h.template last<R>(g, o0, p, v);
#pragma unroll
        for (int s = 0; s < G; ++s)
#pragma unroll
            for (int r = 0; r < R; ++r) out[(s * ngroups + g) * ldp + padx<T>(o0 + r * p)] = v[s][r];
    }
    __syncthreads();
}

struct NdNoHook {
    template <int R, typename V> __device__ __forceinline__ void first(int, int, int, V&) {}
    template <int R, typename V> __device__ __forceinline__ void last(int, int, int, V&) {}
};

// slot indices of the reductions for a (D, S) pair, compile-time (same order as NdSlots)
template <int D, int S> struct Slots {
    static constexpr int norm = 0, pos = 1, epot = 1 + D, acf = 2 + D, mom = 4 + D, ekin = 4 + 2 * D, pop = 5 + 2 * D,
                         abs = 5 + 2 * D + S, absn = 5 + 2 * D + 2 * S, count = 5 + 2 * D + 3 * S;
};

// per-CTA reduction of NV compensated sums into slots [first, first + NV) of the
// slot-major partial array part[NDV][P][2], at column `block` (fixed order).  Only
// the values whose bit is set in `active` (uniform over the CTA) are reduced; the
// others are stored as zero without any work.
template <int NV>
__device__ __forceinline__ void block_partials(const double (&a)[NV], int first, double* __restrict__ part, size_t P,
                                               size_t block, uint32_t active = ~0u) {
    __shared__ double red[16][NV][2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        if (!((active >> v) & 1u)) continue;
        double s = a[v], c = 0.0; // a thread's plain sum over its few points, then compensated combination
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double s2 = __shfl_down_sync(0xffffffffu, s, off), c2 = __shfl_down_sync(0xffffffffu, c, off);
            Acc t;
            t.s = s;
            t.c = c;
            t.add(s2);
            t.c += c2;
            s = t.s;
            c = t.c;
        }
        if (lane == 0) {
            red[warp][v][0] = s;
            red[warp][v][1] = c;
        }
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        Acc t;
        if ((active >> threadIdx.x) & 1u)
            for (int w = 0; w < nw; ++w) {
                t.add(red[w][threadIdx.x][0]);
                t.c += red[w][threadIdx.x][1];
            }
        const size_t o = ((size_t)(first + threadIdx.x) * P + block) * 2;
        part[o] = t.s;
        part[o + 1] = t.c;
    }
    __syncthreads();
}

// Sum of slot v over partial blocks [b0, b1), computed by one whole warp: lane l
// takes blocks b0 + l, b0 + l + 32, ... in order, then a fixed butterfly; the
// result (identical in every lane) does not depend on timing.
__device__ __forceinline__ double warp_sum_partials(const double* __restrict__ part, size_t P, size_t b0, size_t b1,
                                                    int v) {
    const int lane = threadIdx.x & 31;
    const double2* __restrict__ src = reinterpret_cast<const double2*>(part) + (size_t)v * P;
    Acc t;
    size_t b = b0 + lane;
    for (; b + 96 < b1; b += 128) { // four independent loads in flight
        const double2 x0 = src[b], x1 = src[b + 32], x2 = src[b + 64], x3 = src[b + 96];
        t.add(x0.x);
        t.c += x0.y;
        t.add(x1.x);
        t.c += x1.y;
        t.add(x2.x);
        t.c += x2.y;
        t.add(x3.x);
        t.c += x3.y;
    }
    for (; b < b1; b += 32) {
        const double2 x = src[b];
        t.add(x.x);
        t.c += x.y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double s2 = __shfl_xor_sync(0xffffffffu, t.s, off), c2 = __shfl_xor_sync(0xffffffffu, t.c, off);
        // combine in lane order so both partners compute the same value
        Acc u;
        if (lane & off) {
            u.s = s2;
            u.c = c2;
            u.add(t.s);
            u.c += t.c;
        } else {
            u.s = t.s;
            u.c = t.c;
            u.add(s2);
            u.c += c2;
        }
        t = u;
    }
    return t.value();
}

// scalars for the imaginary-time kernels: out[v] = sum of slot v over [b0, b1), v < nv (one warp per slot)
// clear: the summed columns are zeroed afterwards (a sum taken out of a region the step's
// observables row also sums)
static __global__ void nd_reduce_kernel(double* __restrict__ part, size_t P, size_t b0, size_t b1, int nv,
                                        const int* stopped, double* __restrict__ out, int clear) {
    if (*stopped) return;
    const int w = threadIdx.x >> 5;
    if (w >= nv) return;
    const double v = warp_sum_partials(part, P, b0, b1, w);
    if ((threadIdx.x & 31) == 0) out[w] = v;
    if (clear) {
        __syncwarp();
        for (size_t b = b0 + (threadIdx.x & 31); b < b1; b += 32) {
            part[((size_t)w * P + b) * 2] = 0.0;
            part[((size_t)w * P + b) * 2 + 1] = 0.0;
        }
    }
}

// Per-solve bookkeeping on the device.
struct NdBook {
    double pop_abs[4];
    double carry[4];  // absorbed sums of the next step's first accumAbsorbed
    double scal[4];   // reduced sums for the imaginary-time kernels and the eigenvector alignment
    unsigned counter; // CTAs of the current launch that have written their partials
};

// What the last CTA of a row or tile launch does with the partial sums (enabled != 0):
// kind 0: the observables row of step row_index (plus absorbed bookkeeping and stop_norm);
// kind 1: the final observables (no bookkeeping); kind 2: only record the absorbed sums
// of the next step's first accumAbsorbed.  [x0, x1): position-space and absorbed partial
// blocks, [k0, k1): momentum-space blocks.
struct NdFin {
    double* row;
    int* rows_out;
    NdBook* book;
    // kind 0, renormalisation deferred (imaginary time): the launch summed the unnormalised psi.
    // The row is scaled as if psi had been normalised first (every sum by the factor squared, the
    // autocorrelation by the factor), and the raw sum of |psi|^2 goes to *nsum_out, where the next
    // step's first pass (TM_SCALE) or the final observables' pass (RM_SCALE) takes it from.
    double* nsum_out;
    size_t x0, x1, k0, k1;
    double stop_norm;
    uint32_t mask;
    int row_index, kind, has_stop, enabled;
};

// true in the CTA that finishes last (its partials and everyone else's are visible to it)
__device__ __forceinline__ bool nd_last_cta(unsigned* counter, unsigned total) {
    __shared__ bool last;
    if (threadIdx.x < 32) __threadfence(); // the partial sums were written by the first warp
    __syncthreads();
    if (threadIdx.x == 0) {
        last = atomicAdd(counter, 1u) == total - 1;
        if (last) *counter = 0; // every CTA of this launch has counted; ready for the next one
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// Sums the launch's partials in a fixed order and assembles the observables row
// (Observables.init, quantum_dynamics.zig:300-360; accumAbsorbed bookkeeping :470-500;
// stop_norm :933-944).  Run by every thread of one CTA.
template <typename T> __device__ void nd_finalize_cta(const NdJob<T>& J, const NdFin& F) {
    __shared__ double out[NDV];
    const NdSlots sl{J.d, J.S};
    const int nw = blockDim.x >> 5;
    const uint32_t mask = F.mask;
    const bool c_pos = mask & WM_POS, c_mom = mask & WM_MOM, c_pop = mask & WM_POP;
    const bool c_ekin = (mask & WM_EKIN) || (mask & WM_ETOT), c_epot = (mask & WM_EPOT) || (mask & WM_ETOT);
    const bool c_norm = (mask & WM_NORM) || F.has_stop, c_acf = mask & WM_ACF;
    // only the slots this finalize uses are summed (the others are zero or unrecorded): the norm, the
    // recorded observables and, with CAP tracking, the absorbed sums; the rest read as 0
    int list[NDV], nl = 0;
    for (int v = 0; v < sl.count(); ++v) {
        const bool need = v == sl.norm() || (c_pos && v >= sl.pos() && v < sl.pos() + J.d) ||
                          (c_epot && v == sl.epot()) || (c_acf && (v == sl.acf() || v == sl.acf() + 1)) ||
                          (c_mom && v >= sl.mom() && v < sl.mom() + J.d) || (c_ekin && v == sl.ekin()) ||
                          (c_pop && v >= sl.pop() && v < sl.pop() + J.S) || (J.track && v >= sl.abs());
        if (need) list[nl++] = v;
        else if (threadIdx.x == 0) out[v] = 0.0;
    }
    for (int k = threadIdx.x >> 5; k < nl; k += nw) {
        const int v = list[k];
        const bool kslot = v >= sl.mom() && v <= sl.ekin();
        const double x = kslot ? (F.k1 > F.k0 ? warp_sum_partials(J.part, J.nparts, F.k0, F.k1, v) : 0.0)
                               : warp_sum_partials(J.part, J.nparts, F.x0, F.x1, v);
        if ((threadIdx.x & 31) == 0) out[v] = x;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    if (F.nsum_out) {
        const double f = nd_norm_factor(out[sl.norm()], J.dr);
        *F.nsum_out = out[sl.norm()];
        for (int v = 0; v < sl.count(); ++v)
            out[v] *= (v == sl.acf() || v == sl.acf() + 1) ? f : f * f;
    }
    NdBook* book = F.book;
    if (F.kind == 2) {
        for (int s = 0; s < J.S; ++s) book->carry[s] = out[sl.absn() + s];
        return;
    }
    double* row = F.row;
    const RowLayout L{J.d, J.S};
    if (F.kind == 0)
        for (int s = 0; s < J.S; ++s) { // accumAbsorbed adds sum * dr twice per step (quantum_dynamics.zig:497)
            book->pop_abs[s] += book->carry[s] * J.dr;
            book->pop_abs[s] += out[sl.abs() + s] * J.dr;
            book->carry[s] = out[sl.absn() + s];
        }
    const double norm = out[sl.norm()] * J.dr;
    row[L.norm()] = c_norm ? norm : nan("");
    for (int k = 0; k < J.d; ++k) {
        row[L.pos() + k] = c_pos ? out[sl.pos() + k] * J.dr : nan("");
        row[L.mom() + k] = c_mom ? out[sl.mom() + k] * J.dk : nan("");
    }
    for (int s = 0; s < J.S; ++s) row[L.pop() + s] = c_pop ? out[sl.pop() + s] * J.dr + book->pop_abs[s] : nan("");
    row[L.epot()] = c_epot ? out[sl.epot()] * J.dr : nan("");
    row[L.ekin()] = c_ekin ? out[sl.ekin()] * J.dk : nan("");
    row[L.acf()] = c_acf ? out[sl.acf()] * J.dr : nan("");
    row[L.acf() + 1] = c_acf ? out[sl.acf() + 1] * J.dr : nan("");
    if (F.kind == 0) {
        *F.rows_out = F.row_index + 1;
        if (F.has_stop && norm < F.stop_norm) *J.stopped = 1;
    }
}

// index of grid point g along axis j (last axis fastest; n = 2^logn)
template <int D> __device__ __forceinline__ int axis_index(size_t g, int j, int logn) {
    return (int)(g >> (logn * (D - 1 - j))) & ((1 << logn) - 1);
}

// ------------------------------------------------------------ register-resident transforms
// Every Stockham pass reads elements i + r n/R of a line and writes elements o0 + r p.  In
// the first pass (p = 1) and in a last radix-8 pass (p = n/8) both sets are i + r n/8: a
// thread's first-pass inputs and last-pass outputs are the same eight elements of its line.
// So the first pass runs on registers loaded straight from global memory, the last pass
// leaves its outputs in registers (stored straight to global memory, or handed to the next
// transform, whose first pass reads the same elements), and only the passes between them
// go through shared memory.  Schedule: radix 8 first, radix 8/4/2 passes between, radix 8
// last when n >= 64; for n = 16, 32 the last pass runs in shared memory and the thread
// gathers its eight elements afterwards.  The inverse visits the middle passes in reverse.
constexpr int ND_IPT = 1; // items (8-point groups) a thread holds; a CTA has one thread per item

// radix schedule: first pass radix 8; `nmid` passes between (radix 8, the last of them
// radix 2^rem in forward order, the first in inverse order); a last radix-8 pass if last8
struct NdSched {
    int nmid, rem;
    bool last8;
    __device__ __forceinline__ int lr(int j, bool inverse) const { // log2 radix of middle pass j
        const int jj = inverse ? nmid - 1 - j : j;
        return jj < nmid - 1 ? 3 : rem;
    }
};
__device__ __forceinline__ NdSched nd_sched(int logn) {
    NdSched s;
    s.last8 = logn >= 6;
    const int mid = logn - 3 - (s.last8 ? 3 : 0);
    s.nmid = (mid + 2) / 3;
    s.rem = mid - 3 * (s.nmid - 1);
    return s;
}

// Stages the middle-pass twiddles of both directions at dst (after W_n, t < n): the pass of
// span p and radix R in that direction's order holds W_n^(r kk n/(p R)) at [(r - 1) p + kk],
// r = 1..R-1, kk < p, so the pass reads them contiguously (reading W_n at stride n/(p R)
// put up to 8 of a warp's twiddles in the same banks).
template <typename T>
__device__ __forceinline__ void nd_stage_mid_tw(const Tab<T>* __restrict__ tw, Tab<T>* dst, int logn) {
    const NdSched sc = nd_sched(logn);
    const int n = 1 << logn;
    for (int dir = 0; dir < 2; ++dir) {
        Tab<T>* d = dst + dir * nd_mid_tw(n);
        int logp = 3, base = 0;
        for (int j = 0; j < sc.nmid; ++j) {
            const int lr = sc.lr(j, dir == 1 && sc.last8), R = 1 << lr, p = 1 << logp, tshift = logn - logp - lr;
            for (int e = threadIdx.x; e < (R - 1) * p; e += blockDim.x) {
                const int r = e / p + 1, kk = e - (r - 1) * p;
                d[base + e] = tw[(r * kk) << tshift];
            }
            base += (R - 1) * p;
            logp += lr;
        }
    }
}

// item it of the CTA -> (line g, 8-point group i); GFAST: consecutive items walk the lines
template <bool GFAST> __device__ __forceinline__ void nd_item(int it, int logl, int logm, int& g, int& i) {
    if (GFAST) {
        g = it & ((1 << logl) - 1);
        i = it >> logl;
    } else {
        i = it & ((1 << logm) - 1);
        g = it >> logm;
    }
}

// One n-point transform (SIGN -1 forward, +1 inverse, unnormalised) of `lines` lines.
// In: v[k][r] = element i + r n/8 of line g for the thread's items k (it = tid + k blockDim).
// Out: the same elements of the transformed lines.  a, b: shared line buffers (stride ldp).
template <typename T, int SIGN, bool GFAST>
__device__ __forceinline__ void nd_fft_regs(cx<T> (&v)[ND_IPT][8], cx<T>* a, cx<T>* b, int ldp, int logn, int logl,
                                            const Tab<T>* __restrict__ twm, int lines) {
    const NdSched sc = nd_sched(logn);
    const int logm = logn - 3, items = lines << logm;
    if (logn == 3) { // n = 8: the first pass is the last
#pragma unroll
        for (int k = 0; k < ND_IPT; ++k)
            if (threadIdx.x + k * blockDim.x < items) dft<8, SIGN, T>(v[k]);
        return;
    }
#pragma unroll
    for (int k = 0; k < ND_IPT; ++k) { // first pass, p = 1: outputs at 8 i + r
        const int it = threadIdx.x + k * blockDim.x;
        if (it < items) {
            int g, i;
            nd_item<GFAST>(it, logl, logm, g, i);
            dft<8, SIGN, T>(v[k]);
#pragma unroll
            for (int r = 0; r < 8; ++r) a[g * ldp + padx<T>((i << 3) + r)] = v[k][r];
        }
    }
    __syncthreads();
    cx<T>* in = a;
    cx<T>* out = b;
    int logp = 3, tbase = 0;
    NdNoHook none;
    // this direction's dense middle-pass tables (staged by nd_stage_mid_tw after W_n)
    const Tab<T>* twd = twm + (1 << logn) + (SIGN > 0 ? nd_mid_tw(1 << logn) : 0);
    for (int j = 0; j < sc.nmid; ++j) {
        const int lr = sc.lr(j, SIGN > 0 && sc.last8), p = 1 << logp;
        if (lr == 3) tpass<T, 1, 8, SIGN, false, false>(in, out, ldp, logn, p, twd + tbase, lines, none);
        else if (lr == 2) tpass<T, 1, 4, SIGN, false, false>(in, out, ldp, logn, p, twd + tbase, lines, none);
        else tpass<T, 1, 2, SIGN, false, false>(in, out, ldp, logn, p, twd + tbase, lines, none);
        cx<T>* t = in;
        in = out;
        out = t;
        tbase += ((1 << lr) - 1) * p;
        logp += lr;
    }
#pragma unroll
    for (int k = 0; k < ND_IPT; ++k) { // last radix-8 pass (p = n/8, twiddle index r i), or the gather
        const int it = threadIdx.x + k * blockDim.x;
        if (it < items) {
            int g, i;
            nd_item<GFAST>(it, logl, logm, g, i);
#pragma unroll
            for (int r = 0; r < 8; ++r) v[k][r] = in[g * ldp + padx<T>(i + (r << logm))];
            if (sc.last8) {
#pragma unroll
                for (int r = 1; r < 8; ++r) v[k][r] = tmul<SIGN>(v[k][r], twm[r * i]);
                dft<8, SIGN, T>(v[k]);
            }
        }
    }
    __syncthreads(); // a and b are free again
}

// ------------------------------------------------------------ row pass
// the CTA's R entries of one point (complex symmetric, upper triangle stored)
template <typename T, int S> struct RPoint {
    Tab<T> r[S * (S + 1) / 2];
    __device__ __forceinline__ void load(const NdJob<T>& J, size_t g) {
#pragma unroll
        for (int c = 0; c < S * (S + 1) / 2; ++c) r[c] = J.R[(size_t)c * J.N + g];
    }
    // psi <- R psi (Propagator.applyR, quantum_dynamics.zig:501-520)
    __device__ __forceinline__ void apply(cx<T> (&x)[S]) const {
        cx<T> y[S];
#pragma unroll
        for (int i = 0; i < S; ++i) {
            cx<T> a = mk<T>(0, 0);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int p = i < k ? i : k, q = i < k ? k : i;
                a = add<T>(a, tmul<-1>(x[k], r[p * S - p * (p - 1) / 2 + (q - p)]));
            }
            y[i] = a;
        }
#pragma unroll
        for (int i = 0; i < S; ++i) x[i] = y[i];
    }
};

// What the per-point stages of a row sweep read from global memory besides psi.  EAGER:
// loaded for a batch of points before any of them is processed, so that the loads of the
// batch are in flight together; otherwise each value is read where it is used (fewer live
// registers, for several states).  R is loaded up front either way.
template <typename T, int S, bool EAGER> struct NdAux {
    static constexpr int NU = EAGER && S > 1 ? S * S : 1, NV = EAGER ? S * (S + 1) / 2 : 1, NZ = EAGER ? S : 1;
    RPoint<T, S> R;
    double w_;     // CAP weight 1 - decay^2 (accumAbsorbed)
    double U_[NU]; // adiabatic eigenvectors, U_[k * S + i] = U_ki
    double V_[NV]; // diabatic potential: row i from the diagonal on
    cx<T> z_[NZ];  // autocorrelation reference
    __device__ __forceinline__ double w(const NdJob<T>& J, size_t g) const {
        if constexpr (EAGER) return w_;
        else return J.capw[g];
    }
    __device__ __forceinline__ double u(const NdJob<T>& J, size_t g, int k, int i) const {
        if constexpr (EAGER) return U_[NU > 1 ? k * S + i : 0];
        else return J.U[(size_t)(k * S + i) * J.N + g];
    }
    // V_ik (i <= k), entry c of the row-by-row upper triangle
    __device__ __forceinline__ double v(const NdJob<T>& J, size_t g, int c, int i, int k) const {
        if constexpr (EAGER) return V_[NV > 1 ? c : 0];
        else return J.V[(size_t)(i * S + k) * J.N + g];
    }
    __device__ __forceinline__ cx<T> z(const NdJob<T>& J, size_t g, int s) const {
        if constexpr (EAGER) return z_[NZ > 1 ? s : 0];
        else return J.psi0[(size_t)s * J.N + g];
    }
};
// which parts of NdAux a sweep needs
struct NdNeed {
    bool R, w, U, V, z0;
};

template <typename T, int S, bool EAGER>
__device__ __forceinline__ void nd_aux_load(const NdJob<T>& J, size_t g, const NdNeed& nd, NdAux<T, S, EAGER>& a) {
    if (nd.R) a.R.load(J, g);
    if constexpr (EAGER) {
        if (nd.w) a.w_ = J.capw[g];
        if constexpr (S > 1)
            if (nd.U)
#pragma unroll
                for (int e = 0; e < S * S; ++e) a.U_[e] = J.U[(size_t)e * J.N + g];
        if (nd.V) {
            int c = 0;
#pragma unroll
            for (int i = 0; i < S; ++i)
#pragma unroll
                for (int k = i; k < S; ++k) a.V_[c++] = J.V[(size_t)(i * S + k) * J.N + g];
        }
        if (nd.z0)
#pragma unroll
            for (int s = 0; s < S; ++s) a.z_[s] = J.psi0[(size_t)s * J.N + g];
    }
}

// accumAbsorbed at one grid point into slots [SLOT, SLOT + S) (quantum_dynamics.zig:470-500)
template <typename T, int S, int SLOT, int NV, typename A>
__device__ __forceinline__ void nd_absorbed(const NdJob<T>& J, const cx<T> (&x)[S], size_t g, const A& a,
                                            double (&acc)[NV]) {
    const double w = a.w(J, g);
#pragma unroll
    for (int i = 0; i < S; ++i) {
        double are = 0, aim = 0;
        if (J.adiabatic && S > 1) {
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const double u = a.u(J, g, k, i);
                are += (double)x[k].x * u;
                aim += (double)x[k].y * u;
            }
        } else {
            are = (double)x[i].x;
            aim = (double)x[i].y;
        }
        acc[SLOT + i] += w * (are * are + aim * aim);
    }
}

// position-space observables at one point (Observables.init, quantum_dynamics.zig:300-360;
// Wavefunction.norm/pos/pop/epot, wavepacket.zig:206-300)
template <typename T, int D, int S, int NV, typename A>
__device__ __forceinline__ void nd_observe(const NdJob<T>& J, const cx<T> (&x)[S], size_t g, uint32_t obs, const A& a,
                                           double (&acc)[NV]) {
    using SL = Slots<D, S>;
    double m2 = 0;
    const bool adia = J.adiabatic && S > 1;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const double w = (double)x[s].x * (double)x[s].x + (double)x[s].y * (double)x[s].y;
        m2 += w;
        if ((obs & WM_POP) && !adia) acc[SL::pop + s] += w;
    }
    acc[SL::norm] += m2;
    if (obs & WM_POS) {
#pragma unroll
        for (int j = 0; j < D; ++j) // Grid.init coordinate (wavepacket.zig:55-74), tabulated per axis
            acc[SL::pos + j] += m2 * __ldg(&J.axis[j * J.n + axis_index<D>(g, j, J.logn)].x);
    }
    if (obs & (WM_EPOT | WM_ETOT)) { // V is symmetric: diagonal plus twice the upper triangle
        double e = 0;
        int c = 0;
#pragma unroll
        for (int i = 0; i < S; ++i) {
            e += ((double)x[i].x * (double)x[i].x + (double)x[i].y * (double)x[i].y) * a.v(J, g, c++, i, i);
#pragma unroll
            for (int k = i + 1; k < S; ++k)
                e += 2.0 * ((double)x[i].x * (double)x[k].x + (double)x[i].y * (double)x[k].y) * a.v(J, g, c++, i, k);
        }
        acc[SL::epot] += e;
    }
    if (obs & WM_ACF) {
        double re = 0, im = 0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const cx<T> z0 = a.z(J, g, s);
            re += (double)z0.x * (double)x[s].x + (double)z0.y * (double)x[s].y;
            im += (double)z0.x * (double)x[s].y - (double)z0.y * (double)x[s].x;
        }
        acc[SL::acf] += re;
        acc[SL::acf + 1] += im;
    }
    if ((obs & WM_POP) && adia) {
#pragma unroll
        for (int i = 0; i < S; ++i) {
            double are = 0, aim = 0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const double u = a.u(J, g, k, i);
                are += (double)x[k].x * u;
                aim += (double)x[k].y * u;
            }
            acc[SL::pop + i] += are * are + aim * aim;
        }
    }
}

// One sweep over the CTA's points (all S states of a point in one thread):
// end of step i     1/N (after the inverse transform), accumAbsorbed + R, observables;
//                   the values are copied to `phi_src` when given (momentum observables)
// start of step i+1 accumAbsorbed + R
// R is loaded once per point for both applications.  With one state a thread takes its
// points in batches of four and loads the global inputs of the whole batch first (its
// loads would otherwise wait one after the other); several states keep one point at a
// time within the registers.  Returns after a barrier.
// bx(line, x): where point x of line s L + l sits in buf (and phi_src).  OBSMAX: the observables
// this instantiation can record (a compile-time bound on obs, so that a narrower form keeps fewer
// accumulators and loads in registers).
template <typename T, int D, int S, int NV, typename BX, uint32_t OBSMAX = ~0u>
__device__ __forceinline__ void nd_row_sweep(const NdJob<T>& J, cx<T>* buf, cx<T>* phi_src, const BX& bx, int L, size_t row0,
                                             uint32_t mode, uint32_t obs_in, double (&acc)[NV], bool wfn = true) {
    using SL = Slots<D, S>;
    const uint32_t obs = obs_in & OBSMAX;
    constexpr int SB = S == 1 ? 4 : 1;
    using Aux = NdAux<T, S, (SB > 1)>;
    const int logn = J.logn, pts = L << logn, nt = blockDim.x;
    const T inv_n = (T)(1.0 / (double)J.N);
    // RM_SCALE: the normalisation kernel's factors sqrt(dr * sum) and its square
    const double nsq = (mode & RM_SCALE) ? sqrt(*J.nsum * J.dr) : 1.0, nden = nsq * nsq;
    const bool obsv = mode & RM_OBS, adia = J.adiabatic && S > 1;
    NdNeed nd;
    nd.R = mode & (RM_REND | RM_RSTART);
    nd.w = J.track && nd.R;
    const bool wout = wfn && J.wfn_out;
    nd.U = adia && (nd.w || (obsv && (obs & WM_POP)) || wout);
    nd.V = obsv && (obs & (WM_EPOT | WM_ETOT));
    nd.z0 = obsv && (obs & WM_ACF);
    for (int it0 = threadIdx.x; it0 < pts; it0 += SB * nt) {
        Aux a[SB];
#pragma unroll
        for (int b = 0; b < SB; ++b)
            if (it0 + b * nt < pts) nd_aux_load<T, S>(J, row0 + it0 + b * nt, nd, a[b]);
#pragma unroll
        for (int b = 0; b < SB; ++b) {
            const int it = it0 + b * nt;
            if (it >= pts) break;
            const int l = it >> logn, x = it & ((1 << logn) - 1);
            const size_t g = row0 + it;
            cx<T> v[S];
#pragma unroll
            for (int s = 0; s < S; ++s) v[s] = buf[bx(s * L + l, x)];
            if (mode & RM_INV)
#pragma unroll
                for (int s = 0; s < S; ++s) v[s] = scale<T>(v[s], inv_n);
            if (mode & RM_SCALE) // normalize (wavepacket.zig:282-284) with the norm of the previous pass
#pragma unroll
                for (int s = 0; s < S; ++s)
                    v[s] = mk<T>((T)((double)v[s].x * nsq / nden), (T)((double)v[s].y * nsq / nden));
            if (mode & RM_REND) {
                if (J.track) nd_absorbed<T, S, SL::abs>(J, v, g, a[b], acc);
                a[b].R.apply(v);
                if (mode & RM_NORM)
#pragma unroll
                    for (int s = 0; s < S; ++s)
                        acc[SL::norm] += (double)v[s].x * (double)v[s].x + (double)v[s].y * (double)v[s].y;
            }
            if (obsv) nd_observe<T, D, S>(J, v, g, obs, a[b], acc);
            if (wout) { // History.append of the wavefunction (quantum_dynamics.zig:176-180), toAdia first (:919-927)
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    cx<T> y = v[i];
                    if (adia) {
                        double re = 0, im = 0;
#pragma unroll
                        for (int k = 0; k < S; ++k) {
                            const double u = a[b].u(J, g, k, i);
                            re += (double)v[k].x * u;
                            im += (double)v[k].y * u;
                        }
                        y = mk<T>((T)re, (T)im);
                    }
                    J.wfn_out[(size_t)i * J.N + g] = y;
                }
            }
            if (phi_src)
#pragma unroll
                for (int s = 0; s < S; ++s) phi_src[bx(s * L + l, x)] = v[s];
            if (mode & RM_RSTART) {
                if (J.track) nd_absorbed<T, S, SL::absn>(J, v, g, a[b], acc);
                a[b].R.apply(v);
            }
#pragma unroll
            for (int s = 0; s < S; ++s) buf[bx(s * L + l, x)] = v[s];
        }
    }
    __syncthreads();
}

// L rows of the last axis (all S states) per CTA:
// global -> [inverse FFT] -> shared -> sweep -> [phi] -> [forward FFT] -> global
// MAXT bounds the CTA size: the 256-thread form gives several states' sweep (R, the
// observables, their sums) room in registers instead of spilling at 128.
template <typename T, int D, int S, int MAXT>
__global__ void __launch_bounds__(MAXT)
    nd_row_kernel(const __grid_constant__ NdJob<T> J, uint32_t mode, uint32_t obs, size_t part_base,
                  const __grid_constant__ NdFin F) {
    if (*J.stopped) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using SL = Slots<D, S>;
    const int n = J.n, logn = J.logn, L = J.rows_per_cta, logm = logn - 3;
    const int ldp = tile_ldp<T>(n), lines = S * L, pts = L << logn, items = lines << logm;
    cx<T>* buf0 = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* buf1 = buf0 + lines * ldp;
    Tab<T>* twm = reinterpret_cast<Tab<T>*>(smem_raw + nd_tw_offset<T>(2, lines, n));
    for (int t = threadIdx.x; t < n; t += blockDim.x) twm[t] = J.tw[t];
    nd_stage_mid_tw<T>(J.tw, twm + n, logn);
    const size_t row0 = (size_t)blockIdx.x * pts;
    // line g = s * L + l starts at psi[s * N + row0 + l * n]
    auto gaddr = [&](int g) -> size_t { const int s = g / L; return (size_t)s * J.N + row0 + ((size_t)(g - s * L) << logn); };
    cx<T> v[ND_IPT][8];
#pragma unroll
    for (int k = 0; k < ND_IPT; ++k) {
        const int it = threadIdx.x + k * blockDim.x;
        if (it < items) {
            int g, i;
            nd_item<false>(it, 0, logm, g, i);
            const cx<T>* src = J.psi + gaddr(g);
#pragma unroll
            for (int r = 0; r < 8; ++r) v[k][r] = src[i + (r << logm)];
        }
    }
    __syncthreads(); // twiddles staged
    cx<T>* cur = buf0;
    cx<T>* oth = buf1;
    if (mode & RM_INV) nd_fft_regs<T, 1, false>(v, buf0, buf1, ldp, logn, 0, twm, lines);
    const bool sweep = mode & (RM_INV | RM_REND | RM_OBS | RM_RSTART | RM_PHI);
    if (sweep) { // to natural order in shared memory for the per-point stages
#pragma unroll
        for (int k = 0; k < ND_IPT; ++k) {
            const int it = threadIdx.x + k * blockDim.x;
            if (it < items) {
                int g, i;
                nd_item<false>(it, 0, logm, g, i);
#pragma unroll
                for (int r = 0; r < 8; ++r) cur[g * ldp + padx<T>(i + (r << logm))] = v[k][r];
            }
        }
        __syncthreads();
        double acc[SL::count];
#pragma unroll
        for (int q = 0; q < SL::count; ++q) acc[q] = 0.0;
        nd_row_sweep<T, D, S>(J, cur, (mode & RM_PHI) ? oth : nullptr,
                              [ldp](int line, int x) { return line * ldp + padx<T>(x); }, L, row0, mode, obs, acc);
        if (mode & (RM_OBS | RM_REND | RM_RSTART)) {
            // the slots this launch accumulates (nd_observe adds norm always, the rest by mask)
            constexpr uint32_t sm = (1u << S) - 1u;
            uint32_t act = 1u << SL::norm;
            if (mode & RM_OBS) {
                if (obs & WM_POS) act |= ((1u << D) - 1u) << SL::pos;
                if (obs & (WM_EPOT | WM_ETOT)) act |= 1u << SL::epot;
                if (obs & WM_ACF) act |= 3u << SL::acf;
                if (obs & WM_POP) act |= sm << SL::pop;
            }
            if (J.track) act |= (sm << SL::abs) | (sm << SL::absn);
            block_partials<SL::count>(acc, 0, J.part, J.nparts, part_base + blockIdx.x, act);
        }
#pragma unroll
        for (int k = 0; k < ND_IPT; ++k) { // the next step's first-pass inputs; frees cur
            const int it = threadIdx.x + k * blockDim.x;
            if (it < items) {
                int g, i;
                nd_item<false>(it, 0, logm, g, i);
#pragma unroll
                for (int r = 0; r < 8; ++r) v[k][r] = cur[g * ldp + padx<T>(i + (r << logm))];
            }
        }
        __syncthreads();
        if (mode & RM_PHI) { // forward FFT of the end-of-step copy (in oth) into phi, through oth and cur
            cx<T> w[ND_IPT][8];
#pragma unroll
            for (int k = 0; k < ND_IPT; ++k) {
                const int it = threadIdx.x + k * blockDim.x;
                if (it < items) {
                    int g, i;
                    nd_item<false>(it, 0, logm, g, i);
#pragma unroll
                    for (int r = 0; r < 8; ++r) w[k][r] = oth[g * ldp + padx<T>(i + (r << logm))];
                }
            }
            __syncthreads();
            nd_fft_regs<T, -1, false>(w, oth, cur, ldp, logn, 0, twm, lines);
#pragma unroll
            for (int k = 0; k < ND_IPT; ++k) {
                const int it = threadIdx.x + k * blockDim.x;
                if (it < items) {
                    int g, i;
                    nd_item<false>(it, 0, logm, g, i);
                    cx<T>* dst = J.phi + gaddr(g);
#pragma unroll
                    for (int r = 0; r < 8; ++r) dst[i + (r << logm)] = w[k][r];
                }
            }
        }
    }
    if (mode & RM_FWD) nd_fft_regs<T, -1, false>(v, cur, oth, ldp, logn, 0, twm, lines);
    if (mode & RM_STORE)
#pragma unroll
        for (int k = 0; k < ND_IPT; ++k) {
            const int it = threadIdx.x + k * blockDim.x;
            if (it < items) {
                int g, i;
                nd_item<false>(it, 0, logm, g, i);
                cx<T>* dst = J.psi + gaddr(g);
#pragma unroll
                for (int r = 0; r < 8; ++r) dst[i + (r << logm)] = v[k][r];
            }
        }
    if (F.enabled && nd_last_cta(&F.book->counter, gridDim.x)) nd_finalize_cta(J, F);
}

// ------------------------------------------------------------ tile pass
// one state's tile of J.tile consecutive lines along `axis` (stride n^(D-1-axis)):
// global -> forward FFT -> [kinetic phase -> inverse FFT | momentum observables] -> global,
// the elements in registers between the transforms (same elements, same threads)
template <typename T, int D>
__global__ void __launch_bounds__(512)
    nd_tile_kernel(const __grid_constant__ NdJob<T> J, int axis, uint32_t mode, size_t part_base,
                   const __grid_constant__ NdFin F) {
    if (*J.stopped) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = J.n, logn = J.logn, Tn = J.tile, logt = J.logtile, logm = logn - 3;
    const int ldp = tile_ldp<T>(n), items = Tn << logm;
    cx<T>* buf0 = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* buf1 = buf0 + Tn * ldp;
    Tab<T>* twm = reinterpret_cast<Tab<T>*>(smem_raw + nd_tw_offset<T>(2, Tn, n));
    for (int t = threadIdx.x; t < n; t += blockDim.x) twm[t] = J.tw[t];
    nd_stage_mid_tw<T>(J.tw, twm + n, logn);
    const int lstride = logn * (D - 1 - axis);
    const int ltpo = lstride - logt; // log2 of the tiles per outer index
    const size_t outer = (size_t)blockIdx.x >> ltpo, inner0 = ((size_t)blockIdx.x & ((1u << ltpo) - 1)) << logt;
    const size_t c0 = ((outer << logn) << lstride) + inner0;
    cx<T>* data = ((mode & TM_PHI) ? J.phi : J.psi) + (size_t)blockIdx.y * J.N;
    const double nf = (mode & TM_SCALE) ? nd_norm_factor(*J.nsum, J.dr) : 1.0;
    // element t of line g sits at data[c0 + (t << lstride) + g]; consecutive threads take consecutive lines
    cx<T> v[ND_IPT][8];
#pragma unroll
    for (int k = 0; k < ND_IPT; ++k) {
        const int it = threadIdx.x + k * blockDim.x;
        if (it < items) {
            int g, i;
            nd_item<true>(it, logt, logm, g, i);
#pragma unroll
            for (int r = 0; r < 8; ++r) v[k][r] = data[c0 + ((size_t)(i + (r << logm)) << lstride) + g];
            if (mode & TM_SCALE)
#pragma unroll
                for (int r = 0; r < 8; ++r) v[k][r] = nd_scaled<T>(v[k][r], nf);
        }
    }
    __syncthreads(); // twiddles staged
    if (mode & TM_FWD) nd_fft_regs<T, -1, true>(v, buf0, buf1, ldp, logn, logt, twm, Tn);
    if (mode & (TM_KPHASE | TM_KOBS)) {
        double acc[D + 1];
#pragma unroll
        for (int j = 0; j <= D; ++j) acc[j] = 0.0;
#pragma unroll
        for (int k = 0; k < ND_IPT; ++k) {
            const int it = threadIdx.x + k * blockDim.x;
            if (it < items) {
                int g, i;
                nd_item<true>(it, logt, logm, g, i);
                const size_t gbase = c0 + g; // grid index of the line's element 0
                if (mode & TM_KPHASE) {
                    // exp(Complex(0, -K) * dt), K = sum_j k_j^2 / (2 m_j) (quantum_dynamics.zig:397-399), as the
                    // product of per-axis factors (differs from the exponential of the sum by rounding only):
                    // the factor of the line's other axes once, then one product per element
                    double2 fl = make_double2(1.0, 0.0);
#pragma unroll
                    for (int j = 0; j < D; ++j)
                        if (j != axis) {
                            const double2 e = J.kphase[j * n + axis_index<D>(gbase, j, logn)];
                            fl = make_double2(__dsub_rn(__dmul_rn(fl.x, e.x), __dmul_rn(fl.y, e.y)),
                                              __dadd_rn(__dmul_rn(fl.x, e.y), __dmul_rn(fl.y, e.x)));
                        }
                    double2 f0[8];
#pragma unroll
                    for (int r = 0; r < 8; ++r) f0[r] = J.kphase[axis * n + i + (r << logm)];
#pragma unroll
                    for (int r = 0; r < 8; ++r) {
                        const double2 f = make_double2(__dsub_rn(__dmul_rn(f0[r].x, fl.x), __dmul_rn(f0[r].y, fl.y)),
                                                       __dadd_rn(__dmul_rn(f0[r].x, fl.y), __dmul_rn(f0[r].y, fl.x)));
                        v[k][r] = tmul<-1>(v[k][r], mktab<T>(f.x, f.y));
                    }
                } else { // Wavefunction.mom / ekin (wavepacket.zig:224-232, 258-268), per-axis tables
                    double Kl = 0, kl[D];
#pragma unroll
                    for (int j = 0; j < D; ++j) {
                        kl[j] = 0;
                        if (j != axis) {
                            const double4 a = J.axis[j * n + axis_index<D>(gbase, j, logn)];
                            Kl += a.z;
                            kl[j] = a.y;
                        }
                    }
                    double4 a0[8];
#pragma unroll
                    for (int r = 0; r < 8; ++r) a0[r] = J.axis[axis * n + i + (r << logm)];
#pragma unroll
                    for (int r = 0; r < 8; ++r) {
                        const double w = (double)v[k][r].x * (double)v[k][r].x + (double)v[k][r].y * (double)v[k][r].y;
#pragma unroll
                        for (int j = 0; j < D; ++j) acc[j] += w * (j == axis ? a0[r].y : kl[j]);
                        acc[D] += w * (Kl + a0[r].z);
                    }
                }
            }
        }
        if (mode & TM_KOBS) {
            block_partials<D + 1>(acc, Slots<D, 1>::mom, J.part, J.nparts,
                                  part_base + (size_t)blockIdx.y * gridDim.x + blockIdx.x);
            if (F.enabled && nd_last_cta(&F.book->counter, gridDim.x * gridDim.y)) nd_finalize_cta(J, F);
            return;
        }
    }
    if (mode & TM_INV) nd_fft_regs<T, 1, true>(v, buf0, buf1, ldp, logn, logt, twm, Tn);
#pragma unroll
    for (int k = 0; k < ND_IPT; ++k) {
        const int it = threadIdx.x + k * blockDim.x;
        if (it < items) {
            int g, i;
            nd_item<true>(it, logt, logm, g, i);
#pragma unroll
            for (int r = 0; r < 8; ++r) data[c0 + ((size_t)(i + (r << logm)) << lstride) + g] = v[k][r];
        }
    }
}

// ------------------------------------------------------------ tile pass, TMA-staged and persistent
// A tile is W consecutive lines of one state along a strided axis, held as the TMA box lands:
// element t of line g at t * W + g (rows of W * c bytes).  Each CTA loops over the tiles
// k = blockIdx.x + j * gridDim.x; while it transforms tile j in one stage buffer, the TMA load
// of tile j + 1 fills the other, and tile j leaves through a TMA store.  The radix passes run in
// place in the stage buffer (every thread reads its inputs, a barrier, then the writes), so a
// tile needs no second line buffer; the first and last radix-8 passes stay in registers.
// TM_KOBS (the momentum observables of phi after its forward transform along axis 0) stores
// nothing: its sums run over the CTA's tiles and are written once, at column blockIdx.x.
constexpr int NDT_STAGES = 2;
constexpr long long NDT_WAIT_CYCLES = 4000000000LL; // ~2 s: a TMA load that has not landed by then has failed
// (the default budget of the waits; a test of the failure path passes a short one)

struct NdTma {
    int axis;
    uint32_t mode;  // TM_FWD, TM_KPHASE, TM_INV, or TM_FWD | TM_KOBS (momentum sums, no store)
    int logW;       // lines per tile
    int logtiles;   // tiles per state
    int logO;       // outer lines (planes of the tensor map) per state
    unsigned nitems; // tiles of all states
    unsigned ncols;  // TM_KOBS: columns of the partial-sum region (written whole)
    long long wait_cycles; // budget of each mbarrier wait
    int withhold;    // testing: each CTA's first load is not issued, so its wait runs out
};

template <typename T> __host__ __device__ inline size_t ndt_stage_bytes(int W, int n) { return (size_t)W * n * sizeof(cx<T>); }
// stages, twiddles (W_n, then both directions' middle-pass tables), the stage mbarriers, and
// 128 bytes of slack to align the stages
template <typename T> __host__ __device__ inline size_t ndt_smem_bytes(int W, int n) {
    return 128 + (size_t)NDT_STAGES * ndt_stage_bytes<T>(W, n) + (size_t)(n + 2 * nd_mid_tw(n)) * sizeof(Tab<T>) +
           NDT_STAGES * sizeof(uint64_t);
}

// Where element t of line g of a stage sits, and which (line, butterfly) pair item `it` of a
// pass handles.  IxTile: the strided-axis tile, t-major as the TMA box lands (t W + g), lines
// fastest across threads.  IxRow: lines of the last axis, line-major (g n + t) under the 128-byte
// TMA swizzle (16-byte chunk j of 128-byte row q stored at chunk j ^ (q mod 8)), points fastest.
struct IxTile {
    int logW;
    __device__ __forceinline__ int at(int g, int t) const { return (t << logW) + g; }
    __device__ __forceinline__ void item(int it, int logi, int& g, int& i) const {
        g = it & ((1 << logW) - 1);
        i = it >> logW;
        (void)logi;
    }
};
template <typename T> struct IxRow {
    int logn;
    __device__ __forceinline__ int operator()(int g, int t) const { return at(g, t); }
    __device__ __forceinline__ int at(int g, int t) const {
        const int e = (g << logn) + t;
        if constexpr (sizeof(cx<T>) == 16) return e ^ ((e >> 3) & 7);
        else return e ^ (((e >> 4) & 7) << 1);
    }
    __device__ __forceinline__ void item(int it, int logi, int& g, int& i) const {
        i = it & ((1 << logi) - 1);
        g = it >> logi;
    }
};

// In-place radix-R Stockham pass over a stage's lines.  Butterfly (g, i), i < n/R, reads
// elements i + r n/R and writes o0 + r p; all reads come before the barrier, all writes after
// it.  twp: W_n^(r kk n/(p R)) at [(r - 1) p + kk].
template <typename T, int R, int SIGN, typename IX>
__device__ __forceinline__ void ndt_pass(cx<T>* buf, const IX& ix, int logn, int p, const Tab<T>* __restrict__ twp) {
    constexpr int LR = R == 2 ? 1 : R == 4 ? 2 : 3;
    constexpr int B = 8 / R; // butterflies per thread (the CTA has one thread per 8 points)
    const int logmr = logn - LR, nt = blockDim.x;
    cx<T> v[B][R];
#pragma unroll
    for (int b = 0; b < B; ++b) {
        int g, i;
        ix.item(threadIdx.x + b * nt, logmr, g, i);
#pragma unroll
        for (int r = 0; r < R; ++r) v[b][r] = buf[ix.at(g, i + (r << logmr))];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; ++b) {
        int g, i;
        ix.item(threadIdx.x + b * nt, logmr, g, i);
        const int kk = i & (p - 1);
        if (p > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[b][r] = tmul<SIGN>(v[b][r], twp[(r - 1) * p + kk]);
        }
        dft<R, SIGN, T>(v[b]);
        const int o0 = ((i - kk) << LR) + kk;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[ix.at(g, o0 + r * p)] = v[b][r];
    }
    __syncthreads();
}

// One n-point transform of a stage's lines, in place.  In: v[r] = element i + r n/8 of line g
// (the thread's item).  Out: the same elements of the transformed line.  The buffer's contents
// are free on entry (the barrier before the first write lets every thread finish reading it)
// and hold nothing of value on return.
template <typename T, int SIGN, typename IX>
__device__ __forceinline__ void ndt_fft(cx<T> (&v)[8], cx<T>* buf, const IX& ix, int logn, const Tab<T>* __restrict__ twm) {
    dft<8, SIGN, T>(v);
    if (logn == 3) return;
    const NdSched sc = nd_sched(logn);
    const int logm = logn - 3;
    int g, i;
    ix.item(threadIdx.x, logm, g, i);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; ++r) buf[ix.at(g, (i << 3) + r)] = v[r]; // first pass, p = 1: outputs at 8 i + r
    __syncthreads();
    const Tab<T>* twd = twm + (1 << logn) + (SIGN > 0 ? nd_mid_tw(1 << logn) : 0);
    int logp = 3, tbase = 0;
    for (int j = 0; j < sc.nmid; ++j) {
        const int lr = sc.lr(j, SIGN > 0 && sc.last8), p = 1 << logp;
        if (lr == 3) ndt_pass<T, 8, SIGN>(buf, ix, logn, p, twd + tbase);
        else if (lr == 2) ndt_pass<T, 4, SIGN>(buf, ix, logn, p, twd + tbase);
        else ndt_pass<T, 2, SIGN>(buf, ix, logn, p, twd + tbase);
        tbase += ((1 << lr) - 1) * p;
        logp += lr;
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = buf[ix.at(g, i + (r << logm))];
    if (sc.last8) { // last radix-8 pass, p = n/8: twiddle W_n^(r i)
#pragma unroll
        for (int r = 1; r < 8; ++r) v[r] = tmul<SIGN>(v[r], twm[r * i]);
        dft<8, SIGN, T>(v);
    }
}

// map: 3-D tensor map of this axis over psi in 8-byte words: [E * stride] words (the inner
// lines), [n] rows along the axis, [S * O] planes (outer index and state); box [E W, min(n, 256), 1]
template <typename T, int D>
__global__ void __launch_bounds__(512)
    nd_tile_tma_kernel(const __grid_constant__ NdJob<T> J, const __grid_constant__ CUtensorMap map, const NdTma P,
                       size_t part_base, const __grid_constant__ NdFin F) {
    if (*J.stopped) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    const int n = J.n, logn = J.logn, logm = logn - 3, logW = P.logW, W = 1 << logW;
    const int lstride = logn * (D - 1 - P.axis);
    constexpr int E = (int)(sizeof(cx<T>) / 8);
    const size_t sb = ndt_stage_bytes<T>(W, n);
    cx<T>* stage0 = reinterpret_cast<cx<T>*>(base);
    Tab<T>* twm = reinterpret_cast<Tab<T>*>(base + NDT_STAGES * sb);
    uint64_t* bars = reinterpret_cast<uint64_t*>(twm + n + 2 * nd_mid_tw(n));
    const int tid = threadIdx.x, g = tid & (W - 1), i = tid >> logW;
    const int rows = n < 256 ? n : 256;
    // tile k: state s = k >> logtiles, lines l0 = (k mod tiles) W of that state; box origin
    // x = E (l0 mod stride) words, plane z = s O + l0 / stride
    auto origin = [&](unsigned k, int& x, int& z, size_t& gbase) {
        const unsigned s = k >> P.logtiles;
        const size_t l0 = (size_t)(k & ((1u << P.logtiles) - 1u)) << logW;
        const size_t inner0 = l0 & (((size_t)1 << lstride) - 1), outer = l0 >> lstride;
        x = E * (int)inner0;
        z = (int)(((size_t)s << P.logO) + outer);
        gbase = ((outer << logn) << lstride) + inner0; // grid index of element 0 of the tile's line 0
    };
    auto issue = [&](unsigned k, int st) {
        int x, z;
        size_t gb;
        origin(k, x, z, gb);
        cx<T>* dst = stage0 + (size_t)st * W * n;
        mbar_arrive_expect_tx(&bars[st], (unsigned)sb);
        for (int y = 0; y < n; y += rows) tma_load_3d(dst + (size_t)y * W, &map, x, y, z, &bars[st]);
    };
    if (tid == 0) {
        prefetch_tensormap(&map);
#pragma unroll
        for (int s = 0; s < NDT_STAGES; ++s) mbar_init(&bars[s], 1);
        fence_barrier_init();
        // the first load overlaps the twiddle staging (the stages and the twiddles do not overlap)
        if (blockIdx.x < P.nitems && !P.withhold) issue(blockIdx.x, 0);
    }
    for (int t = tid; t < n; t += blockDim.x) twm[t] = J.tw[t];
    nd_stage_mid_tw<T>(J.tw, twm + n, logn);
    __syncthreads();
    const bool kobs = P.mode & TM_KOBS;
    const double nf = (P.mode & TM_SCALE) ? nd_norm_factor(*J.nsum, J.dr) : 1.0;
    double acc[D + 1]; // TM_KOBS: <k_j> sums and the kinetic energy's, over the CTA's tiles
#pragma unroll
    for (int a = 0; a <= D; ++a) acc[a] = 0.0;
    bool failed = false;
    int j = 0;
    for (unsigned k = blockIdx.x; k < P.nitems; k += gridDim.x, ++j) {
        const int st = j & 1;
        const unsigned kn = k + gridDim.x;
        if (j > 0 && kobs) __syncthreads(); // every thread is done with tile j - 1's stage (not stored)
        if (tid == 0 && kn < P.nitems) {
            bulk_wait_read_all(); // the store of tile j - 1 has read the other stage
            issue(kn, st ^ 1);
        }
        const bool ok = mbar_wait_bounded(&bars[st], (unsigned)(j >> 1) & 1u, P.wait_cycles);
        if (!__syncthreads_and(ok)) { // the load never landed: record it, let the prefetch land, stop
            if (tid == 0) {
                atomicExch(J.err, 1);
                if (kn < P.nitems) mbar_wait_bounded(&bars[st ^ 1], (unsigned)((j + 1) >> 1) & 1u, P.wait_cycles);
            }
            failed = true;
            break;
        }
        cx<T>* buf = stage0 + (size_t)st * W * n;
        int x, z;
        size_t gbase;
        origin(k, x, z, gbase);
        const IxTile ix{logW};
        cx<T> v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = buf[ix.at(g, i + (r << logm))];
        if (P.mode & TM_SCALE)
#pragma unroll
            for (int r = 0; r < 8; ++r) v[r] = nd_scaled<T>(v[r], nf);
        if (P.mode & TM_FWD) ndt_fft<T, -1>(v, buf, ix, logn, twm);
        if (P.mode & TM_KPHASE) {
            // exp(Complex(0, -K) * dt), K = sum_j k_j^2 / (2 m_j) (quantum_dynamics.zig:397-399), as the
            // product of per-axis factors: the line's other axes once, then one product per element
            const size_t gl = gbase + g;
            double2 fl = make_double2(1.0, 0.0);
#pragma unroll
            for (int a = 0; a < D; ++a)
                if (a != P.axis) {
                    const double2 e = J.kphase[a * n + axis_index<D>(gl, a, logn)];
                    fl = make_double2(__dsub_rn(__dmul_rn(fl.x, e.x), __dmul_rn(fl.y, e.y)),
                                      __dadd_rn(__dmul_rn(fl.x, e.y), __dmul_rn(fl.y, e.x)));
                }
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const double2 f0 = J.kphase[P.axis * n + i + (r << logm)];
                const double2 f = make_double2(__dsub_rn(__dmul_rn(f0.x, fl.x), __dmul_rn(f0.y, fl.y)),
                                               __dadd_rn(__dmul_rn(f0.x, fl.y), __dmul_rn(f0.y, fl.x)));
                v[r] = tmul<-1>(v[r], mktab<T>(f.x, f.y));
            }
        }
        if (kobs) { // Wavefunction.mom / ekin (wavepacket.zig:224-232, 258-268), per-axis tables
            const size_t gl = gbase + g;
            double Kl = 0, kl[D];
#pragma unroll
            for (int a = 0; a < D; ++a) {
                kl[a] = 0;
                if (a != P.axis) {
                    const double4 e = J.axis[a * n + axis_index<D>(gl, a, logn)];
                    Kl += e.z;
                    kl[a] = e.y;
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const double4 a0 = J.axis[P.axis * n + i + (r << logm)];
                const double w = (double)v[r].x * (double)v[r].x + (double)v[r].y * (double)v[r].y;
#pragma unroll
                for (int a = 0; a < D; ++a) acc[a] += w * (a == P.axis ? a0.y : kl[a]);
                acc[D] += w * (Kl + a0.z);
            }
            continue; // no store
        }
        if (P.mode & TM_INV) ndt_fft<T, 1>(v, buf, ix, logn, twm);
        __syncthreads(); // every thread's last-pass reads are done
#pragma unroll
        for (int r = 0; r < 8; ++r) buf[ix.at(g, i + (r << logm))] = v[r];
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            for (int y = 0; y < n; y += rows) tma_store_3d(&map, x, y, z, buf + (size_t)y * W);
            bulk_commit();
        }
    }
    if (tid == 0) bulk_wait_all();
    if (!kobs || failed) return;
    block_partials<D + 1>(acc, Slots<D, 1>::mom, J.part, J.nparts, part_base + blockIdx.x);
    for (size_t col = blockIdx.x + gridDim.x; col < P.ncols; col += gridDim.x) // columns no CTA owns
        for (int a = tid; a <= D; a += blockDim.x) {
            const size_t o = ((size_t)(Slots<D, 1>::mom + a) * J.nparts + part_base + col) * 2;
            J.part[o] = 0.0;
            J.part[o + 1] = 0.0;
        }
    if (F.enabled && nd_last_cta(&F.book->counter, gridDim.x)) nd_finalize_cta(J, F);
}

// ------------------------------------------------------------ row pass, TMA-staged and persistent
// An item is a block of L rows of the last axis with all S states (the row pass's unit of work);
// its stage holds line g = s L + l (g n + t, 128-byte swizzled, IxRow) as the TMA boxes land.
// Each CTA loops over the blocks k = blockIdx.x + j * gridDim.x with the next block's load in
// flight and the next block's propagator table prefetched into L2.  The observables' sums run
// over all of a CTA's blocks and are written once, at column blockIdx.x of the partial array
// (the grid's size is fixed per job and device); the columns no CTA owns are written as zero so
// that the region stays whole.  Modes: any
// combination of the row-pass modes.  RM_PHI keeps the end-of-step state in registers while the
// start of the next step is applied, and transforms it through the stage after the psi store has
// read it; it leaves through map_phi.
struct NdRowTma {
    uint32_t mode, obs;
    int logL;        // rows per block
    unsigned nitems; // blocks, and columns of the partial-sum region
    long long wait_cycles; // budget of each mbarrier wait
    int withhold;    // testing: each CTA's first load is not issued, so its wait runs out
};

template <typename T> __host__ __device__ inline size_t ndr_stage_bytes(int S, int L, int n) {
    return (size_t)S * L * n * sizeof(cx<T>);
}
// 1024 bytes of slack to align the stages (the 128-byte swizzle repeats every 1024 bytes), the
// stages, the twiddles, the stage mbarriers
template <typename T> __host__ __device__ inline size_t ndr_smem_bytes(int S, int L, int n) {
    return 1024 + (size_t)NDT_STAGES * ndr_stage_bytes<T>(S, L, n) + (size_t)(n + 2 * nd_mid_tw(n)) * sizeof(Tab<T>) +
           NDT_STAGES * sizeof(uint64_t);
}

__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(reinterpret_cast<uint64_t>(p)), "r"(bytes) : "memory");
}

// map: 3-D tensor map over psi as rows of 128 bytes: [16 words] x [S N c / 128 rows] x [1],
// box [16, min(256, L n c / 128), 1], 128-byte swizzle
// The TMA row pass's CTA size bound MAXT: 256 threads, two CTAs per SM (128 registers) for the
// plain forms, one for the form with the momentum copy (its registers hold the end-of-step state
// as well); 512 threads, one CTA per SM (128 registers), for the plain forms of one or two
// states on long lines.
constexpr int NDR_THREADS = 256, NDR_THREADS_WIDE = 512;

// POP: the form for steps that record only the populations and the norm (the other observables'
// code and accumulators compiled out), three CTAs per SM (80 registers) for one or two states.
template <typename T, int D, int S, bool PHI, int MAXT = NDR_THREADS, bool POP = false>
__global__ void __launch_bounds__(MAXT, MAXT == NDR_THREADS && !PHI ? (POP && S <= 2 ? 3 : 2) : 1)
    nd_row_tma_kernel(const __grid_constant__ NdJob<T> J, const __grid_constant__ CUtensorMap map,
                      const __grid_constant__ CUtensorMap map_phi, const NdRowTma P, size_t part_base,
                      const __grid_constant__ NdFin F) {
    if (*J.stopped) return;
    using SL = Slots<D, S>;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const int n = J.n, logn = J.logn, logm = logn - 3, L = 1 << P.logL;
    const size_t sb = ndr_stage_bytes<T>(S, L, n), blk = (size_t)L * n; // points of one state in a block
    cx<T>* stage0 = reinterpret_cast<cx<T>*>(base);
    Tab<T>* twm = reinterpret_cast<Tab<T>*>(base + NDT_STAGES * sb);
    uint64_t* bars = reinterpret_cast<uint64_t*>(twm + n + 2 * nd_mid_tw(n));
    const int tid = threadIdx.x;
    const unsigned rows_state = (unsigned)(blk * sizeof(cx<T>) / 128), rows_box = rows_state < 256 ? rows_state : 256;
    const uint32_t mode = PHI ? P.mode : (P.mode & ~(uint32_t)RM_PHI);
    const bool needR = mode & (RM_REND | RM_RSTART);
    auto issue = [&](unsigned k, int st) {
        unsigned char* dst = base + (size_t)st * sb;
        mbar_arrive_expect_tx(&bars[st], (unsigned)sb);
        for (int s = 0; s < S; ++s) {
            const size_t row = ((size_t)s * J.N + (size_t)k * blk) * sizeof(cx<T>) / 128;
            for (unsigned y = 0; y < rows_state; y += rows_box)
                tma_load_3d(dst + ((size_t)s * rows_state + y) * 128, &map, 0, (int)(row + y), 0, &bars[st]);
        }
        if (needR) // the block's propagator entries, for the sweep's loads
            for (int c = 0; c < S * (S + 1) / 2; ++c) prefetch_l2(J.R + (size_t)c * J.N + (size_t)k * blk, (unsigned)(blk * sizeof(Tab<T>)));
    };
    if (tid == 0) {
        prefetch_tensormap(&map);
#pragma unroll
        for (int s = 0; s < NDT_STAGES; ++s) mbar_init(&bars[s], 1);
        fence_barrier_init();
        // the first load overlaps the twiddle staging (the stages and the twiddles do not overlap)
        if (blockIdx.x < P.nitems && !P.withhold) issue(blockIdx.x, 0);
    }
    for (int t = tid; t < n; t += blockDim.x) twm[t] = J.tw[t];
    nd_stage_mid_tw<T>(J.tw, twm + n, logn);
    __syncthreads();
    const bool sums = mode & (RM_OBS | RM_REND | RM_RSTART);
    uint32_t act = 1u << SL::norm; // the slots this launch accumulates (nd_observe adds norm always)
    {
        constexpr uint32_t sm = (1u << S) - 1u;
        if (mode & RM_OBS) {
            if (P.obs & WM_POS) act |= ((1u << D) - 1u) << SL::pos;
            if (P.obs & (WM_EPOT | WM_ETOT)) act |= 1u << SL::epot;
            if (P.obs & WM_ACF) act |= 3u << SL::acf;
            if (P.obs & WM_POP) act |= sm << SL::pop;
        }
        if (J.track) act |= (sm << SL::abs) | (sm << SL::absn);
    }
    double acc[SL::count];
#pragma unroll
    for (int q = 0; q < SL::count; ++q) acc[q] = 0.0;
    const IxRow<T> ix{logn};
    int g, i;
    ix.item(tid, logm, g, i);
    bool failed = false;
    int j = 0;
    for (unsigned k = blockIdx.x; k < P.nitems; k += gridDim.x, ++j) {
        const int st = j & 1;
        const unsigned kn = k + gridDim.x;
        if (j > 0) __syncthreads(); // every thread is done with block j - 1's stage (a block need not be stored)
        if (tid == 0 && kn < P.nitems) {
            bulk_wait_read_all(); // the store of block j - 1 has read the other stage
            issue(kn, st ^ 1);
        }
        const bool ok = mbar_wait_bounded(&bars[st], (unsigned)(j >> 1) & 1u, P.wait_cycles);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) {
                atomicExch(J.err, 1);
                if (kn < P.nitems) mbar_wait_bounded(&bars[st ^ 1], (unsigned)((j + 1) >> 1) & 1u, P.wait_cycles);
            }
            failed = true;
            break;
        }
        cx<T>* buf = stage0 + (size_t)st * S * blk;
        const size_t row0 = (size_t)k * blk;
        cx<T> v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = buf[ix.at(g, i + (r << logm))];
        if (mode & RM_INV) ndt_fft<T, 1>(v, buf, ix, logn, twm);
        cx<T> w[8]; // RM_PHI: the end-of-step state, for its forward transform into phi
        if (mode & (RM_INV | RM_REND | RM_OBS | RM_RSTART | RM_PHI)) { // per-point stages in natural order
            __syncthreads();
#pragma unroll
            for (int r = 0; r < 8; ++r) buf[ix.at(g, i + (r << logm))] = v[r];
            __syncthreads();
            constexpr uint32_t OBSMAX = POP ? (uint32_t)(WM_POP | WM_NORM) : ~0u;
            if (PHI) { // end of step i, the copy, then the start of step i+1
                nd_row_sweep<T, D, S, SL::count, IxRow<T>, OBSMAX>(J, buf, (cx<T>*)nullptr, ix, L, row0,
                                                                   mode & ~(uint32_t)RM_RSTART, P.obs, acc);
#pragma unroll
                for (int r = 0; r < 8; ++r) w[r] = buf[ix.at(g, i + (r << logm))];
                if (mode & RM_RSTART) {
                    __syncthreads();
                    nd_row_sweep<T, D, S, SL::count, IxRow<T>, OBSMAX>(J, buf, (cx<T>*)nullptr, ix, L, row0, RM_RSTART, 0u,
                                                                       acc, false);
                }
            } else {
                nd_row_sweep<T, D, S, SL::count, IxRow<T>, OBSMAX>(J, buf, (cx<T>*)nullptr, ix, L, row0, mode, P.obs, acc);
            }
            if (mode & (RM_FWD | RM_STORE))
#pragma unroll
                for (int r = 0; r < 8; ++r) v[r] = buf[ix.at(g, i + (r << logm))];
        }
        if (mode & RM_FWD) ndt_fft<T, -1>(v, buf, ix, logn, twm);
        if (mode & RM_STORE) {
            __syncthreads();
#pragma unroll
            for (int r = 0; r < 8; ++r) buf[ix.at(g, i + (r << logm))] = v[r];
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                for (int s = 0; s < S; ++s) {
                    const size_t row = ((size_t)s * J.N + row0) * sizeof(cx<T>) / 128;
                    for (unsigned y = 0; y < rows_state; y += rows_box)
                        tma_store_3d(&map, 0, (int)(row + y), 0,
                                     reinterpret_cast<unsigned char*>(buf) + ((size_t)s * rows_state + y) * 128);
                }
                bulk_commit();
            }
        }
        if (PHI) { // forward transform of the end-of-step copy, through the same stage, into phi
            if (tid == 0) bulk_wait_read_all(); // the psi store has read the stage
            ndt_fft<T, -1>(w, buf, ix, logn, twm);
            __syncthreads();
#pragma unroll
            for (int r = 0; r < 8; ++r) buf[ix.at(g, i + (r << logm))] = w[r];
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                for (int s = 0; s < S; ++s) {
                    const size_t row = ((size_t)s * J.N + row0) * sizeof(cx<T>) / 128;
                    for (unsigned y = 0; y < rows_state; y += rows_box)
                        tma_store_3d(&map_phi, 0, (int)(row + y), 0,
                                     reinterpret_cast<unsigned char*>(buf) + ((size_t)s * rows_state + y) * 128);
                }
                bulk_commit();
            }
        }
    }
    if (tid == 0) bulk_wait_all();
    if (failed) return;
    if (sums) {
        block_partials<SL::count>(acc, 0, J.part, J.nparts, part_base + blockIdx.x, act);
        for (size_t col = blockIdx.x + gridDim.x; col < P.nitems; col += gridDim.x) // columns no CTA owns
            for (int v = tid; v < SL::count; v += blockDim.x) {
                const size_t o = ((size_t)v * J.nparts + part_base + col) * 2;
                J.part[o] = 0.0;
                J.part[o + 1] = 0.0;
            }
    }
    if (F.enabled && nd_last_cta(&F.book->counter, gridDim.x)) nd_finalize_cta(J, F);
}

// per-axis kinetic phase exp(Complex(0, -k_i^2 / (2 m_j)) * dt) (Propagator.init, quantum_dynamics.zig:397-399)
// and the per-axis grid table: r (Grid.init, wavepacket.zig:55-74), k (:66-68), 0.5 k^2 / m_j (:109-119)
template <typename T> __global__ void nd_kphase_kernel(const __grid_constant__ NdJob<T> J, double2* out, double4* axis) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= J.d * J.n) return;
    const int j = e / J.n, idx = e - j * J.n;
    const double k = __dmul_rn(idx < J.n / 2 ? (double)idx : __dsub_rn((double)idx, (double)J.n), J.dkunit[j]);
    const double K = __dmul_rn(__dmul_rn(0.5, k), k) / J.mass[j];
    axis[e] = make_double4(__dadd_rn(J.lo[j], __dmul_rn((double)idx, J.span[j]) / (double)J.n), k, K, 0.0);
    const double zre = __dsub_rn(__dmul_rn(0.0, J.dt_re), __dmul_rn(-K, J.dt_im));
    const double zim = __dadd_rn(__dmul_rn(0.0, J.dt_im), __dmul_rn(-K, J.dt_re));
    double ore, oim;
    cexp_dev(zre, zim, ore, oim);
    out[e] = make_double2(ore, oim);
}

// ------------------------------------------------------------ setup, imaginary time, bookkeeping
// V(r, t), eigh, R (with_R) and cap weights at every grid point (wavepacket.zig:96-168,
// quantum_dynamics.zig:387-468); no sign continuity in more than one dimension
// Hamiltonian.update (wavepacket.zig:137-143) and, with_R, Propagator.update (quantum_dynamics.zig:430-468)
// at grid point g; the new eigenvectors are left in Ul.
template <typename T, int S>
__device__ __forceinline__ void nd_table_point(const NdJob<T>& J, size_t g, double t, int with_R, double (&Ul)[S * S]) {
    double r[3];
    grid_coords(J, g, r);
    double Vl[S * S], Vu[S * S], Wl[S];
    pot_eval(J.pot, r, t, Vl);
    for (int a = 0; a < S; ++a)
        for (int b = 0; b < S; ++b) Vu[a * S + b] = Vl[(a < b ? a : b) * S + (a < b ? b : a)];
    eigh_dev<S>(Vu, Wl, Ul);
    for (int e = 0; e < S * S; ++e) J.V[(size_t)e * J.N + g] = Vl[e];
    if (S > 1)
        for (int e = 0; e < S * S; ++e) J.U[(size_t)e * J.N + g] = Ul[e];
    if (!with_R) return;
    double cap_sum = 0;
    if (J.has_cap)
        for (int j = 0; j < J.d; ++j) {
            const double dist = fmax(0.0, fmax(J.cap_lo[j] - r[j], r[j] - J.cap_hi[j]));
            if (dist > 0) cap_sum = __dadd_rn(cap_sum, exp(__dmul_rn(J.cap_exp, dist)) - 1);
        }
    const double decay = exp(__dmul_rn(__dmul_rn(-0.5, cap_sum), hypot(J.dt_re, J.dt_im)));
    if (J.capw) J.capw[g] = 1 - decay * decay;
    int k = 0;
    for (int a = 0; a < S; ++a)
        for (int b = a; b < S; ++b) {
            double re, im;
            propagator_entry<S>(Wl, Ul, J.dt_re, J.dt_im, decay, a, b, re, im);
            J.R[(size_t)k * J.N + g] = mktab<T>(re, im);
            ++k;
        }
}

template <typename T, int S> __global__ void nd_table_kernel(const __grid_constant__ NdJob<T> J, double t, int with_R) {
    if (*J.stopped) return;
    const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (g >= J.N) return;
    double Ul[S * S];
    nd_table_point<T, S>(J, g, t, with_R, Ul);
}

// The same update for a time-dependent potential whose eigenvector signs are observed: per
// eigenvector j the partial sums of sum_k U_new[k][j] U_prev[k][j] over the grid (the global
// alignment with the previous update, wavepacket.zig:157-167), grid-stride over <= 1024 blocks of
// at most 16 warps.  nd_sign_flip_kernel applies the decision after the sums are reduced.
template <typename T, int S>
__global__ void nd_table_sign_kernel(const __grid_constant__ NdJob<T> J, double t, int with_R, size_t part_base) {
    if (*J.stopped) return;
    double acc[S];
#pragma unroll
    for (int j = 0; j < S; ++j) acc[j] = 0.0;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < J.N; g += (size_t)gridDim.x * blockDim.x) {
        double Uold[S * S], Ul[S * S];
        for (int e = 0; e < S * S; ++e) Uold[e] = J.U[(size_t)e * J.N + g];
        nd_table_point<T, S>(J, g, t, with_R, Ul);
#pragma unroll
        for (int j = 0; j < S; ++j) {
            double d = 0;
            for (int k = 0; k < S; ++k) d = __dadd_rn(d, __dmul_rn(Ul[k * S + j], Uold[k * S + j]));
            acc[j] += d;
        }
    }
    block_partials<S>(acc, 0, J.part, J.nparts, part_base + blockIdx.x);
}

// U[:, j] <- -U[:, j] at every point for the eigenvectors whose total overlap with the previous
// update's is negative (tot[j] < 0)
template <int S> __global__ void nd_sign_flip_kernel(double* __restrict__ U, size_t N, const double* __restrict__ tot,
                                                     const int* stopped) {
    if (*stopped) return;
    bool any = false;
    for (int j = 0; j < S; ++j) any |= tot[j] < 0;
    if (!any) return;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < N; g += (size_t)gridDim.x * blockDim.x)
        for (int j = 0; j < S; ++j)
            if (tot[j] < 0)
                for (int k = 0; k < S; ++k) U[(size_t)(k * S + j) * N + g] = -U[(size_t)(k * S + j) * N + g];
}

// setGaussian (wavepacket.zig:355-371) and the partial norms
template <typename T> __global__ void nd_gauss_kernel(const __grid_constant__ NdJob<T> J, size_t part_base) {
    double acc[1] = {0.0};
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < J.N; g += (size_t)gridDim.x * blockDim.x) {
        double r[3];
        grid_coords(J, g, r);
        double ere = 0, eim = 0;
        for (int j = 0; j < J.d; ++j) {
            const double dx = __dsub_rn(r[j], J.x0[j]);
            ere = __dadd_rn(ere, __dmul_rn(__dmul_rn(__dmul_rn(-0.5, J.gamma[j]), dx), dx));
            eim = __dadd_rn(eim, __dmul_rn(J.p0[j], dx));
        }
        double zr, zi;
        cexp_dev(ere, eim, zr, zi);
        for (int s = 0; s < J.S; ++s) {
            const cx<T> z = J.psi_init ? J.psi_init[(size_t)s * J.N + g] : s == J.ic_state ? mk<T>((T)zr, (T)zi) : mk<T>(0, 0);
            J.psi[(size_t)s * J.N + g] = z;
            acc[0] += (double)z.x * (double)z.x + (double)z.y * (double)z.y;
        }
    }
    block_partials<1>(acc, 0, J.part, J.nparts, part_base + blockIdx.x);
}

// psi /= sqrt(norm) (Complex.div by (s, 0), wavepacket.zig:282-284); optionally toDia and the acf reference
template <typename T, int S>
__global__ void nd_normalize_kernel(const __grid_constant__ NdJob<T> J, const double* __restrict__ sum, int to_dia,
                                    int save_psi0) {
    if (*J.stopped) return;
    const double sq = sqrt(sum[0] * J.dr), den = sq * sq;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < J.N; g += (size_t)gridDim.x * blockDim.x) {
        cx<T> x[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const cx<T> z = J.psi[(size_t)s * J.N + g];
            x[s] = mk<T>((T)((double)z.x * sq / den), (T)((double)z.y * sq / den));
        }
        if (to_dia && S > 1) { // toDia (wavepacket.zig:398-419)
            cx<T> y[S];
#pragma unroll
            for (int i = 0; i < S; ++i) {
                double re = 0, im = 0;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    const double u = J.U[(size_t)(i * S + k) * J.N + g];
                    re += (double)x[k].x * u;
                    im += (double)x[k].y * u;
                }
                y[i] = mk<T>((T)re, (T)im);
            }
#pragma unroll
            for (int i = 0; i < S; ++i) x[i] = y[i];
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            J.psi[(size_t)s * J.N + g] = x[s];
            if (save_psi0) J.psi0[(size_t)s * J.N + g] = x[s];
        }
    }
}

// partial sums of |psi|^2 (slot 0) or of <phi_o|psi> (slots 0, 1)
template <typename T> __global__ void nd_dot_kernel(const __grid_constant__ NdJob<T> J, int o, size_t part_base) {
    if (*J.stopped) return;
    double acc[2] = {0.0, 0.0};
    const cx<T>* ph = o >= 0 ? J.orth + (size_t)o * J.S * J.N : nullptr;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)J.S * J.N;
         e += (size_t)gridDim.x * blockDim.x) {
        const cx<T> z = J.psi[e];
        if (ph) {
            const cx<T> p = ph[e];
            acc[0] += (double)p.x * (double)z.x + (double)p.y * (double)z.y;
            acc[1] += (double)p.x * (double)z.y - (double)p.y * (double)z.x;
        } else {
            acc[0] += (double)z.x * (double)z.x + (double)z.y * (double)z.y;
        }
    }
    block_partials<2>(acc, 0, J.part, J.nparts, part_base + blockIdx.x);
}

// psi -= <phi_o|psi> dr phi_o (quantum_dynamics.zig:898-904)
template <typename T>
__global__ void nd_orth_apply_kernel(const __grid_constant__ NdJob<T> J, int o, const double* __restrict__ sum) {
    if (*J.stopped) return;
    const double ore = sum[0] * J.dr, oim = sum[1] * J.dr;
    const cx<T>* ph = J.orth + (size_t)o * J.S * J.N;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)J.S * J.N;
         e += (size_t)gridDim.x * blockDim.x) {
        const cx<T> p = ph[e], z = J.psi[e];
        J.psi[e] = mk<T>((T)((double)z.x - (ore * (double)p.x - oim * (double)p.y)),
                         (T)((double)z.y - (ore * (double)p.y + oim * (double)p.x)));
    }
}

} // namespace zqd
