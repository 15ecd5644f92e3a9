// line_kernel.cuh -- the resident 1-D split-operator propagator.
//
// One thread-block cluster of C CTAs advances one 1-D job through a whole
// solve (src/quantum_dynamics.zig:860-950) in a single launch.  The
// wavefunction never leaves shared memory between steps: CTA c owns the grid
// points x = c + C*j (j < m = n/C) of every state.  A step is
//   applyR -> forward FFT -> exp(-i K dt) -> inverse FFT -> applyR
// (Propagator.step, :417-427) where the n-point FFT is a four-step transform:
// m-point Stockham FFTs inside each CTA, a twiddle exp(-2 pi i c k1/n), and
// C-point DFTs across the cluster, exchanged through distributed shared
// memory (plain ld.shared::cluster, no TMA multicast).  After the forward
// transform CTA c' owns the wavenumbers k = c'q + u + m*k2 (q = m/C).
// Observables (Observables.init, :295-366) are reduced inside the cluster in
// FP64 with compensated sums and written to a history row per step.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "cx.cuh"
#include "physics.cuh"

namespace zqd {
namespace cg = cooperative_groups;

// history / final-observable row layout: norm | pos[d] | mom[d] | pop[S] | epot | ekin | acf re | acf im
struct RowLayout {
    int d, S;
    __host__ __device__ constexpr int norm() const { return 0; }
    __host__ __device__ constexpr int pos() const { return 1; }
    __host__ __device__ constexpr int mom() const { return 1 + d; }
    __host__ __device__ constexpr int pop() const { return 1 + 2 * d; }
    __host__ __device__ constexpr int epot() const { return 1 + 2 * d + S; }
    __host__ __device__ constexpr int ekin() const { return 2 + 2 * d + S; }
    __host__ __device__ constexpr int acf() const { return 3 + 2 * d + S; }
    __host__ __device__ constexpr int width() const { return 5 + 2 * d + S; }
};

enum : uint32_t {
    WM_ACF = 1u << 0,
    WM_EKIN = 1u << 1,
    WM_MOM = 1u << 2,
    WM_NORM = 1u << 3,
    WM_POP = 1u << 4,
    WM_POS = 1u << 5,
    WM_EPOT = 1u << 6,
    WM_ETOT = 1u << 7,
    WM_WFN = 1u << 8,
    WM_ALL_OBS = WM_EKIN | WM_MOM | WM_NORM | WM_POP | WM_POS | WM_EPOT,
};

template <typename T> struct LineJob {
    int n, m, logm, q;
    double lo, hi, dr, dk, mass;
    int iters;
    double dt_re, dt_im, tstep;
    int itp;
    int ic_state, ic_adia;
    double x0, p0, gamma;
    uint32_t wmask;
    int log, log_interval, adiabatic, calc_acf;
    int track, has_stop;
    double stop_norm;
    int td, has_cap;
    double cap_lo, cap_hi, cap_exp;
    // tables in the cluster-permuted layout (position p = c*m + j <-> grid index c + C*j)
    Tab<T>* R;          // [S(S+1)/2][n] upper triangle, row-major pair order
    const Tab<T>* expk; // [n], position p = c*m + k2*q + u <-> wavenumber index c*q + u + m*k2
    double* V;         // [S*S][n]
    double* U;         // [S*S][n]
    const double* capw;
    const Tab<T>* tw; // [n] exp(-2 pi i t / n), natural order
    cx<T>* psi_save; // [S][n] permuted, written at the end of the solve
    cx<T>* psi0;     // [S][n] permuted, autocorrelation reference
    const cx<T>* orth;
    const cx<T>* psi_init; // [S][n] permuted initial wavefunction replacing the Gaussian, or null
    int r_global;          // R read from global memory instead of shared memory
    int lrmax;             // log2 of the largest local radix (threads per CTA = m >> lrmax)
    int u_smem;            // the shape reserved shared memory for the eigenvectors of the CTA's points
    cx<T>* wfn_hist;       // [step][S][n] permuted wavefunction history of this solve, or null
    // time-dependent potentials whose eigenvector signs are observed (the adiabatic wavefunction
    // history, or the toDia of a later imaginary-time solve): after every update the 1-D
    // continuity rule and the global alignment with the previous update (wavepacket.zig:145-167)
    int sign_track;
    double* sgn; // [S][n] natural order: overlap of each new eigenvector with the previous one
    int northo;
    double* hist;
    double* fin;
    int* rows; // rows of the history written so far
    // Step range of this launch: rows i0..i1 of the solve (0..iters for the whole solve).  A launch
    // with i0 > 0 resumes from psi_save and the carried absorbed populations; a launch that ends
    // before the last step (and before stop_norm) saves both instead of the final observables.
    int i0, i1;
    double* carry; // [S] absorbed populations between launches of one solve
    int* done;     // 1 once the solve has ended (last step or stop_norm)
    int* progress; // or null: rows written so far, published to the host after every row (pinned memory)
    PotDev pot;
};

constexpr int NRED = 16;

template <typename T> struct PadOf;
template <> struct PadOf<double> { static constexpr int sh = 3; };
template <> struct PadOf<float> { static constexpr int sh = 4; };
template <typename T> __device__ __forceinline__ int padx(int e) { return e + (e >> PadOf<T>::sh); }
template <typename T> __host__ __device__ inline int padded_len(int m) { return m + (m >> PadOf<T>::sh); }
// elements each thread holds per FFT pass
template <typename T> struct ElemsOf;
template <> struct ElemsOf<double> { static constexpr int E = 8; };
template <> struct ElemsOf<float> { static constexpr int E = 16; };

// ------------------------------------------------------------ local FFT
template <typename T, int R, int SIGN, int E>
__device__ __forceinline__ void stockham_pass(cx<T>* buf, int ldp, int logm, int nlines, int p, int logp,
                                              const Tab<T>* __restrict__ tw, int twstride) {
    constexpr int B = E / R;
    constexpr int LR = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
    const int logmr = logm - LR;
    const int mr = 1 << logmr;
    const int nb = nlines << logmr;
    const int nt = blockDim.x;
    cx<T> v[B][R];
#pragma unroll
    for (int k = 0; k < B; ++k) {
        int b = threadIdx.x + k * nt;
        if (b < nb) {
            int s = b >> logmr, i = b & (mr - 1);
            const cx<T>* line = buf + s * ldp;
#pragma unroll
            for (int r = 0; r < R; ++r) v[k][r] = line[padx<T>(i + r * mr)];
        }
    }
    __syncthreads();
    // twiddle index for (r, kk): r * kk * (m / (p R)) * twstride
    const int tshift = logm - logp - LR;
#pragma unroll
    for (int k = 0; k < B; ++k) {
        int b = threadIdx.x + k * nt;
        if (b < nb) {
            int s = b >> logmr, i = b & (mr - 1);
            int kk = i & (p - 1);
            if (p > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    v[k][r] = tmul<SIGN>(v[k][r], __ldg(&tw[((r * kk) << tshift) * twstride]));
                }
            }
            dft<R, SIGN, T>(v[k]);
            cx<T>* line = buf + s * ldp;
            int base = ((i - kk) << LR) + kk;
#pragma unroll
            for (int r = 0; r < R; ++r) line[padx<T>(base + r * p)] = v[k][r];
        }
    }
    __syncthreads();
}

// nlines lines of m = 2^logm points, natural order in and out, unnormalised.
template <typename T, int SIGN, int E>
__device__ __forceinline__ void fft_local(cx<T>* buf, int ldp, int logm, int nlines, const Tab<T>* __restrict__ tw,
                                       int twstride) {
    int p = 1, logp = 0, rem = logm;
    while (rem > 0) {
        if (rem >= 3) {
            stockham_pass<T, 8, SIGN, E>(buf, ldp, logm, nlines, p, logp, tw, twstride);
            p <<= 3;
            logp += 3;
            rem -= 3;
        } else if (rem == 2) {
            stockham_pass<T, 4, SIGN, E>(buf, ldp, logm, nlines, p, logp, tw, twstride);
            p <<= 2;
            logp += 2;
            rem -= 2;
        } else {
            stockham_pass<T, 2, SIGN, E>(buf, ldp, logm, nlines, p, logp, tw, twstride);
            p <<= 1;
            logp += 1;
            rem -= 1;
        }
    }
}

// Cluster barrier without memory ordering (a relaxed arrive carries no release fence): for
// write-after-read protection only, where every remote read before it has been consumed.
__device__ __forceinline__ void cluster_barrier_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
}

// ------------------------------------------------------------ reductions
struct RedSmem {
    double warp[32][NRED][2];
    double slot[2][NRED][2];
    double res[NRED];
    int slot_idx; // alternates between the two cluster-visible slots
};

// Sums NV compensated accumulators over the cluster; every thread of every
// CTA receives the same totals (fixed combination order: deterministic).
// Only the values whose bit is set in `active` (uniform over the cluster) are
// reduced, the others come back as 0: a step that records one observable
// pays for that one.  Consecutive calls alternate between two slots, so one
// cluster barrier per call suffices: a CTA can only overwrite a slot after
// every CTA has passed the barrier of the following call, i.e. after it
// finished reading.
template <int NV, int C>
__device__ __forceinline__ void cluster_sum(Acc (&a)[NV], double (&out)[NV], RedSmem* rs, uint32_t active = ~0u) {
    static_assert(NV <= NRED, "too many reduction values");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    const int slot = rs->slot_idx;
    const bool mine = threadIdx.x < NV && ((active >> threadIdx.x) & 1u);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        if (!((active >> v) & 1u)) continue;
        double s = a[v].s, c = a[v].c;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            double s2 = __shfl_down_sync(0xffffffffu, s, off);
            double c2 = __shfl_down_sync(0xffffffffu, c, off);
            Acc t;
            t.s = s;
            t.c = c;
            t.add(s2);
            t.c += c2;
            s = t.s;
            c = t.c;
        }
        if (lane == 0) {
            rs->warp[warp][v][0] = s;
            rs->warp[warp][v][1] = c;
        }
    }
    __syncthreads();
    if (mine) {
        Acc t;
        for (int w = 0; w < nw; ++w) {
            t.add(rs->warp[w][threadIdx.x][0]);
            t.c += rs->warp[w][threadIdx.x][1];
        }
        rs->slot[slot][threadIdx.x][0] = t.s;
        rs->slot[slot][threadIdx.x][1] = t.c;
    }
    if constexpr (C > 1) {
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        if (threadIdx.x < NV && !mine) rs->res[threadIdx.x] = 0.0;
        if (mine) {
            Acc t;
            for (int cc = 0; cc < C; ++cc) {
                const double* rem = cl.map_shared_rank(&rs->slot[slot][threadIdx.x][0], cc);
                t.add(rem[0]);
                t.c += rem[1];
            }
            rs->res[threadIdx.x] = t.value();
        }
    } else {
        __syncthreads();
        if (threadIdx.x < NV) rs->res[threadIdx.x] = mine ? rs->slot[slot][threadIdx.x][0] + rs->slot[slot][threadIdx.x][1] : 0.0;
    }
    if (threadIdx.x == 0) rs->slot_idx = slot ^ 1; // every thread read slot_idx before the first barrier
    __syncthreads();
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = rs->res[v];
}

// One grid point of a time-dependent Hamiltonian/propagator update: V(r,t),
// its eigensystem and, with_R, the potential propagator (tables are
// component-major with n entries per component; idx is the point's slot).
template <typename T, int S>
__device__ __noinline__ void td_point_update(const PotDev& pot, double r, double t, bool with_R, double dt_re,
                                             double dt_im, double decay, double* V, double* U, size_t n, size_t idx,
                                             Tab<T>* R, size_t rstride, size_t ridx) {
    double Vl[S * S], Wl[S], Ul[S * S], Vu[S * S];
    pot_eval(pot, &r, t, Vl);
    for (int a = 0; a < S; ++a)
        for (int b = 0; b < S; ++b) Vu[a * S + b] = Vl[(a < b ? a : b) * S + (a < b ? b : a)];
    eigh_dev<S>(Vu, Wl, Ul);
    for (int e = 0; e < S * S; ++e) V[(size_t)e * n + idx] = Vl[e];
    if (S > 1)
        for (int e = 0; e < S * S; ++e) U[(size_t)e * n + idx] = Ul[e];
    if (with_R) {
        int k = 0;
        for (int a = 0; a < S; ++a)
            for (int b = a; b < S; ++b) {
                double re, im;
                propagator_entry<S>(Wl, Ul, dt_re, dt_im, decay, a, b, re, im);
                R[(size_t)k * rstride + ridx] = mktab<T>(re, im);
                ++k;
            }
    }
}

struct LaunchShape {
    int S, C, E, threads;
    size_t smem;
    cudaStream_t stream;
    int lrmax = 2; // log2 of the largest local radix: 2 (radix 4) or 3 (radix 8, 16-CTA clusters only)
};


} // namespace zqd
