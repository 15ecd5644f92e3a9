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
    __host__ __device__ int norm() const { return 0; }
    __host__ __device__ int pos() const { return 1; }
    __host__ __device__ int mom() const { return 1 + d; }
    __host__ __device__ int pop() const { return 1 + 2 * d; }
    __host__ __device__ int epot() const { return 1 + 2 * d + S; }
    __host__ __device__ int ekin() const { return 2 + 2 * d + S; }
    __host__ __device__ int acf() const { return 3 + 2 * d + S; }
    __host__ __device__ int width() const { return 5 + 2 * d + S; }
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
    cx<T>* R;          // [S(S+1)/2][n] upper triangle, row-major pair order
    const cx<T>* expk; // [n], position p = c*m + k2*q + u <-> wavenumber index c*q + u + m*k2
    double* V;         // [S*S][n]
    double* U;         // [S*S][n]
    const double* capw;
    const cx<T>* tw; // [n] exp(-2 pi i t / n), natural order
    cx<T>* psi_save; // [S][n] permuted, written at the end of the solve
    cx<T>* psi0;     // [S][n] permuted, autocorrelation reference
    const cx<T>* orth;
    int northo;
    double* hist;
    double* fin;
    int* rows;
    PotDev pot;
};

constexpr int NRED = 12;

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
                                              const cx<T>* __restrict__ tw, int twstride) {
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
                    cx<T> w = __ldg(&tw[((r * kk) << tshift) * twstride]);
                    v[k][r] = mul<T>(v[k][r], twiddle<SIGN, T>(w));
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
__device__ __noinline__ void fft_local(cx<T>* buf, int ldp, int logm, int nlines, const cx<T>* __restrict__ tw,
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

// ------------------------------------------------------------ reductions
struct RedSmem {
    double warp[32][NRED][2];
    double slot[2][NRED][2];
    double res[NRED];
};

// Sums NV compensated accumulators over the cluster; every thread of every
// CTA receives the same totals (fixed combination order: deterministic).
template <int NV, int C> __device__ __forceinline__ void cluster_sum(Acc (&a)[NV], double (&out)[NV], RedSmem* rs, int& slot) {
    static_assert(NV <= NRED, "too many reduction values");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
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
    if (threadIdx.x < NV) {
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
        if (threadIdx.x < NV) {
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
        if (threadIdx.x < NV) rs->res[threadIdx.x] = rs->slot[slot][threadIdx.x][0] + rs->slot[slot][threadIdx.x][1];
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = rs->res[v];
    slot ^= 1;
}

// One grid point of a time-dependent Hamiltonian/propagator update: V(r,t),
// its eigensystem and, with_R, the potential propagator (tables are
// component-major with n entries per component; idx is the point's slot).
template <typename T, int S>
__device__ __noinline__ void td_point_update(const PotDev& pot, double r, double t, bool with_R, double dt_re,
                                             double dt_im, double decay, double* V, double* U, cx<T>* R, size_t n,
                                             size_t idx) {
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
                R[(size_t)k * n + idx] = mk<T>((T)re, (T)im);
                ++k;
            }
    }
}

struct LaunchShape {
    int S, C, E, threads;
    size_t smem;
    cudaStream_t stream;
};

// ------------------------------------------------------------ solve pieces
// Per-CTA view of the job shared by the solve phases below.
template <typename T> struct LineCtx {
    const LineJob<T>* J; // shared-memory copy of the job descriptor
    cx<T>* psi;          // [S][ldp] position-space lines (local points j)
    cx<T>* kbuf;         // [S][ldp] wavenumber slots (C > 1)
    RedSmem* rs;
    int m, n, logm, q, ldp, cta, slot;
    size_t base; // offset of this CTA in the permuted tables
    double inv_n, dkunit;
};

template <typename T, int C> __device__ __forceinline__ double rpos(const LineCtx<T>& X, int j) {
    // grid coordinate of local point j (Grid.init, wavepacket.zig:66)
    double nn = (double)(X.cta + C * j);
    return __dadd_rn(X.J->lo, __dmul_rn(nn, X.J->hi - X.J->lo) / (double)X.n);
}
template <typename T> __device__ __forceinline__ double kval(const LineCtx<T>& X, int kidx) {
    // wavenumber (wavepacket.zig:68-70)
    double nn = (double)kidx;
    return __dmul_rn(kidx < X.n / 2 ? nn : __dsub_rn(nn, (double)X.n), X.dkunit);
}
template <typename T, int C> __device__ __forceinline__ int kindex(const LineCtx<T>& X, int e) {
    if constexpr (C > 1) {
        int k2 = e / X.q, u = e - k2 * X.q;
        return X.cta * X.q + u + X.m * k2;
    } else {
        return e;
    }
}
template <typename T> __device__ __forceinline__ cx<T>& at(const LineCtx<T>& X, cx<T>* buf, int s, int e) {
    return buf[s * X.ldp + padx<T>(e)];
}

// forward n-point transform across the cluster; result in kspace buffer
template <typename T, int S, int C>
__device__ __noinline__ void line_fft_forward(LineCtx<T>& X) {
    constexpr int E = ElemsOf<T>::E;
    const int nt = blockDim.x, tid = threadIdx.x, m = X.m, q = X.q;
    fft_local<T, -1, E>(X.psi, X.ldp, X.logm, S, X.J->tw, C);
    if constexpr (C > 1) {
        if (X.cta > 0)
            for (int e = tid; e < S * m; e += nt) {
                int s = e / m, k1 = e - s * m;
                cx<T>& z = at(X, X.psi, s, k1);
                z = mul<T>(z, __ldg(&X.J->tw[X.cta * k1]));
            }
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        for (int it = tid; it < S * q; it += nt) {
            int s = it / q, u = it - s * q, k1 = X.cta * q + u;
            cx<T> v[C];
#pragma unroll
            for (int cc = 0; cc < C; ++cc) v[cc] = *cl.map_shared_rank(&at(X, X.psi, s, k1), cc);
            dft<C, -1, T>(v);
#pragma unroll
            for (int k2 = 0; k2 < C; ++k2) at(X, X.kbuf, s, k2 * q + u) = v[k2];
        }
        __syncthreads();
    }
}

// inverse transform; leaves n * psi in position space (the caller applies 1/n)
template <typename T, int S, int C>
__device__ __noinline__ void line_fft_inverse(LineCtx<T>& X) {
    constexpr int E = ElemsOf<T>::E;
    const int nt = blockDim.x, tid = threadIdx.x, m = X.m, q = X.q;
    if constexpr (C > 1) {
        for (int it = tid; it < S * q; it += nt) {
            int s = it / q, u = it - s * q;
            cx<T> v[C];
#pragma unroll
            for (int k2 = 0; k2 < C; ++k2) v[k2] = at(X, X.kbuf, s, k2 * q + u);
            dft<C, 1, T>(v);
#pragma unroll
            for (int cc = 0; cc < C; ++cc) at(X, X.kbuf, s, cc * q + u) = v[cc];
        }
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        for (int e = tid; e < S * m; e += nt) {
            int s = e / m, k1 = e - s * m;
            int owner = k1 / q, u = k1 - owner * q;
            cx<T> v = *cl.map_shared_rank(&at(X, X.kbuf, s, X.cta * q + u), owner);
            if (X.cta > 0) v = mul<T>(v, conj<T>(__ldg(&X.J->tw[X.cta * k1])));
            at(X, X.psi, s, k1) = v;
        }
        __syncthreads();
    }
    fft_local<T, 1, E>(X.psi, X.ldp, X.logm, S, X.J->tw, C);
}

// kinetic phase (applyK, quantum_dynamics.zig:509-511)
template <typename T, int S, int C> __device__ __noinline__ void line_kphase(LineCtx<T>& X) {
    cx<T>* kb = C > 1 ? X.kbuf : X.psi;
    for (int e = threadIdx.x; e < S * X.m; e += blockDim.x) {
        int s = e / X.m, el = e - s * X.m;
        cx<T>& z = at(X, kb, s, el);
        z = mul<T>(__ldg(&X.J->expk[X.base + el]), z);
    }
    __syncthreads();
}

template <typename T, int S> __device__ __noinline__ void line_scale(LineCtx<T>& X, T sc) {
    for (int e = threadIdx.x; e < S * X.m; e += blockDim.x) {
        int s = e / X.m, j = e - s * X.m;
        cx<T>& z = at(X, X.psi, s, j);
        z = scale<T>(z, sc);
    }
    __syncthreads();
}

// psi_i <- sum_k R_ik psi_k (applyR, quantum_dynamics.zig:515-534); psi scaled by sc first
template <typename T, int S> __device__ __noinline__ void line_apply_r(LineCtx<T>& X, T sc) {
    constexpr int NSYM = S * (S + 1) / 2;
    const LineJob<T>& J = *X.J;
    for (int j = threadIdx.x; j < X.m; j += blockDim.x) {
        cx<T> r[NSYM], x[S], y[S];
#pragma unroll
        for (int c = 0; c < NSYM; ++c) r[c] = J.R[(size_t)c * X.n + X.base + j];
#pragma unroll
        for (int s = 0; s < S; ++s) x[s] = scale<T>(at(X, X.psi, s, j), sc);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            cx<T> acc = mk<T>(0, 0);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int a = i < k ? i : k, b = i < k ? k : i;
                const int idx = a * S - a * (a - 1) / 2 + (b - a);
                acc = add<T>(acc, mul<T>(r[idx], x[k]));
            }
            y[i] = acc;
        }
#pragma unroll
        for (int s = 0; s < S; ++s) at(X, X.psi, s, j) = y[s];
    }
    __syncthreads();
}

template <typename T, int S> __device__ __forceinline__ double Uat(const LineCtx<T>& X, int j, int k, int i) {
    // U[point][k*S+i]
    if constexpr (S == 1) return 1.0;
    else return X.J->U[(size_t)(k * S + i) * X.n + X.base + j];
}

template <typename T> __device__ __forceinline__ double capdecay(const LineJob<T>& J, double r) {
    // quantum_dynamics.zig:434-449
    double cap_sum = 0;
    if (J.has_cap) {
        double dist = fmax(0.0, fmax(J.cap_lo - r, r - J.cap_hi));
        if (dist > 0) cap_sum = __dadd_rn(cap_sum, exp(__dmul_rn(J.cap_exp, dist)) - 1);
    }
    return exp(__dmul_rn(__dmul_rn(-0.5, cap_sum), hypot(J.dt_re, J.dt_im)));
}

// time-dependent Hamiltonian.update (wavepacket.zig:137-143) and, with_R, Propagator.update
template <typename T, int S, int C> __device__ __noinline__ void line_ham_update(LineCtx<T>& X, double t, bool with_R) {
    const LineJob<T>& J = *X.J;
    for (int j = threadIdx.x; j < X.m; j += blockDim.x) {
        double r = rpos<T, C>(X, j);
        td_point_update<T, S>(J.pot, r, t, with_R, J.dt_re, J.dt_im, with_R ? capdecay(J, r) : 1.0, J.V, J.U, J.R,
                              (size_t)X.n, X.base + j);
    }
    __syncthreads();
}

// accumAbsorbed (quantum_dynamics.zig:471-499)
template <typename T, int S, int C> __device__ __noinline__ void line_absorbed(LineCtx<T>& X, double* pop_abs) {
    const LineJob<T>& J = *X.J;
    Acc a[S];
    for (int j = threadIdx.x; j < X.m; j += blockDim.x) {
        double w = J.capw[X.base + j];
        cx<T> x[S];
#pragma unroll
        for (int s = 0; s < S; ++s) x[s] = at(X, X.psi, s, j);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            if (J.adiabatic) {
                double are = 0, aim = 0;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    double u = Uat<T, S>(X, j, k, i);
                    are += (double)x[k].x * u;
                    aim += (double)x[k].y * u;
                }
                a[i].add(w * (are * are + aim * aim));
            } else {
                a[i].add(w * ((double)x[i].x * (double)x[i].x + (double)x[i].y * (double)x[i].y));
            }
        }
    }
    double out[S];
    cluster_sum<S, C>(a, out, X.rs, X.slot);
#pragma unroll
    for (int i = 0; i < S; ++i) pop_abs[i] += out[i] * J.dr;
}

// Observables.init (quantum_dynamics.zig:295-366); returns the norm
template <typename T, int S, int C>
__device__ __noinline__ double line_observe(LineCtx<T>& X, uint32_t mask, bool acf_on, double* row,
                                            const double* pop_abs) {
    const LineJob<T>& J = *X.J;
    const RowLayout L{1, S};
    const int m = X.m, nt = blockDim.x, tid = threadIdx.x;
    const bool c_pos = mask & WM_POS, c_mom = mask & WM_MOM, c_pop = mask & WM_POP;
    const bool c_ekin = (mask & WM_EKIN) || (mask & WM_ETOT), c_epot = (mask & WM_EPOT) || (mask & WM_ETOT);
    const bool c_norm = (mask & WM_NORM) || J.has_stop;
    // position-space sums: 0 norm, 1 pos, 2 epot, 3 acf re, 4 acf im, 5.. pop
    Acc a[5 + S];
    for (int j = tid; j < m; j += nt) {
        cx<T> x[S];
#pragma unroll
        for (int s = 0; s < S; ++s) x[s] = at(X, X.psi, s, j);
        const double r = rpos<T, C>(X, j);
        double m2 = 0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            double w = (double)x[s].x * (double)x[s].x + (double)x[s].y * (double)x[s].y;
            m2 += w;
            if (c_pop && !J.adiabatic) a[5 + s].add(w);
        }
        if (c_norm) a[0].add(m2);
        if (c_pos) a[1].add(m2 * r);
        if (c_epot) {
            double e = 0;
#pragma unroll
            for (int i = 0; i < S; ++i)
#pragma unroll
                for (int k = 0; k < S; ++k)
                    e += ((double)x[i].x * (double)x[k].x + (double)x[i].y * (double)x[k].y) *
                         J.V[(size_t)(i * S + k) * X.n + X.base + j];
            a[2].add(e);
        }
        if (acf_on) {
            double re = 0, im = 0;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                cx<T> z0 = J.psi0[(size_t)s * X.n + X.base + j];
                re += (double)z0.x * (double)x[s].x + (double)z0.y * (double)x[s].y;
                im += (double)z0.x * (double)x[s].y - (double)z0.y * (double)x[s].x;
            }
            a[3].add(re);
            a[4].add(im);
        }
        if (c_pop && J.adiabatic) {
#pragma unroll
            for (int i = 0; i < S; ++i) {
                double are = 0, aim = 0;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    double u = Uat<T, S>(X, j, k, i);
                    are += (double)x[k].x * u;
                    aim += (double)x[k].y * u;
                }
                a[5 + i].add(are * are + aim * aim);
            }
        }
    }
    double out[5 + S];
    cluster_sum<5 + S, C>(a, out, X.rs, X.slot);
    const double norm = out[0] * J.dr;
    row[L.norm()] = c_norm ? norm : nan("");
    row[L.pos()] = c_pos ? out[1] * J.dr : nan("");
    row[L.epot()] = c_epot ? out[2] * J.dr : nan("");
    row[L.acf()] = acf_on ? out[3] * J.dr : nan("");
    row[L.acf() + 1] = acf_on ? out[4] * J.dr : nan("");
#pragma unroll
    for (int s = 0; s < S; ++s) row[L.pop() + s] = c_pop ? out[5 + s] * J.dr + pop_abs[s] : nan("");
    row[L.mom()] = nan("");
    row[L.ekin()] = nan("");
    if (c_mom || c_ekin) { // momentum-space round trip (quantum_dynamics.zig:347-363)
        line_fft_forward<T, S, C>(X);
        cx<T>* kb = C > 1 ? X.kbuf : X.psi;
        Acc b[2];
        for (int e = tid; e < S * m; e += nt) {
            int s = e / m, el = e - s * m;
            cx<T> z = at(X, kb, s, el);
            double w = (double)z.x * (double)z.x + (double)z.y * (double)z.y;
            double kv = kval(X, kindex<T, C>(X, el));
            if (c_mom) b[0].add(w * kv);
            if (c_ekin) b[1].add(w * (0.5 * kv * kv / J.mass));
        }
        double o2[2];
        cluster_sum<2, C>(b, o2, X.rs, X.slot);
        row[L.mom()] = c_mom ? o2[0] * J.dk : nan("");
        row[L.ekin()] = c_ekin ? o2[1] * J.dk : nan("");
        line_fft_inverse<T, S, C>(X);
        line_scale<T, S>(X, (T)X.inv_n);
    }
    return norm;
}

// psi <- psi / sqrt(norm) as std.math.Complex.div by (s, 0) (wavepacket.zig:282-284)
template <typename T, int S, int C> __device__ __noinline__ void line_normalize(LineCtx<T>& X) {
    Acc a[1];
    for (int e = threadIdx.x; e < S * X.m; e += blockDim.x) {
        int s = e / X.m, j = e - s * X.m;
        cx<T> z = at(X, X.psi, s, j);
        a[0].add((double)z.x * (double)z.x + (double)z.y * (double)z.y);
    }
    double o[1];
    cluster_sum<1, C>(a, o, X.rs, X.slot);
    const double sq = sqrt(o[0] * X.J->dr), den = sq * sq;
    for (int e = threadIdx.x; e < S * X.m; e += blockDim.x) {
        int s = e / X.m, j = e - s * X.m;
        cx<T>& z = at(X, X.psi, s, j);
        double re = (double)z.x * sq / den, im = (double)z.y * sq / den;
        z = mk<T>((T)re, (T)im);
    }
    __syncthreads();
}

// imaginary-time Gram-Schmidt against the relaxed states (quantum_dynamics.zig:898-904)
template <typename T, int S, int C> __device__ __noinline__ void line_orthogonalize(LineCtx<T>& X) {
    const LineJob<T>& J = *X.J;
    for (int o = 0; o < J.northo; ++o) {
        const cx<T>* ph = J.orth + (size_t)o * S * X.n;
        Acc a[2];
        for (int e = threadIdx.x; e < S * X.m; e += blockDim.x) {
            int s = e / X.m, j = e - s * X.m;
            cx<T> p = ph[(size_t)s * X.n + X.base + j], z = at(X, X.psi, s, j);
            a[0].add((double)p.x * (double)z.x + (double)p.y * (double)z.y);
            a[1].add((double)p.x * (double)z.y - (double)p.y * (double)z.x);
        }
        double ov[2];
        cluster_sum<2, C>(a, ov, X.rs, X.slot);
        const double ore = ov[0] * J.dr, oim = ov[1] * J.dr;
        for (int e = threadIdx.x; e < S * X.m; e += blockDim.x) {
            int s = e / X.m, j = e - s * X.m;
            cx<T> p = ph[(size_t)s * X.n + X.base + j];
            cx<T>& z = at(X, X.psi, s, j);
            double re = (double)z.x - (ore * (double)p.x - oim * (double)p.y);
            double im = (double)z.y - (ore * (double)p.y + oim * (double)p.x);
            z = mk<T>((T)re, (T)im);
        }
        __syncthreads();
    }
}

// setGaussian (wavepacket.zig:355-371), toDia (:398-419), autocorrelation reference
template <typename T, int S, int C> __device__ __noinline__ void line_initial_state(LineCtx<T>& X) {
    const LineJob<T>& J = *X.J;
    const int m = X.m;
    for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
        int s = e / m, j = e - s * m;
        cx<T> z = mk<T>(0, 0);
        if (s == J.ic_state) {
            double dx = __dsub_rn(rpos<T, C>(X, j), J.x0);
            double ere = __dmul_rn(__dmul_rn(__dmul_rn(-0.5, J.gamma), dx), dx);
            double eim = __dmul_rn(J.p0, dx);
            double zr, zi;
            cexp_dev(ere, eim, zr, zi);
            z = mk<T>((T)zr, (T)zi);
        }
        at(X, X.psi, s, j) = z;
    }
    __syncthreads();
    line_normalize<T, S, C>(X);
    if (J.ic_adia && S > 1) {
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            cx<T> x[S];
#pragma unroll
            for (int s = 0; s < S; ++s) x[s] = at(X, X.psi, s, j);
#pragma unroll
            for (int i = 0; i < S; ++i) {
                double re = 0, im = 0;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    double u = Uat<T, S>(X, j, i, k);
                    re += (double)x[k].x * u;
                    im += (double)x[k].y * u;
                }
                at(X, X.psi, i, j) = mk<T>((T)re, (T)im);
            }
        }
        __syncthreads();
    }
    if (J.calc_acf) {
        for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
            int s = e / m, j = e - s * m;
            J.psi0[(size_t)s * X.n + X.base + j] = at(X, X.psi, s, j);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ the kernel
template <typename T, int S, int C>
__global__ void __launch_bounds__(512, 1) line_solve_kernel(const LineJob<T>* __restrict__ jobs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ LineJob<T> J;
    __shared__ RedSmem rs;

    const int cta = (C > 1) ? (int)cg::this_cluster().block_rank() : 0;
    const int jid = blockIdx.x / C;
    if (threadIdx.x == 0) J = jobs[jid];
    __syncthreads();

    LineCtx<T> X;
    X.J = &J;
    X.m = J.m;
    X.n = J.n;
    X.logm = J.logm;
    X.q = J.q;
    X.ldp = padded_len<T>(J.m);
    X.cta = cta;
    X.slot = 0;
    X.psi = reinterpret_cast<cx<T>*>(smem_raw);
    X.kbuf = X.psi + S * X.ldp;
    X.rs = &rs;
    X.base = (size_t)cta * J.m;
    X.inv_n = 1.0 / (double)J.n;
    X.dkunit = 6.283185307179586476925286766559 / (J.hi - J.lo);

    double pop_abs[S];
#pragma unroll
    for (int s = 0; s < S; ++s) pop_abs[s] = 0;

    line_initial_state<T, S, C>(X);
    const int HC = RowLayout{1, S}.width();
    int rows = J.iters + 1;
    double row[16];
    for (int i = 0; i <= J.iters; ++i) {
        if (i > 0) { // Propagator.step (quantum_dynamics.zig:417-427)
            if (J.td) line_ham_update<T, S, C>(X, ((double)i - 0.5) * J.tstep, true);
            if (J.track) line_absorbed<T, S, C>(X, pop_abs);
            line_apply_r<T, S>(X, (T)1);
            line_fft_forward<T, S, C>(X);
            line_kphase<T, S, C>(X);
            line_fft_inverse<T, S, C>(X);
            if (J.track) {
                line_scale<T, S>(X, (T)X.inv_n);
                line_absorbed<T, S, C>(X, pop_abs);
                line_apply_r<T, S>(X, (T)1);
            } else {
                line_apply_r<T, S>(X, (T)X.inv_n); // the 1/N of the inverse FFT, fused (power of two: exact)
            }
        }
        if (J.itp) {
            line_orthogonalize<T, S, C>(X);
            line_normalize<T, S, C>(X);
        }
        if (J.td) line_ham_update<T, S, C>(X, (double)i * J.tstep, false);
        const bool logstep = J.log && ((i % J.log_interval == 0) || (i == J.iters));
        const uint32_t mask = J.wmask | (logstep ? (uint32_t)WM_ALL_OBS : 0u);
        const double nrm = line_observe<T, S, C>(X, mask, J.calc_acf != 0, row, pop_abs);
        if (cta == 0 && threadIdx.x == 0)
            for (int c = 0; c < HC; ++c) J.hist[(size_t)i * HC + c] = row[c];
        if (J.has_stop && nrm < J.stop_norm) { // stop_norm (quantum_dynamics.zig:933-944)
            rows = i + 1;
            break;
        }
    }
    line_observe<T, S, C>(X, WM_ALL_OBS, J.calc_acf != 0, row, pop_abs);
    if (cta == 0 && threadIdx.x == 0) {
        for (int c = 0; c < HC; ++c) J.fin[c] = row[c];
        *J.rows = rows;
    }
    for (int e = threadIdx.x; e < S * X.m; e += blockDim.x) {
        int s = e / X.m, j = e - s * X.m;
        J.psi_save[(size_t)s * X.n + X.base + j] = at(X, X.psi, s, j);
    }
    if constexpr (C > 1) cg::this_cluster().sync(); // keep shared memory alive for remote readers
}

} // namespace zqd
