// line_solve.cuh -- the fused resident 1-D solve (src/quantum_dynamics.zig:860-950).
//
// Shared memory of a CTA holds two wavefunction buffers (the Stockham passes
// ping-pong between them, one barrier per pass), the local passes' twiddles
// (pass by pass, so that a warp reads them contiguously), the cluster twiddles
// exp(-2 pi i c k1/n), the potential propagator R at the CTA's grid points and
// the kinetic phase at its wavenumbers.  One time step (Propagator.step,
// :417-427) is
//   forward FFT   first pass: [accumAbsorbed], psi <- R psi, butterflies
//                 last pass : butterflies, cluster twiddle (C > 1) or kinetic phase (C = 1)
//   exchange      C-point DFTs across the cluster with the kinetic phase between them (C > 1)
//   inverse FFT   first pass: remote gather of the exchanged values (C > 1), butterflies
//                 last pass : butterflies, 1/N, [accumAbsorbed], psi <- R psi, observables
// followed by one cluster reduction of the observables the step records.  The two
// passes that apply R take all states of a butterfly in one thread; the other passes
// and the exchange take one (butterfly or column, state) pair per thread.
#pragma once

#include "line_kernel.cuh"

namespace zqd {

// dynamic shared memory of one CTA
// r_global: the R table is read from global memory (L2) instead of being staged, for the
// largest lines whose R slice does not fit next to the wavefunction buffers
// lrm: log2 of the largest local radix; the inverse transform's pass schedule needs a twiddle table
// of its own when m is not a power of 2^lrm
__host__ __device__ inline bool line_two_schedules(int m, int lrm) {
    int logm = 0;
    while ((1 << logm) < m) ++logm;
    return logm % lrm != 0;
}
// u_smem: room for the S x S eigenvectors of the CTA's points (FP64) after the tables
template <typename T>
__host__ __device__ inline size_t line_smem_bytes(int S, int C, int m, bool r_global, int lrm, bool u_smem = false) {
    const size_t ld = (size_t)padded_len<T>(m), nsym = r_global ? 0 : (size_t)S * (S + 1) / 2;
    const size_t ntw = line_two_schedules(m, lrm) ? 2 : 1;
    return 2 * (size_t)S * ld * sizeof(cx<T>) + ((C > 1 ? 1 : 0) + ntw + nsym + 1) * (size_t)m * sizeof(Tab<T>) +
           (u_smem ? (size_t)S * S * m * sizeof(double) : 0);
}

// reduction slots of a step
enum : int { A_NORM = 0, A_POS, A_EPOT, A_ACFR, A_ACFI, A_MOM, A_EKIN, A_POP };
template <int S> struct NAcc { static constexpr int value = A_POP + 2 * S; }; // pop[S] then absorbed[S]

struct ObsFlags {
    bool norm, pos, epot, acf, pop, mom, ekin, adia, track;
};

template <typename T> __device__ __forceinline__ const cx<T>* remote(const cx<T>* p, int rank) {
    return cg::this_cluster().map_shared_rank(p, rank);
}

template <int C> __device__ __forceinline__ double grid_r(double lo, double span, int n, int cta, int j) {
    // grid coordinate of local point j: min + x (max - min) / n (Grid.init, wavepacket.zig:66)
    return __dadd_rn(lo, __dmul_rn((double)(cta + C * j), span) / (double)n);
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

// psi_i <- sum_k R_ik psi_k at one point (applyR, quantum_dynamics.zig:515-534)
template <typename T, int S>
__device__ __forceinline__ void apply_r_point(cx<T>* x, const Tab<T>* __restrict__ Rs, int m, int j) {
    constexpr int NSYM = S * (S + 1) / 2;
    Tab<T> r[NSYM];
#pragma unroll
    for (int c = 0; c < NSYM; ++c) r[c] = Rs[c * m + j];
    cx<T> y[S];
#pragma unroll
    for (int i = 0; i < S; ++i) {
        cx<T> acc = mk<T>(0, 0);
#pragma unroll
        for (int k = 0; k < S; ++k) {
            const int a = i < k ? i : k, b = i < k ? k : i;
            acc = add<T>(acc, tmul<-1>(x[k], r[a * S - a * (a - 1) / 2 + (b - a)]));
        }
        y[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < S; ++i) x[i] = y[i];
}

// cap_weight-weighted populations at one point (accumAbsorbed, quantum_dynamics.zig:471-499)
template <typename T, int S>
__device__ __forceinline__ void absorbed_point(Acc* acc, const cx<T>* x, double w, const double* __restrict__ U, int n,
                                               int j, bool adia) {
#pragma unroll
    for (int i = 0; i < S; ++i) {
        if (adia && S > 1) {
            double are = 0, aim = 0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const double u = U[(size_t)(k * S + i) * n + j];
                are += (double)x[k].x * u;
                aim += (double)x[k].y * u;
            }
            acc[A_POP + S + i].add(w * (are * are + aim * aim));
        } else {
            acc[A_POP + S + i].add(w * ((double)x[i].x * (double)x[i].x + (double)x[i].y * (double)x[i].y));
        }
    }
}

// position-space observables of one point (wavepacket.zig:235-352, Observables.init :321-345)
// U: the eigenvectors of the CTA's points, component e of point j at U[e * us + j]
template <typename T, int S>
__device__ __forceinline__ void observe_point(Acc* acc, const cx<T>* x, double r, const LineJob<T>& J, size_t gidx,
                                              const ObsFlags& f, const double* __restrict__ U, int us, int j) {
    double m2 = 0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const double w = (double)x[s].x * (double)x[s].x + (double)x[s].y * (double)x[s].y;
        m2 += w;
        if (f.pop && !(f.adia && S > 1)) acc[A_POP + s].add(w);
    }
    if (f.norm) acc[A_NORM].add(m2);
    if (f.pos) acc[A_POS].add(m2 * r);
    if (f.epot) {
        double e = 0;
#pragma unroll
        for (int i = 0; i < S; ++i)
#pragma unroll
            for (int k = 0; k < S; ++k)
                e += ((double)x[i].x * (double)x[k].x + (double)x[i].y * (double)x[k].y) *
                     J.V[(size_t)(i * S + k) * J.n + gidx];
        acc[A_EPOT].add(e);
    }
    if (f.acf) {
        double re = 0, im = 0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const cx<T> z0 = J.psi0[(size_t)s * J.n + gidx];
            re += (double)z0.x * (double)x[s].x + (double)z0.y * (double)x[s].y;
            im += (double)z0.x * (double)x[s].y - (double)z0.y * (double)x[s].x;
        }
        acc[A_ACFR].add(re);
        acc[A_ACFI].add(im);
    }
    if (f.pop && f.adia && S > 1) {
#pragma unroll
        for (int i = 0; i < S; ++i) {
            double are = 0, aim = 0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const double u = U[(size_t)(k * S + i) * us + j];
                are += (double)x[k].x * u;
                aim += (double)x[k].y * u;
            }
            acc[A_POP + i].add(are * are + aim * aim);
        }
    }
}

// momentum-space observables of one wavenumber slot (wavepacket.zig:224-232, 258-268)
template <typename T, int S>
__device__ __forceinline__ void observe_k(Acc* acc, const cx<T>* z, int kidx, int n, double dkunit, double mass,
                                          const ObsFlags& f) {
    double w = 0;
#pragma unroll
    for (int s = 0; s < S; ++s) w += (double)z[s].x * (double)z[s].x + (double)z[s].y * (double)z[s].y;
    const double nn = (double)kidx;
    const double kv = __dmul_rn(kidx < n / 2 ? nn : __dsub_rn(nn, (double)n), dkunit); // wavepacket.zig:68-70
    if (f.mom) acc[A_MOM].add(w * kv);
    if (f.ekin) acc[A_EKIN].add(w * (0.5 * kv * kv / mass));
}

// observe_k for the wavenumber slot of one state: the state's share of the k-space sums
template <typename T>
__device__ __forceinline__ void observe_k1(Acc* acc, const cx<T>& z, int kidx, int n, double dkunit, double mass,
                                           const ObsFlags& f) {
    const double w = (double)z.x * (double)z.x + (double)z.y * (double)z.y;
    const double nn = (double)kidx;
    const double kv = __dmul_rn(kidx < n / 2 ? nn : __dsub_rn(nn, (double)n), dkunit); // wavepacket.zig:68-70
    if (f.mom) acc[A_MOM].add(w * kv);
    if (f.ekin) acc[A_EKIN].add(w * (0.5 * kv * kv / mass));
}

// ------------------------------------------------------------ rare phases
// (initial state, imaginary time, time-dependent updates): out of line
template <typename T> struct LineCtx {
    const LineJob<T>* J;
    cx<T>* psi; // current wavefunction buffer
    cx<T>* spare;
    RedSmem* rs;
    int m, n, logm, q, ldp, cta;
    size_t base;
};

// psi <- psi / sqrt(norm) as std.math.Complex.div by (s, 0) (wavepacket.zig:282-284)
template <typename T, int S, int C> __device__ __noinline__ void line_normalize(const LineCtx<T>& X) {
    const int m = X.m, ldp = X.ldp;
    cx<T>* __restrict__ psi = X.psi;
    Acc a[1];
    for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
        const int s = e / m, j = e - s * m;
        const cx<T> z = psi[s * ldp + padx<T>(j)];
        a[0].add((double)z.x * (double)z.x + (double)z.y * (double)z.y);
    }
    double o[1];
    cluster_sum<1, C>(a, o, X.rs);
    const double sq = sqrt(o[0] * X.J->dr), den = sq * sq;
    for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
        const int s = e / m, j = e - s * m;
        cx<T>& z = psi[s * ldp + padx<T>(j)];
        z = mk<T>((T)((double)z.x * sq / den), (T)((double)z.y * sq / den));
    }
    __syncthreads();
}

// imaginary-time Gram-Schmidt against the relaxed states (quantum_dynamics.zig:898-904)
template <typename T, int S, int C> __device__ __noinline__ void line_orthogonalize(const LineCtx<T>& X) {
    const int m = X.m, ldp = X.ldp, n = X.n, northo = X.J->northo;
    cx<T>* __restrict__ psi = X.psi;
    const double dr = X.J->dr;
    for (int o = 0; o < northo; ++o) {
        const cx<T>* __restrict__ ph = X.J->orth + (size_t)o * S * n + X.base;
        Acc a[2];
        for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
            const int s = e / m, j = e - s * m;
            const cx<T> p = ph[(size_t)s * n + j], z = psi[s * ldp + padx<T>(j)];
            a[0].add((double)p.x * (double)z.x + (double)p.y * (double)z.y);
            a[1].add((double)p.x * (double)z.y - (double)p.y * (double)z.x);
        }
        double ov[2];
        cluster_sum<2, C>(a, ov, X.rs);
        const double ore = ov[0] * dr, oim = ov[1] * dr;
        for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
            const int s = e / m, j = e - s * m;
            const cx<T> p = ph[(size_t)s * n + j];
            cx<T>& z = psi[s * ldp + padx<T>(j)];
            const double re = (double)z.x - (ore * (double)p.x - oim * (double)p.y);
            const double im = (double)z.y - (ore * (double)p.y + oim * (double)p.x);
            z = mk<T>((T)re, (T)im);
        }
        __syncthreads();
    }
}

// Sign maps of the 1-D eigenvector continuity scan, two bits: 0 s -> s, 1 s -> -s, 2 s -> +1,
// 3 s -> -1 (a sign s is the bit 0 for +1, 1 for -1).  map_after(f, g) is f applied after g.
__device__ __forceinline__ int map_after(int f, int g) { return (f & 2) ? f : (g ^ (f & 1)); }

// Eigenvector signs after a time-dependent update (Hamiltonian.update, wavepacket.zig:145-167).
// J.U holds this update's raw eigenvectors, J.sgn their overlaps d_x with the previous update's
// (natural order).  Continuity (:145-155): at x > 0 the vector is flipped when its overlap with
// the already fixed vector at x - 1 is negative, i.e. s_x = s_{x-1}, -s_{x-1} or +1 for a
// positive, negative or zero raw overlap, s_0 = +1: a scan of sign maps.  CTA c scans the natural
// points [c m, (c+1) m) -- per thread a run of points, then warps, the CTA and the cluster.
// Global alignment (:157-167): g_j = sign of sum_x s_x d_x (the new vectors after continuity
// against the previous ones), and U <- g_j s_x U.  The overlaps are rounded like the reference's
// (separate multiply and add, in k order), so the decisions are its decisions.
template <typename T, int S, int C> __device__ __noinline__ void line_sign_align(const LineCtx<T>& X) {
    const LineJob<T>& J = *X.J;
    const int m = X.m, n = X.n, cta = X.cta, nt = blockDim.x, t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5, nw = (nt + 31) >> 5;
    double* __restrict__ U = J.U;
    __shared__ int wmap[32][S];
    __shared__ int cmap[S]; // this CTA's composed map, read by the later CTAs of the cluster
    // the spare wavefunction buffer holds the per-point codes; remote CTAs may still gather from
    // it until every CTA has left the step
    if constexpr (C > 1) cg::this_cluster().sync();
    signed char* code = reinterpret_cast<signed char*>(X.spare);
    auto pos = [&](int x) { return (size_t)(x % C) * m + x / C; };
    const int chunk = (m + nt - 1) / nt;
    const int x0 = cta * m + min(m, t * chunk), x1 = cta * m + min(m, (t + 1) * chunk);
    int tm[S];
#pragma unroll
    for (int jc = 0; jc < S; ++jc) {
        int f = 0;
        for (int x = x0; x < x1; ++x) {
            int cd = 2; // s_0 = +1
            if (x > 0) {
                double ov = 0;
                for (int k = 0; k < S; ++k)
                    ov = __dadd_rn(ov, __dmul_rn(U[(size_t)(k * S + jc) * n + pos(x)], U[(size_t)(k * S + jc) * n + pos(x - 1)]));
                cd = ov > 0 ? 0 : (ov < 0 ? 1 : 2);
            }
            code[(size_t)(x - cta * m) * S + jc] = (signed char)cd;
            f = map_after(cd, f);
        }
        // inclusive scan over the warp's lanes (later lanes apply after earlier ones)
        int inc = f;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, inc, off);
            if (lane >= off) inc = map_after(inc, o);
        }
        const int exc = __shfl_up_sync(0xffffffffu, inc, 1);
        tm[jc] = lane ? exc : 0;
        if (lane == 31) wmap[warp][jc] = inc;
    }
    __syncthreads();
    if (t < S) { // exclusive scan over the warps; the CTA's own composed map
        int acc = 0;
        for (int w = 0; w < nw; ++w) {
            const int wm = wmap[w][t];
            wmap[w][t] = acc;
            acc = map_after(wm, acc);
        }
        cmap[t] = acc;
    }
    if constexpr (C > 1) cg::this_cluster().sync();
    else __syncthreads();
    Acc tot[S];
#pragma unroll
    for (int jc = 0; jc < S; ++jc) {
        int entry = 0; // the earlier CTAs' maps, in order
        if constexpr (C > 1)
            for (int c = 0; c < cta; ++c) entry = map_after(*cg::this_cluster().map_shared_rank(&cmap[jc], c), entry);
        int f = map_after(tm[jc], map_after(wmap[warp][jc], entry));
        for (int x = x0; x < x1; ++x) {
            f = map_after(code[(size_t)(x - cta * m) * S + jc], f);
            const double d = J.sgn[(size_t)jc * n + x];
            tot[jc].add((f & 1) ? -d : d);
        }
        tm[jc] = map_after(tm[jc], map_after(wmap[warp][jc], entry)); // the sign map entering this thread's run
    }
    double g[S];
    cluster_sum<S, C>(tot, g, X.rs);
#pragma unroll
    for (int jc = 0; jc < S; ++jc) {
        const int gneg = g[jc] < 0 ? 1 : 0;
        int f = tm[jc];
        for (int x = x0; x < x1; ++x) {
            f = map_after(code[(size_t)(x - cta * m) * S + jc], f);
            if ((f & 1) ^ gneg)
                for (int k = 0; k < S; ++k) {
                    double* u = &U[(size_t)(k * S + jc) * n + pos(x)];
                    *u = -*u;
                }
        }
    }
    __threadfence();
    if constexpr (C > 1) cg::this_cluster().sync(); // every CTA reads U at its own points next
    else __syncthreads();
}

// time-dependent Hamiltonian.update (wavepacket.zig:137-143) and, with_R,
// Propagator.update into the shared-memory R table
template <typename T, int S, int C>
__device__ __noinline__ void line_ham_update(const LineCtx<T>& X, double t, bool with_R, Tab<T>* Rs, int rstride,
                                             double lo, double span) {
    const LineJob<T>& J = *X.J;
    const bool track = S > 1 && J.sign_track;
    for (int j = threadIdx.x; j < X.m; j += blockDim.x) {
        const double r = grid_r<C>(lo, span, X.n, X.cta, j);
        const size_t idx = X.base + j;
        double Uold[S * S];
        if (track)
            for (int e = 0; e < S * S; ++e) Uold[e] = J.U[(size_t)e * X.n + idx];
        td_point_update<T, S>(J.pot, r, t, with_R, J.dt_re, J.dt_im, with_R ? capdecay(J, r) : 1.0, J.V, J.U,
                              (size_t)X.n, idx, Rs, (size_t)rstride, (size_t)j);
        if (track) { // overlap of every new (raw) eigenvector with the previous one at this point
            const int x = X.cta + C * j;
            for (int jc = 0; jc < S; ++jc) {
                double d = 0;
                for (int k = 0; k < S; ++k)
                    d = __dadd_rn(d, __dmul_rn(J.U[(size_t)(k * S + jc) * X.n + idx], Uold[k * S + jc]));
                J.sgn[(size_t)jc * X.n + x] = d;
            }
        }
    }
    __syncthreads();
    if constexpr (S > 1)
        if (track) line_sign_align<T, S, C>(X);
}

// setGaussian (wavepacket.zig:355-371), toDia (:398-419), autocorrelation reference
template <typename T, int S, int C>
__device__ __noinline__ void line_initial_state(const LineCtx<T>& X, double lo, double span) {
    const LineJob<T>& J = *X.J;
    const int m = X.m, ldp = X.ldp, n = X.n;
    cx<T>* __restrict__ psi = X.psi;
    for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
        const int s = e / m, j = e - s * m;
        cx<T> z = mk<T>(0, 0);
        if (J.psi_init) {
            z = J.psi_init[(size_t)s * n + X.base + j];
        } else if (s == J.ic_state) {
            const double dx = __dsub_rn(grid_r<C>(lo, span, n, X.cta, j), J.x0);
            const double ere = __dmul_rn(__dmul_rn(__dmul_rn(-0.5, J.gamma), dx), dx);
            const double eim = __dmul_rn(J.p0, dx);
            double zr, zi;
            cexp_dev(ere, eim, zr, zi);
            z = mk<T>((T)zr, (T)zi);
        }
        psi[s * ldp + padx<T>(j)] = z;
    }
    __syncthreads();
    line_normalize<T, S, C>(X);
    if (J.ic_adia && S > 1) {
        const double* __restrict__ U = J.U + X.base;
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            cx<T> x[S];
#pragma unroll
            for (int s = 0; s < S; ++s) x[s] = psi[s * ldp + padx<T>(j)];
#pragma unroll
            for (int i = 0; i < S; ++i) {
                double re = 0, im = 0;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    const double u = U[(size_t)(i * S + k) * n + j];
                    re += (double)x[k].x * u;
                    im += (double)x[k].y * u;
                }
                psi[i * ldp + padx<T>(j)] = mk<T>((T)re, (T)im);
            }
        }
        __syncthreads();
    }
    if (J.calc_acf) {
        cx<T>* __restrict__ psi0 = J.psi0 + X.base;
        for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
            const int s = e / m, j = e - s * m;
            psi0[(size_t)s * n + j] = psi[s * ldp + padx<T>(j)];
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ the kernel
// threads per CTA: m/8; FP64 CTAs are capped at 256 threads (m <= 2048) so a
// thread may use up to 255 registers for the S x 8 complex values of a butterfly
template <typename T> struct LineMaxThreads { static constexpr int value = 512; };
template <> struct LineMaxThreads<double> { static constexpr int value = 256; };

// FUSE_NEXT (with INV_LAST): the pass also runs the next step's forward first pass on the same
// points (the last inverse pass leaves point i + r m/R with the thread of butterfly i, which is
// where the forward first pass takes it from)
enum PassKind : int { FWD_FIRST = 1, FWD_LAST = 2, INV_FIRST = 4, INV_LAST = 8, FUSE_NEXT = 16 };

// log2 of the radix of local pass `idx` of an m = 2^logm point transform: 2^lrm (8, or 4 with twice
// the threads and only the radix-4/2 code compiled, which keeps the kernel's instruction footprint
// small), except for one smaller remainder pass: the forward transform's first, the inverse's last.
// The inverse's last pass and the forward's first pass then have the same radix and the same
// points per butterfly, and the passes with state-mixing hooks (R) have the most butterflies.
__host__ __device__ __forceinline__ int local_passes(int logm, int lrm) { return (logm + lrm - 1) / lrm; }
__host__ __device__ __forceinline__ int local_pass_lr(int logm, int lrm, int idx, bool inverse) {
    const int np = local_passes(logm, lrm);
    return idx == (inverse ? np - 1 : 0) ? logm - (np - 1) * lrm : lrm;
}

// All state of one CTA's solve.  Every member function is force-inlined into
// the kernel, so the members stay in registers (no closure objects, no stack).
template <typename T, int S, int C, int LRM> struct LineSolver {
    static constexpr int NSYM = S * (S + 1) / 2;
    static constexpr int NV = NAcc<S>::value;

    const LineJob<T>* J; // shared-memory copy of the job
    RedSmem* rs;
    cx<T>* bufA;
    cx<T>* bufB;
    cx<T>* cur; // holds psi between steps
    const Tab<T>* twm; // local-pass twiddles of the forward schedule, pass by pass (see the staging in the kernel)
    const Tab<T>* twi; // ... of the inverse schedule (twm when the two schedules are the same)
    const Tab<T>* twp; // the current pass's table: W at [(r - 1) p + kk]
    const Tab<T>* twc;
    const Tab<T>* Rs;
    int rstride; // component stride of Rs: m when staged in shared memory, n when read from global
    const Tab<T>* eks;
    const double* capw; // this CTA's slice of the global tables
    const double* Ug; // the eigenvectors of the CTA's points: component e of point j at Ug[e * ustride + j]
    int ustride;
    const double* Vg;
    const cx<T>* psi0;
    int m, n, logm, q, ldp, cta;
    size_t base;
    double lo, span, dr, dk, dkunit, mass;
    T inv_n;
    bool prop;     // propagation step (true) or momentum-observation round trip (false)
    bool fuse_obs; // accumulate the position-space observables in the last inverse pass
    ObsFlags f;
    Acc acc[NV];
    double pop_abs[S];

    // ---------------------------------------------------------------- hooks
    // forward, first pass: accumAbsorbed before the first applyR, then R
    template <int R> __device__ __forceinline__ void fwd_first(int i, int mr, cx<T> (&v)[S][R]) {
        if (!prop) return;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int j = i + r * mr;
            cx<T> x[S];
#pragma unroll
            for (int s = 0; s < S; ++s) x[s] = v[s][r];
            if (f.track) absorbed_point<T, S>(acc, x, capw[j], Ug, ustride, j, f.adia);
            apply_r_point<T, S>(x, Rs, rstride, j);
#pragma unroll
            for (int s = 0; s < S; ++s) v[s][r] = x[s];
        }
    }
    // forward, last pass: cluster twiddle (C > 1) or, for C = 1, kinetic phase / k-space observables
    template <int R> __device__ __forceinline__ void fwd_last(int o0, int p, cx<T> (&v)[S][R]) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = o0 + r * p;
            if constexpr (C > 1) {
                if (cta > 0) {
                    const Tab<T> w = twc[k];
#pragma unroll
                    for (int s = 0; s < S; ++s) v[s][r] = tmul<-1>(v[s][r], w);
                }
            } else if (prop) {
                const Tab<T> w = eks[k];
#pragma unroll
                for (int s = 0; s < S; ++s) v[s][r] = tmul<-1>(v[s][r], w);
            } else {
                cx<T> z[S];
#pragma unroll
                for (int s = 0; s < S; ++s) z[s] = v[s][r];
                observe_k<T, S>(acc, z, k, n, dkunit, mass, f);
            }
        }
    }
    // inverse, first pass (C > 1): gather the exchanged values from their owners
    template <int R> __device__ __forceinline__ void inv_first(int i, int mr, cx<T> (&v)[S][R], const cx<T>* xbuf) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k1 = i + r * mr, owner = k1 / q, u = k1 - owner * q;
            const cx<T>* src = remote<T>(xbuf, owner);
#pragma unroll
            for (int s = 0; s < S; ++s) v[s][r] = src[s * ldp + padx<T>(cta * q + u)];
            if (cta > 0) {
                const Tab<T> w = twc[k1];
#pragma unroll
                for (int s = 0; s < S; ++s) v[s][r] = tmul<1>(v[s][r], w);
            }
        }
    }
    // inverse, last pass: 1/N, accumAbsorbed, R and the observables of the step
    template <int R> __device__ __forceinline__ void inv_last(int o0, int p, cx<T> (&v)[S][R]) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int j = o0 + r * p;
            cx<T> x[S];
#pragma unroll
            for (int s = 0; s < S; ++s) x[s] = scale<T>(v[s][r], inv_n);
            if (prop) {
                if (f.track) absorbed_point<T, S>(acc, x, capw[j], Ug, ustride, j, f.adia);
                apply_r_point<T, S>(x, Rs, rstride, j);
                if (fuse_obs) observe_point<T, S>(acc, x, grid_r<C>(lo, span, n, cta, j), *J, base + j, f, Ug, ustride, j);
            }
#pragma unroll
            for (int s = 0; s < S; ++s) v[s][r] = x[s];
        }
    }

    // One radix-R Stockham pass over S lines of m points, `in` -> `out`.  Thread t
    // handles the butterflies i = t, t + nt, ... of every state, so all S states of
    // a grid point meet in one thread.  KIND selects the hooks of first/last passes.
    template <int R, int SIGN, int KIND>
    __device__ __forceinline__ void pass(const cx<T>* __restrict__ in, cx<T>* __restrict__ out, int p,
                                         const cx<T>* xbuf) {
        constexpr int LR = R == 2 ? 1 : R == 4 ? 2 : 3;
        const int logmr = logm - LR, mr = 1 << logmr, nt = blockDim.x;
        // passes whose hooks do not mix states take one (butterfly, state) pair per thread;
        // the forward first pass (R) and the inverse last pass (R, observables) take all
        // states of a butterfly in one thread
        constexpr bool SPLIT = S > 1 && !(KIND & FWD_FIRST) && !(KIND & INV_LAST);
        if constexpr (SPLIT) {
            for (int t = threadIdx.x; t < (S << logmr); t += nt) {
                const int s = t >> logmr, i = t & (mr - 1);
                cx<T> v[R];
                if constexpr ((KIND & INV_FIRST) && C > 1) {
#pragma unroll
                    for (int r = 0; r < R; ++r) { // inv_first for one state
                        const int k1 = i + r * mr, owner = k1 / q, u = k1 - owner * q;
                        v[r] = remote<T>(xbuf, owner)[s * ldp + padx<T>(cta * q + u)];
                        if (cta > 0) v[r] = tmul<1>(v[r], twc[k1]);
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r) v[r] = in[s * ldp + padx<T>(i + r * mr)];
                }
                const int kk = i & (p - 1);
                if (p > 1) {
#pragma unroll
                    for (int r = 1; r < R; ++r) v[r] = tmul<SIGN>(v[r], twp[(r - 1) * p + kk]);
                }
                dft<R, SIGN, T>(v);
                const int o0 = ((i - kk) << LR) + kk;
                if constexpr (KIND & FWD_LAST) {
#pragma unroll
                    for (int r = 0; r < R; ++r) { // fwd_last for one state
                        const int k = o0 + r * p;
                        if constexpr (C > 1) {
                            if (cta > 0) v[r] = tmul<-1>(v[r], twc[k]);
                        } else if (prop) {
                            v[r] = tmul<-1>(v[r], eks[k]);
                        } else {
                            observe_k1<T>(acc, v[r], k, n, dkunit, mass, f);
                        }
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r) out[s * ldp + padx<T>(o0 + r * p)] = v[r];
            }
            __syncthreads();
            return;
        }
        for (int i = threadIdx.x; i < mr; i += nt) {
            cx<T> v[S][R];
            if constexpr ((KIND & INV_FIRST) && C > 1) {
                inv_first<R>(i, mr, v, xbuf);
            } else {
#pragma unroll
                for (int s = 0; s < S; ++s)
#pragma unroll
                    for (int r = 0; r < R; ++r) v[s][r] = in[s * ldp + padx<T>(i + r * mr)];
            }
            if constexpr (KIND & FWD_FIRST) fwd_first<R>(i, mr, v);
            const int kk = i & (p - 1);
            if (p > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    const Tab<T> w = twp[(r - 1) * p + kk];
#pragma unroll
                    for (int s = 0; s < S; ++s) v[s][r] = tmul<SIGN>(v[s][r], w);
                }
            }
#pragma unroll
            for (int s = 0; s < S; ++s) dft<R, SIGN, T>(v[s]);
            const int o0 = ((i - kk) << LR) + kk;
            if constexpr (KIND & FWD_LAST) fwd_last<R>(o0, p, v);
            if constexpr (KIND & INV_LAST) inv_last<R>(o0, p, v);
            if constexpr (KIND & FUSE_NEXT) { // last pass: o0 = i, p = mr; the next step's first pass (p = 1)
                fwd_first<R>(i, mr, v);
#pragma unroll
                for (int s = 0; s < S; ++s) dft<R, -1, T>(v[s]);
#pragma unroll
                for (int s = 0; s < S; ++s)
#pragma unroll
                    for (int r = 0; r < R; ++r) out[s * ldp + padx<T>((i << LR) + r)] = v[s][r];
            } else {
#pragma unroll
                for (int s = 0; s < S; ++s)
#pragma unroll
                    for (int r = 0; r < R; ++r) out[s * ldp + padx<T>(o0 + r * p)] = v[s][r];
            }
        }
        __syncthreads();
    }

    // one local pass of radix R, its kind from its place in the schedule.  The remainder radix
    // (below 2^LRM) is only ever the forward's first or the inverse's last pass.
    template <int R, int SIGN>
    __device__ __forceinline__ void pass_at(bool first, bool last, bool fuse_next, cx<T>* in, cx<T>* out, int p,
                                            const cx<T>* xbuf) {
        constexpr int KF = SIGN < 0 ? FWD_FIRST : INV_FIRST, KL = SIGN < 0 ? FWD_LAST : INV_LAST;
        constexpr bool REM = R < (1 << LRM);
        if (first && last) {
            pass<R, SIGN, KF | KL>(in, out, p, xbuf);
        } else if constexpr (REM && SIGN < 0) {
            pass<R, SIGN, KF>(in, out, p, xbuf);
        } else if constexpr (REM && SIGN > 0) {
            if (fuse_next) pass<R, SIGN, KL | FUSE_NEXT>(in, out, p, xbuf);
            else pass<R, SIGN, KL>(in, out, p, xbuf);
        } else {
            if (first) pass<R, SIGN, KF>(in, out, p, xbuf);
            else if (!last) pass<R, SIGN, 0>(in, out, p, xbuf);
            else if constexpr (SIGN > 0) {
                if (fuse_next) pass<R, SIGN, KL | FUSE_NEXT>(in, out, p, xbuf);
                else pass<R, SIGN, KL>(in, out, p, xbuf);
            } else {
                pass<R, SIGN, KL>(in, out, p, xbuf);
            }
        }
    }

    // local m-point transform ping-ponging between a (input) and b; returns the result buffer.
    // start: passes already run (1: the first pass ran as part of the previous step's last pass);
    // fuse_next (inverse only): the last pass also runs the next step's forward first pass
    template <int SIGN>
    __device__ __forceinline__ cx<T>* local_fft(cx<T>* a, cx<T>* b, const cx<T>* xbuf, int start = 0,
                                                bool fuse_next = false) {
        const int np = local_passes(logm, LRM);
        const Tab<T>* tw = SIGN < 0 ? twm : twi;
        int p = 1, tbase = 0;
        cx<T>* in = a;
        cx<T>* out = b;
        for (int idx = 0; idx < np; ++idx) {
            const int LR = local_pass_lr(logm, LRM, idx, SIGN > 0);
            if (idx >= start) {
                const bool first = idx == 0, last = idx == np - 1;
                twp = tw + tbase;
                if (LR == 3) {
                    if constexpr (LRM == 3) pass_at<8, SIGN>(first, last, fuse_next, in, out, p, xbuf);
                } else if (LR == 2) {
                    pass_at<4, SIGN>(first, last, fuse_next, in, out, p, xbuf);
                } else {
                    pass_at<2, SIGN>(first, last, fuse_next, in, out, p, xbuf);
                }
                // the inverse's first pass read other CTAs' exchange buffers: none may be
                // overwritten before every CTA of the cluster has finished that gather.  The
                // gathered values were consumed (butterflies, stored locally) before the arrive,
                // so the barrier publishes nothing and its arrive can be relaxed (no fence)
                if (C > 1 && SIGN > 0 && first) cluster_barrier_relaxed();
                cx<T>* t = in;
                in = out;
                out = t;
            }
            tbase += ((1 << LR) - 1) * p;
            p <<= LR;
        }
        return in;
    }
    // the last inverse pass can take the next step's forward first pass: at least two passes
    __device__ __forceinline__ bool can_fuse_steps() const { return local_passes(logm, LRM) >= 2; }

    __device__ __forceinline__ cx<T>* other(const cx<T>* b) const { return b == bufA ? bufB : bufA; }

    // forward transform of cur (start = 1: its first pass already ran); returns the buffer the
    // inverse starts from
    __device__ __forceinline__ cx<T>* forward(int start = 0) {
        cx<T>* res = local_fft<-1>(cur, other(cur), nullptr, start);
        if constexpr (C > 1) { // C-point DFTs across the cluster, kinetic phase in between
            cx<T>* xb = other(res);
            cg::cluster_group cl = cg::this_cluster();
            cl.sync();
            // one (column u, state s) pair per thread: S times the threads of one column each
            for (int t = threadIdx.x; t < S * q; t += blockDim.x) {
                const int s = t / q, u = t - s * q;
                cx<T> w[C];
#pragma unroll
                for (int cc = 0; cc < C; ++cc) w[cc] = remote<T>(res, cc)[s * ldp + padx<T>(cta * q + u)];
                dft<C, -1, T>(w);
#pragma unroll
                for (int k2 = 0; k2 < C; ++k2) {
                    if (prop) w[k2] = tmul<-1>(w[k2], eks[k2 * q + u]);
                    else observe_k1<T>(acc, w[k2], cta * q + u + m * k2, n, dkunit, mass, f);
                }
                dft<C, 1, T>(w);
#pragma unroll
                for (int cc = 0; cc < C; ++cc) xb[s * ldp + padx<T>(cc * q + u)] = w[cc];
            }
            cl.sync();
            return xb;
        }
        return res;
    }
    // inverse transform (from forward's buffer) into cur; fuse_next: cur then holds the next step's
    // forward first pass instead of psi
    __device__ __forceinline__ void inverse(cx<T>* kb, bool fuse_next = false) {
        if constexpr (C > 1) cur = local_fft<1>(kb, other(kb), kb, 0, fuse_next); // first pass gathers remote kb
        else cur = local_fft<1>(kb, other(kb), nullptr, 0, fuse_next);
    }

    __device__ __forceinline__ void zero_acc() {
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = Acc();
    }
    // position-space observables of cur in a pass of their own
    __device__ __forceinline__ void observe_x() {
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            cx<T> x[S];
#pragma unroll
            for (int s = 0; s < S; ++s) x[s] = cur[s * ldp + padx<T>(j)];
            observe_point<T, S>(acc, x, grid_r<C>(lo, span, n, cta, j), *J, base + j, f, Ug, ustride, j);
        }
    }
    // momentum-space round trip (quantum_dynamics.zig:347-363): psi <- IFFT(FFT(psi)) as in the reference
    __device__ __forceinline__ void roundtrip() {
        prop = false;
        inverse(forward());
        prop = true;
    }
    __device__ __forceinline__ void set_flags(uint32_t mask) {
        f.pos = mask & WM_POS;
        f.mom = mask & WM_MOM;
        f.pop = mask & WM_POP;
        f.ekin = (mask & WM_EKIN) || (mask & WM_ETOT);
        f.epot = (mask & WM_EPOT) || (mask & WM_ETOT);
        f.norm = (mask & WM_NORM) || J->has_stop;
        f.acf = J->calc_acf != 0;
        f.adia = J->adiabatic != 0;
        f.track = J->track != 0;
    }
    // reduce the step's accumulators; the row is written by one thread of the cluster
    __device__ __forceinline__ double finish_row(double* dst) {
        // the values this step accumulated (the observe_* helpers add to no other slot)
        uint32_t act = (f.norm ? 1u << A_NORM : 0u) | (f.pos ? 1u << A_POS : 0u) | (f.epot ? 1u << A_EPOT : 0u) |
                       (f.acf ? 3u << A_ACFR : 0u) | (f.mom ? 1u << A_MOM : 0u) | (f.ekin ? 1u << A_EKIN : 0u);
        if (f.pop) act |= ((1u << S) - 1u) << A_POP;
        if (f.track) act |= ((1u << S) - 1u) << (A_POP + S);
        double out[NV];
        cluster_sum<NV, C>(acc, out, rs, act);
#pragma unroll
        for (int s = 0; s < S; ++s) pop_abs[s] += out[A_POP + S + s] * dr;
        const double norm = out[A_NORM] * dr;
        if (cta == 0 && threadIdx.x == 0) {
            constexpr RowLayout L{1, S};
            dst[L.norm()] = f.norm ? norm : nan("");
            dst[L.pos()] = f.pos ? out[A_POS] * dr : nan("");
            dst[L.epot()] = f.epot ? out[A_EPOT] * dr : nan("");
            dst[L.acf()] = f.acf ? out[A_ACFR] * dr : nan("");
            dst[L.acf() + 1] = f.acf ? out[A_ACFI] * dr : nan("");
            dst[L.mom()] = f.mom ? out[A_MOM] * dk : nan("");
            dst[L.ekin()] = f.ekin ? out[A_EKIN] * dk : nan("");
#pragma unroll
            for (int s = 0; s < S; ++s) dst[L.pop() + s] = f.pop ? out[A_POP + s] * dr + pop_abs[s] : nan("");
        }
        return norm;
    }
};

// system-scope release store / acquire load: the host polls and writes these words in pinned memory
__device__ __forceinline__ void st_release_sys(int* p, int v) {
    asm volatile("st.release.sys.global.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_acquire_sys(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.sys.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The solve of job J (already in shared memory) on this CTA / cluster.
template <typename T, int S, int C, int LRM>
__device__ __forceinline__ void line_solve_run(LineJob<T>& J, RedSmem& rs, unsigned char* smem_raw, int cta) {
    using Solver = LineSolver<T, S, C, LRM>;
    constexpr int NSYM = Solver::NSYM;

    Solver X;
    X.J = &J;
    X.rs = &rs;
    X.m = J.m;
    X.n = J.n;
    X.logm = J.logm;
    X.q = J.q;
    X.ldp = padded_len<T>(J.m);
    X.cta = cta;
    X.base = (size_t)cta * J.m;
    X.lo = J.lo;
    X.span = J.hi - J.lo;
    X.dr = J.dr;
    X.dk = J.dk;
    X.dkunit = 6.283185307179586476925286766559 / X.span;
    X.mass = J.mass;
    X.inv_n = (T)(1.0 / (double)J.n);
    X.bufA = reinterpret_cast<cx<T>*>(smem_raw);
    X.bufB = X.bufA + S * X.ldp;
    Tab<T>* twm = reinterpret_cast<Tab<T>*>(X.bufB + S * X.ldp);
    const bool two = line_two_schedules(X.m, LRM);
    Tab<T>* twi = two ? twm + X.m : twm;
    Tab<T>* twc = twi + X.m;
    Tab<T>* Rs = J.r_global ? J.R + X.base : twc + (C > 1 ? X.m : 0);
    Tab<T>* eks = twc + (C > 1 ? X.m : 0) + (J.r_global ? 0 : NSYM * X.m);
    X.twm = twm;
    X.twi = twi;
    X.twc = twc;
    X.Rs = Rs;
    X.rstride = J.r_global ? J.n : J.m;
    X.eks = eks;
    X.capw = J.capw ? J.capw + X.base : nullptr;
    X.Ug = J.U ? J.U + X.base : nullptr;
    X.ustride = J.n;
    X.Vg = J.V + X.base;
    X.psi0 = J.psi0 ? J.psi0 + X.base : nullptr;
    X.cur = X.bufA;
    X.prop = true;
    X.fuse_obs = false;
#pragma unroll
    for (int s = 0; s < S; ++s) X.pop_abs[s] = 0;

    // stage the time-independent tables
    const int m = X.m, n = X.n;
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
        if (C > 1) twc[t] = J.tw[cta * t];
        eks[t] = J.expk[X.base + t];
    }
    // Twiddles of the local passes in pass order (the radix schedule of local_fft): the pass
    // of span p and radix R holds W_m^(r kk m/(p R)) = exp(-2 pi i r kk / (p R)) at
    // [(r - 1) p + kk], r = 1..R-1, kk < p.  A warp's twiddle reads are then contiguous
    // (reading W_m^t at stride m/(p R) put up to 16 of them in the same banks); the tables
    // take sum (R - 1) p = m - 1 entries.
    for (int dir = 0; dir < (two ? 2 : 1); ++dir) {
        Tab<T>* tw = dir ? twi : twm;
        int p = 1, logp = 0, tbase = 0;
        for (int idx = 0; idx < local_passes(X.logm, LRM); ++idx) {
            const int LR = local_pass_lr(X.logm, LRM, idx, dir == 1), R = 1 << LR, tshift = X.logm - logp - LR;
            for (int e = threadIdx.x; e < (R - 1) * p; e += blockDim.x) {
                const int r = e / p + 1, kk = e - (r - 1) * p;
                tw[tbase + e] = J.tw[((r * kk) << tshift) * C];
            }
            tbase += (R - 1) * p;
            p <<= LR;
            logp += LR;
        }
    }
    if (!J.r_global)
        for (int e = threadIdx.x; e < NSYM * m; e += blockDim.x) {
            const int c = e / m, j = e - c * m;
            Rs[e] = J.R[(size_t)c * n + X.base + j];
        }
    // the eigenvectors (adiabatic populations, absorbed populations) after the tables, where the
    // shape reserved room for them and they do not change during the solve
    if (J.u_smem && J.U && !J.td) {
        double* Us = reinterpret_cast<double*>(eks + m);
        for (int e = threadIdx.x; e < S * S * m; e += blockDim.x) {
            const int c = e / m, j = e - c * m;
            Us[e] = J.U[(size_t)c * n + X.base + j];
        }
        X.Ug = Us;
        X.ustride = m;
    }
    __syncthreads();

    LineCtx<T> ctx{&J, X.cur, nullptr, &rs, m, n, X.logm, X.q, X.ldp, cta, X.base};
    auto spare_of = [&](cx<T>* c) { return c == X.bufA ? X.bufB : X.bufA; };
    if (J.i0 == 0) {
        line_initial_state<T, S, C>(ctx, X.lo, X.span);
    } else { // resume: the wavefunction and the absorbed populations of the previous launch
        for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
            const int s = e / m, j = e - s * m;
            X.cur[s * X.ldp + padx<T>(j)] = J.psi_save[(size_t)s * n + X.base + j];
        }
#pragma unroll
        for (int s = 0; s < S; ++s) X.pop_abs[s] = J.carry[s];
        __syncthreads();
    }
    constexpr int HC = RowLayout{1, S}.width();
    const int iters = J.iters;
    int rows = J.i1 + 1;
    bool ended = J.i1 >= iters;
    // Step i's last inverse pass also runs step i+1's forward first pass (the applyR that ends step
    // i and the one that begins step i+1 act on the same grid points, quantum_dynamics.zig:417-427)
    // wherever nothing needs the end-of-step wavefunction in between: no momentum round trip, no
    // wavefunction history, no stop test, no absorbed-population tracking (its sums belong to the
    // next row), no imaginary time or time-dependent update, and not the launch's last step.
    const bool fusable = X.can_fuse_steps() && !J.itp && !J.td && !J.wfn_hist && !J.has_stop && !J.track;
    bool pre = false; // cur holds step i's forward first pass (run by step i-1's last pass)
    for (int i = J.i0; i <= J.i1; ++i) {
        const bool logstep = J.log && ((i % J.log_interval == 0) || (i == iters));
        X.set_flags(J.wmask | (logstep ? (uint32_t)WM_ALL_OBS : 0u));
        X.zero_acc();
        X.fuse_obs = i > 0 && !J.itp && !J.td;
        if (i > 0) { // Propagator.step (quantum_dynamics.zig:417-427)
            if (J.td) {
                ctx.spare = spare_of(X.cur);
                line_ham_update<T, S, C>(ctx, ((double)i - 0.5) * J.tstep, true, Rs, X.rstride, X.lo, X.span);
            }
            X.prop = true;
            const bool fuse = fusable && i < J.i1 && !(X.f.mom || X.f.ekin);
            X.inverse(X.forward(pre ? 1 : 0), fuse);
            pre = fuse;
            ctx.psi = X.cur;
        }
        if (J.itp) { // quantum_dynamics.zig:898-906
            line_orthogonalize<T, S, C>(ctx);
            line_normalize<T, S, C>(ctx);
        }
        if (J.td) {
            ctx.spare = spare_of(X.cur);
            line_ham_update<T, S, C>(ctx, (double)i * J.tstep, false, Rs, X.rstride, X.lo, X.span);
        }
        if (!X.fuse_obs) X.observe_x();
        if (X.f.mom || X.f.ekin) {
            X.roundtrip();
            ctx.psi = X.cur;
        }
        const double nrm = X.finish_row(J.hist + (size_t)i * HC);
        if (J.progress && cta == 0 && threadIdx.x == 0) { // row i is in memory: publish it to the host
            __threadfence_system();
            st_release_sys(J.progress, i + 1);
        }
        if (J.wfn_hist) { // History.append of the wavefunction (quantum_dynamics.zig:176-180), toAdia first (:919-927)
            cx<T>* __restrict__ dst = J.wfn_hist + (size_t)i * S * n;
            for (int j = threadIdx.x; j < m; j += blockDim.x) {
                cx<T> x[S];
#pragma unroll
                for (int s = 0; s < S; ++s) x[s] = X.cur[s * X.ldp + padx<T>(j)];
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    cx<T> y = x[s];
                    if (J.adiabatic && S > 1) {
                        double re = 0, im = 0;
#pragma unroll
                        for (int k = 0; k < S; ++k) {
                            const double u = J.U[(size_t)(k * S + s) * n + X.base + j];
                            re += (double)x[k].x * u;
                            im += (double)x[k].y * u;
                        }
                        y = mk<T>((T)re, (T)im);
                    }
                    dst[(size_t)s * n + X.base + j] = y;
                }
            }
            __syncthreads(); // the next step's passes overwrite the buffers read here
        }
        if (J.has_stop && nrm < J.stop_norm) { // stop_norm (quantum_dynamics.zig:933-944)
            rows = i + 1;
            ended = true;
            break;
        }
    }
    if (ended) { // final Observables.init(..., log = true) (quantum_dynamics.zig:949)
        X.set_flags(WM_ALL_OBS);
        X.zero_acc();
        X.observe_x();
        X.roundtrip();
        X.finish_row(J.fin);
    } else if (cta == 0 && threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < S; ++s) J.carry[s] = X.pop_abs[s];
    }
    if (cta == 0 && threadIdx.x == 0) {
        *J.rows = rows;
        if (J.done) *J.done = ended ? 1 : 0;
    }
    for (int e = threadIdx.x; e < S * m; e += blockDim.x) {
        const int s = e / m, j = e - s * m;
        J.psi_save[(size_t)s * n + X.base + j] = X.cur[s * X.ldp + padx<T>(j)];
    }
    if constexpr (C > 1) cg::this_cluster().sync(); // keep shared memory alive for remote readers
}

// One cluster of C CTAs per job of the array: a group of jobs in one launch.
// MAXT: the CTA size the kernel is compiled for (LineMaxThreads by default; FP32 launches of at
// most 256 threads per CTA take a 256-thread form, which leaves a thread 255 registers instead of 128)
template <typename T, int S, int C, int LRM, int MAXT = LineMaxThreads<T>::value>
__global__ void __launch_bounds__(MAXT, 1) line_solve_kernel(const LineJob<T>* __restrict__ jobs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ LineJob<T> J;
    __shared__ RedSmem rs;
    const int cta = (C > 1) ? (int)cg::this_cluster().block_rank() : 0;
    if (threadIdx.x == 0) {
        J = jobs[blockIdx.x / C];
        rs.slot_idx = 0;
    }
    __syncthreads();
    line_solve_run<T, S, C, LRM>(J, rs, smem_raw, cta);
}

// ------------------------------------------------------------ the persistent service kernel
// Words the host writes and the device reads, in pinned host memory.
struct LineServiceCtl {
    unsigned tail;   // jobs posted so far (slot k % capacity holds job k)
    unsigned closed; // exit once every posted job has been claimed
};
template <typename T> struct LineService {
    const LineJob<T>* jobs; // [capacity] descriptors, pinned host memory
    const LineServiceCtl* ctl;
    int* done;              // [capacity] pinned host memory: 1 once job k's solve has ended
    unsigned* counters;     // device memory: [0] jobs claimed so far, [1] CTAs that left idle
    unsigned capacity;
    long long idle_cycles;  // clock64 budget of one idle wait for work
};

// Persistent CTAs working through a job table the host keeps appending to (continuous batching
// of single-CTA 1-D jobs of uneven sizes): a CTA claims the next posted job, runs its whole solve
// with the wavefunction resident in shared memory, publishes each history row and the end of the
// solve to the host, and claims the next.  A CTA that finds no work waits at most idle_cycles
// (clock64) and then exits; the host relaunches when it posts work to a kernel that has ended.
template <typename T, int S, int LRM>
__global__ void __launch_bounds__(LineMaxThreads<T>::value, 1) line_service_kernel(LineService<T> svc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ LineJob<T> J;
    __shared__ RedSmem rs;
    __shared__ long long claimed;
    for (;;) {
        if (threadIdx.x == 0) {
            claimed = -1;
            const long long t0 = clock64();
            for (;;) {
                const unsigned tail = ld_acquire_sys(&svc.ctl->tail);
                const unsigned c = atomicAdd(&svc.counters[0], 0u);
                if (c < tail) {
                    if (atomicCAS(&svc.counters[0], c, c + 1) == c) {
                        claimed = c;
                        break;
                    }
                    continue;
                }
                if (ld_acquire_sys(&svc.ctl->closed)) break;
                if (clock64() - t0 > svc.idle_cycles) { // bounded: nothing posted within the budget
                    atomicAdd(&svc.counters[1], 1u);
                    break;
                }
                __nanosleep(1000);
            }
            if (claimed >= 0) {
                J = svc.jobs[(unsigned)claimed % svc.capacity];
                rs.slot_idx = 0;
            }
        }
        __syncthreads();
        if (claimed < 0) return;
        line_solve_run<T, S, 1, LRM>(J, rs, smem_raw, 0);
        __syncthreads(); // every thread's results are written
        if (threadIdx.x == 0) {
            __threadfence_system();
            st_release_sys(&svc.done[(unsigned)claimed % svc.capacity], 1);
        }
        __syncthreads(); // J and claimed are rewritten by the next claim
    }
}

} // namespace zqd
