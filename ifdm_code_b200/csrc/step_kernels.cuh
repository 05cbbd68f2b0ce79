// step_kernels.cuh -- the fused passes of one leap-frog step (sm_100a).
//
// One step of the reference (src/CosmoBEC_MPI.cpp:218-219 then :121-159) is
//   poisson; timestep; kick/2; FFT; drift; iFFT; poisson; kick/2
// Here the two half kicks that meet between consecutive steps are merged
// (same phi, same |psi| -- the kick only rotates phases), the Poisson solve
// before the timestep reuses the one at the end of the previous step, and
// every elementwise operation rides inside an FFT axis pass.  Per step:
//
//   T  timestep   device quadrature, merged kick coefficients, drift tables
//   P1 z-pass     load psi + phi, kick, forward FFT along z
//   P2 y-pass     forward FFT along y
//   P3 x-pass     forward FFT along x, drift, inverse FFT along x
//   P4 y-pass     inverse FFT along y
//   P5 z-pass     inverse FFT along z -> psi; rho = |psi|^2 - mu; max|psi|^2;
//                 real-to-half-complex FFT of rho along z
//   P6 y-pass     forward FFT along y (half spectrum)
//   P7 x-pass     forward FFT along x, phi_k = -rho_k / kappa^2, inverse FFT
//   P8 y-pass     inverse FFT along y (half spectrum)
//   P9 z-pass     half-complex-to-real FFT along z, /N^3 -> phi; max|phi|
//
// Units: psi is stored as psi/S with S^2 = rho_c / m_solar, so |psi_s|^2 is
// the density in units of the mean (this keeps FP32 in range: |psi| ~ 1e50
// in the reference's units).  phi is stored as phi/Phi0 with
// Phi0 = 4 pi G m_solar S^2 (xmax/pi)^2, so the Poisson multiplier is
// -1/kappa^2 with integer kappa.  All scale factors are FP64 and folded into
// the coefficients the timestep kernel writes.
#pragma once

#include "fft_engine.cuh"

#include <type_traits>
#include "state_types.hpp"

namespace ifdm {

// ------------------------------------------------------------ tile config --
// R: element type in HBM, K: arithmetic type in registers and shared memory.
// (double, double) is the FP64 drop-in, (float, float) FP32, and
// (float, double) the mixed mode: FP32 traffic, FP64 butterflies.
// ZR: tiles of whole contiguous rows (z passes), which coalesce whatever the
// line count, so L only has to fill a shared-memory phase; strided lines (y/x
// passes) take enough lines for 128-byte segments.
template <typename R, typename K, int N, bool ZR = false> struct Tile {
    using G = cx<R>;
    using C = cx<K>;
    static constexpr int GB = (int)sizeof(G);
    static constexpr int PH = sizeof(C) == 16 ? 8 : 16;            // threads per smem phase
    static constexpr int LC = ZR ? 1 : 128 / GB;                    // lines for 128-byte rows
    // elements per thread: the plan's, doubled for mixed y/x lines at N >= 256
    // and for every tile at N >= 1024 (the lines of a 1024-point tile would
    // otherwise need more than 1024 threads)
    static constexpr int E0 = Plan<N>::E * ((!ZR && sizeof(C) == 16 && GB == 8 && N >= 256) ? 2 : 1) *
                              (N >= 1024 ? 2 : 1);
    static constexpr int T = N / E0;                                // threads per line
    static constexpr int LT = 256 / T;                              // lines for >= 256 threads
    static constexpr int L1 = LT > LC ? LT : LC;
    static constexpr int L = L1 > PH ? L1 : PH;                     // lines per tile
    static constexpr int E = E0;
    static constexpr int LP = L + 1;
    static constexpr int NT = L * T;                                // threads per block
    // half-length lines: the real-to-complex transform of P5 runs the radix-4
    // plan in FP32 (measured at 512^3: P5 1.10 -> 1.02 ms; slower in FP64 and
    // mixed, and for the complex-to-real P9), everything else the default plan
    using HP = std::conditional_t<sizeof(C) == 8, HalfPlan<N / 2>, Plan<N / 2>>;
    static constexpr int EH = elems_for<N / 2, T, HP>(0);
    static constexpr int EHD = elems_for<N / 2, T>(0);
    static constexpr size_t SMEM = size_t(N) * LP * sizeof(C);
    static constexpr size_t SMEM9 = size_t(N + 1) * LP * sizeof(C);
    static_assert(N / E0 * E0 == N, "E must divide N");
    static_assert((N / 2) / EH <= T && (N / 2) / EHD <= T, "half-length lines must fit the block");
};
template <typename R, typename K, int N> using TileZ = Tile<R, K, N, true>;

// r2c / c2r post-twiddle: w^k * a (DIR -1) or conj(w^k) * a (DIR +1), table of length TN
template <int DIR, int TN, typename C> __device__ __forceinline__ C post_tw(const C *__restrict__ tw, int k, C a) {
    if constexpr (sizeof(C) == 16) return DIR < 0 ? cmul(__ldg(tw + k), a) : cmul(cconj(__ldg(tw + k)), a);
    else return twmul<DIR, TN>(a, tw, k);
}

// Half-spectrum row pitch: N/2+1 rounded up so rows start on 128-byte lines.
template <typename R> __host__ __device__ constexpr int half_pitch(int n) {
    return sizeof(R) == 8 ? ((n / 2 + 1 + 7) / 8) * 8 : ((n / 2 + 1 + 15) / 16) * 16;
}

__host__ __device__ constexpr int kappa(int i, int n) { return i < n / 2 ? i : i - n; }

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *addr, double v) {
    // non-negative IEEE doubles order like their bit patterns
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

template <typename R> __device__ __forceinline__ R warp_max(R v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ------------------------------------------------------- storage rounding --
// Mixed mode rounds FP64 results to FP32 stochastically: the magnitude is
// rounded up with probability equal to the discarded fraction of an ulp.
// Consecutive steps see nearly the same data, so round-to-nearest would
// repeat the same errors every step and let them add up linearly; stochastic
// rounding makes them independent (unbiased, growing like sqrt(steps)).
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ float sr_to_float(double v, uint32_t r) {
    long long b = __double_as_longlong(v);
    b += (long long)(r >> 3);        // 29 random bits below float precision
    b &= ~((1ll << 29) - 1);
    return __double2float_rz(__longlong_as_double(b));
}
// salt: per step and pass; idx: element index
__device__ __forceinline__ uint32_t sr_key(uint32_t salt, size_t idx) {
    return mix32(salt ^ (uint32_t)idx ^ mix32((uint32_t)(idx >> 32) + 0x9e3779b9u));
}
template <typename R, typename K> struct Cvt {
    __device__ __forceinline__ static cx<R> out(cx<K> v, uint32_t, size_t) { return v; }
    __device__ __forceinline__ static R outr(K v, uint32_t, size_t) { return v; }
};
template <> struct Cvt<float, double> {
    __device__ __forceinline__ static float2 out(double2 v, uint32_t salt, size_t idx) {
        const uint32_t k = sr_key(salt, idx);
        return make_float2(sr_to_float(v.x, k), sr_to_float(v.y, mix32(k ^ 0x5bd1e995u)));
    }
    __device__ __forceinline__ static float outr(double v, uint32_t salt, size_t idx) {
        return sr_to_float(v, sr_key(salt, idx));
    }
};
template <typename K, typename G> __device__ __forceinline__ cx<K> cin(G g) {
    return mkc((K)g.x, (K)g.y);
}
__device__ __forceinline__ uint32_t pass_salt(const TState *ts, int pass) {
    return mix32((uint32_t)ts->steps * 16u + (uint32_t)pass);
}

// Deterministic block sum of three doubles; thread 0 writes out[0..2].
__device__ __forceinline__ void block_sum3(double a, double b, double c, double *out) {
    __shared__ double red[3][32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = a; red[1][w] = b; red[2][w] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0, s2 = 0;
        for (int i = 0; i < nw; ++i) { s0 += red[0][i]; s1 += red[1][i]; s2 += red[2][i]; }
        out[0] = s0; out[1] = s1; out[2] = s2;
    }
}

// exp(-i p) for the kick; FP32 reduces the FP64 argument mod 2 pi first.
template <typename R> __device__ __forceinline__ cx<R> expmi(double p);
template <> __device__ __forceinline__ double2 expmi<double>(double p) {
    double s, c;
    sincos(p, &s, &c);
    return mkc(c, -s);
}
template <> __device__ __forceinline__ float2 expmi<float>(double p) {
    const double twopi = 6.283185307179586476925286766559;
    const double pr = p - twopi * rint(p * (1.0 / twopi));
    float s, c;
    sincosf((float)pr, &s, &c);
    // put the pair back on the unit circle (first-order Newton step for
    // 1/sqrt(c^2 + s^2)): the kick must not change |psi|, and a modulus error
    // with a sign preference would change the norm by the same amount every
    // step instead of averaging out
    const float f = fmaf(-0.5f, fmaf(c, c, fmaf(s, s, -1.0f)), 1.0f);
    return mkc(c * f, -s * f);
}

// ------------------------------------------------------------- z-passes ---
// Tiles of L consecutive rows (row r = x*N + y), row pitch N, contiguous.

template <typename R, typename K, int N, int DIR>
__global__ void __launch_bounds__(TileZ<R, K, N>::NT)
    k_fft_z(cx<R> *__restrict__ data, const cx<K> *__restrict__ tw, uint32_t salt) {
    using TL = TileZ<R, K, N>;
    using C = typename TL::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sm = reinterpret_cast<C *>(smraw);
    const size_t base = size_t(blockIdx.x) * TL::L * N;
    for (int f = threadIdx.x; f < TL::L * N; f += TL::NT) sm[(f % N) * TL::LP + f / N] = cin<K>(data[base + f]);
    __syncthreads();
    fft_tile<C, N, TL::E, DIR, TL::L, TL::LP>(sm, tw);
    for (int f = threadIdx.x; f < TL::L * N; f += TL::NT)
        data[base + f] = Cvt<R, K>::out(sm[(f % N) * TL::LP + f / N], salt, base + f);
}

// P1: kick with the merged coefficients, remove the offset c, forward FFT along z.
template <typename R, typename K, int N>
__global__ void __launch_bounds__(TileZ<R, K, N>::NT)
    k_kick_fft_z(cx<R> *__restrict__ psi, const R *__restrict__ phi, const TState *__restrict__ ts,
                 const cx<K> *__restrict__ tw) {
    using TL = TileZ<R, K, N>;
    using C = typename TL::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sm = reinterpret_cast<C *>(smraw);
    const double cp = ts->coefP, cq = ts->coefQ, alpha = ts->alpha;
    const C c0 = mkc((K)ts->cre, (K)ts->cim);
    const uint32_t salt = pass_salt(ts, 1);
    const size_t base = size_t(blockIdx.x) * TL::L * N;
    if constexpr (sizeof(typename TL::G) != sizeof(C)) {
        // mixed: all of this thread's loads first (PER of psi and of phi in
        // flight), then the kicks (measured at 512^3: 1.42 -> 1.19 ms; in FP64
        // and FP32 the extra registers cost a resident block and it was slower,
        // and so were loading the whole psi and phi tile into shared memory
        // with cp.async first (FP32 0.77 -> 0.83 ms, FP64 1.45 -> 1.53 ms) and
        // unrolling the FP32 loop by two under a 32-register cap (0.76 -> 0.81 ms))
        constexpr int PER = TL::L * N / TL::NT;
        static_assert(PER * TL::NT == TL::L * N, "whole rows per thread block");
        typename TL::G g[PER];
        R ph[PER];
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            g[i] = psi[base + threadIdx.x + i * TL::NT];
            ph[i] = phi[base + threadIdx.x + i * TL::NT];
        }
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int f = threadIdx.x + i * TL::NT;
            const C v = cin<K>(g[i]);
            const double p = cp * (double)ph[i] + cq * (double)cnorm2(v) + alpha;
            sm[(f % N) * TL::LP + f / N] = cmul(v, expmi<K>(p)) - c0;
        }
    } else {
        for (int f = threadIdx.x; f < TL::L * N; f += TL::NT) {
            const C v = cin<K>(psi[base + f]);
            const double p = cp * (double)phi[base + f] + cq * (double)cnorm2(v) + alpha;
            sm[(f % N) * TL::LP + f / N] = cmul(v, expmi<K>(p)) - c0;
        }
    }
    __syncthreads();
    fft_tile<C, N, TL::E, -1, TL::L, TL::LP>(sm, tw);
    for (int f = threadIdx.x; f < TL::L * N; f += TL::NT)
        psi[base + f] = Cvt<R, K>::out(sm[(f % N) * TL::LP + f / N], salt, base + f);
}

// P5 (DO_IFFT) / initial density (no IFFT): psi = IFFT + c, rho = |psi|^2 - mu,
// max |psi|^2, real-to-half-complex FFT of rho along z into rhok (pitch NHP).
// The initial pass (no IFFT) also writes per-block partial sums of psi and
// |psi|^2 to `part` (3 doubles per block) for the offset c and the mean mu.
template <typename R, typename K, int N, bool DO_IFFT>
__global__ void __launch_bounds__(TileZ<R, K, N>::NT)
    k_density_r2c_z(cx<R> *__restrict__ psi, cx<R> *__restrict__ rhok, TState *__restrict__ ts,
                    double *__restrict__ part, const cx<K> *__restrict__ tw, const cx<K> *__restrict__ twh) {
    using TL = TileZ<R, K, N>;
    using C = typename TL::C;
    constexpr int NH = N / 2 + 1;
    constexpr int NHP = half_pitch<R>(N);
    constexpr int M = N / 2;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sm = reinterpret_cast<C *>(smraw);
    const size_t row0 = size_t(blockIdx.x) * TL::L;
    const size_t base = row0 * N;
    const uint32_t salt = pass_salt(ts, 5), salt2 = pass_salt(ts, 10);
    if (DO_IFFT) {
        typename TL::G g[TL::E];  // all of this thread's loads first
#pragma unroll
        for (int i = 0; i < TL::E; ++i) g[i] = psi[base + threadIdx.x + i * TL::NT];
#pragma unroll
        for (int i = 0; i < TL::E; ++i) {
            const int f = threadIdx.x + i * TL::NT;
            sm[(f % N) * TL::LP + f / N] = cin<K>(g[i]);
        }
        __syncthreads();
        fft_tile<C, N, TL::E, +1, TL::L, TL::LP>(sm, tw);
    }
    // rho values: thread keeps its E elements (fixed stride NT over the tile)
    K rho[TL::E];
    double mx = 0.0;
    const double mu = DO_IFFT ? ts->mu : 0.0;
    const C c0 = DO_IFFT ? mkc((K)ts->cre, (K)ts->cim) : mkc(K(0), K(0));
    double sre = 0.0, sim = 0.0, sn2 = 0.0;
#pragma unroll
    for (int i = 0; i < TL::E; ++i) {
        const int f = threadIdx.x + i * TL::NT;
        C v;
        if (DO_IFFT) {
            const typename TL::G g = Cvt<R, K>::out(sm[(f % N) * TL::LP + f / N] + c0, salt, base + f);
            psi[base + f] = g;
            v = cin<K>(g);  // the stored value defines the density
        } else {
            v = cin<K>(psi[base + f]);
            sre += (double)v.x;
            sim += (double)v.y;
        }
        const double n2 = (double)cnorm2(v);
        sn2 += n2;
        mx = fmax(mx, n2);
        rho[i] = (K)(n2 - mu);
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&ts->maxrho_bits, mx);
    if (!DO_IFFT) block_sum3(sre, sim, sn2, part + 3 * blockIdx.x);
    __syncthreads();
    // pack z_m = rho_{2m} + i rho_{2m+1} into the half tile (rows m < N/2)
    K *smr = reinterpret_cast<K *>(sm);
#pragma unroll
    for (int i = 0; i < TL::E; ++i) {
        const int f = threadIdx.x + i * TL::NT;
        const int l = f / N, n = f % N;
        smr[2 * ((n >> 1) * TL::LP + l) + (n & 1)] = rho[i];
    }
    __syncthreads();
    fft_tile<C, M, TL::EH, -1, TL::L, TL::LP, typename TL::HP>(sm, twh);
    // X_k = (Z_k + conj Z_{M-k})/2 - i w^k (Z_k - conj Z_{M-k})/2, k = 0..M
    constexpr int TPR = TL::NT / TL::L;  // threads per row: no division by N/2+1
    static_assert(TPR * TL::L == TL::NT, "whole rows per thread block");
    const int l = threadIdx.x / TPR;
    for (int k = threadIdx.x % TPR; k < NH; k += TPR) {
        const C zk = sm[(k % M) * TL::LP + l];
        const C zc = cconj(sm[((M - k) % M) * TL::LP + l]);
        const C e = cscale(zk + zc, K(0.5));
        const C o = cscale(zk - zc, K(0.5));
        const C wo = post_tw<-1, N>(tw, k % N, o);  // X = e - i w o
        const size_t gi = (row0 + l) * NHP + k;
        rhok[gi] = Cvt<R, K>::out(mkc(e.x + wo.y, e.y - wo.x), salt2, gi);
    }
}

// P9: half-complex-to-real FFT along z, scale by 1/N^3, store phi, max|phi|
// over the reference's scan window (rows below win_rows, plus win_tail
// elements of row win_rows; see the timestep kernel).
template <typename R, typename K, int N>
__global__ void __launch_bounds__(TileZ<R, K, N>::NT)
    k_c2r_z_phi(const cx<R> *__restrict__ rhok, R *__restrict__ phi, TState *__restrict__ ts, long win_rows,
                int win_tail, const cx<K> *__restrict__ tw, const cx<K> *__restrict__ twh) {
    using TL = TileZ<R, K, N>;
    using C = typename TL::C;
    constexpr int NHP = half_pitch<R>(N);
    constexpr int M = N / 2;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sm = reinterpret_cast<C *>(smraw);
    C *xs = sm + M * TL::LP;  // X_k rows k = 0..M staged after the Z tile
    const size_t row0 = size_t(blockIdx.x) * TL::L;
    const uint32_t salt = pass_salt(ts, 9);
    // all of this thread's loads first, then the shared-memory stores; TPR
    // threads per row, so no division by N/2+1
    constexpr int TPR = TL::NT / TL::L;
    static_assert(TPR * TL::L == TL::NT, "whole rows per thread block");
    constexpr int PER = (M + 1 + TPR - 1) / TPR;
    const int l = threadIdx.x / TPR, k0 = threadIdx.x % TPR;
    typename TL::G g[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i)
        if (k0 + i * TPR <= M) g[i] = rhok[(row0 + l) * NHP + k0 + i * TPR];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int k = k0 + i * TPR;
        if (k <= M) {
            C x = cin<K>(g[i]);
            if (k == 0 || k == M) x.y = K(0);  // c2r ignores these imaginary parts
            xs[k * TL::LP + l] = x;
        }
    }
    __syncthreads();
    // Z'_k = (X_k + conj X_{M-k}) + i conj(w^k) (X_k - conj X_{M-k}), k < M
    for (int f = threadIdx.x; f < TL::L * M; f += TL::NT) {
        const int l = f % TL::L, k = f / TL::L;
        const C xk = xs[k * TL::LP + l];
        const C xc = cconj(xs[(M - k) * TL::LP + l]);
        const C e = xk + xc;
        const C d = post_tw<+1, N>(tw, k, xk - xc);
        sm[k * TL::LP + l] = mkc(e.x - d.y, e.y + d.x);
    }
    __syncthreads();
    fft_tile<C, M, TL::EHD, +1, TL::L, TL::LP>(sm, twh);
    const K *smr = reinterpret_cast<const K *>(sm);
    constexpr KSplit<K> inv(1.0 / ((double)N * N * N));
    R *out = phi + row0 * N;
    // max|phi| over the reference's scan window: element f of the tile is in
    // it when (row0 + f / N) * N + f % N < win_rows * N + win_tail, one
    // comparison against a per-tile limit (the loop is integer-bound otherwise)
    const bool inside = (long)(row0 + TL::L) <= win_rows;
    const int lim = inside ? TL::L * N : (int)max(0L, min((long)TL::L * N, (win_rows - (long)row0) * N + win_tail));
    // the running max on the pipe the pass leaves idle: FP64 for FP32, whose
    // integer pipe is the busy one (measured at 512^3: 0.53 ms with a
    // per-element window test and an FP64 max, 0.60 with the tile limit and a
    // float max, 0.45 with the tile limit and an FP64 max); the storage type
    // for FP64 and mixed, whose FP64 pipe is busy (0.67 -> 0.64 and
    // 0.73 -> 0.65 ms)
    using MX = std::conditional_t<sizeof(K) == 4, double, R>;
    MX mx = MX(0);
    for (int f = threadIdx.x; f < TL::L * N; f += TL::NT) {
        const int l = f / N, n = f % N;
        const R v = Cvt<R, K>::outr(mulk(smr[2 * ((n >> 1) * TL::LP + l) + (n & 1)], inv.hi, inv.lo), salt, row0 * N + f);
        out[f] = v;
        if (f < lim) mx = fmax(mx, (MX)fabs(v));
    }
    const double m = warp_max((double)mx);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&ts->maxphi_bits, m);
}

// --------------------------------------------------------- y / x passes ---
// AXIS 1 (y): line g -> (x, z) = (g / W, g % W), element n at (x*N + n)*W + z.
// AXIS 2 (x): line g = column q, element n at n*N*W + q.
// Lines with (g % W) >= VW are padding: loads and stores skipped.
template <int AXIS> __device__ __forceinline__ size_t line_base(long g, int N, int W) {
    return AXIS == 1 ? size_t(g / W) * N * W + (g % W) : size_t(g);
}

template <typename R, typename K, int N, int DIR, int AXIS>
__global__ void __launch_bounds__(Tile<R, K, N>::NT)
    k_fft_yx(cx<R> *__restrict__ data, int W, int VW, const TState *__restrict__ ts, int pass,
             const cx<K> *__restrict__ tw) {
    using TL = Tile<R, K, N>;
    using C = typename TL::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sm = reinterpret_cast<C *>(smraw);
    const int l = threadIdx.x % TL::L;
    const long g = long(blockIdx.x) * TL::L + l;
    const bool valid = (g % W) < VW;
    const size_t b = line_base<AXIS>(g, N, W);
    const size_t S = AXIS == 1 ? size_t(W) : size_t(N) * W;
    const uint32_t salt = ts ? pass_salt(ts, pass) : 0x9e3779b9u;
    for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
        sm[n * TL::LP + l] = valid ? cin<K>(data[b + n * S]) : mkc(K(0), K(0));
    __syncthreads();
    fft_tile<C, N, TL::E, DIR, TL::L, TL::LP>(sm, tw);
    if (valid)
        for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
            data[b + n * S] = Cvt<R, K>::out(sm[n * TL::LP + l], salt, b + n * S);
}

// P3: x-pass forward, drift exp(-i s kappa^2) / N^3 from separable tables,
// x-pass inverse.  drift[i] = exp(-i s kappa_i^2) written by the timestep.
// The data are FFT(kicked psi - c); the drift leaves k = 0 unchanged, so c
// is added back after the inverse z-pass (P5).
template <typename R, typename K, int N>
__global__ void __launch_bounds__(Tile<R, K, N>::NT)
    k_fft_x_drift(cx<R> *__restrict__ psi, const cx<K> *__restrict__ drift, TState *__restrict__ ts,
                  const cx<K> *__restrict__ tw) {
    using TL = Tile<R, K, N>;
    using C = typename TL::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sm = reinterpret_cast<C *>(smraw);
    const int l = threadIdx.x % TL::L;
    const long q = long(blockIdx.x) * TL::L + l;  // column = y*N + z
    const size_t S = size_t(N) * N;
    const uint32_t salt = pass_salt(ts, 3);
    for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L) sm[n * TL::LP + l] = cin<K>(psi[q + n * S]);
    __syncthreads();
    fft_tile<C, N, TL::E, -1, TL::L, TL::LP>(sm, tw);
    if (q == 0 && threadIdx.x == 0) {
        // k = 0 coefficient = sum(kicked psi - c): the kicked field's mean, the next offset
        const double inv = 1.0 / ((double)N * N * N);
        ts->cnext_re = ts->cre + (double)sm[0].x * inv;
        ts->cnext_im = ts->cim + (double)sm[0].y * inv;
    }
    const int y = int(q / N), z = int(q % N);
    constexpr KSplit<K> inv3(1.0 / ((double)N * N * N));
    const C dyz = cmul(__ldg(drift + y), __ldg(drift + z));
    const C lf = mkc(mulk(dyz.x, inv3.hi, inv3.lo), mulk(dyz.y, inv3.hi, inv3.lo));
    for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
        sm[n * TL::LP + l] = cmul(sm[n * TL::LP + l], cmul(lf, __ldg(drift + n)));
    __syncthreads();
    fft_tile<C, N, TL::E, +1, TL::L, TL::LP>(sm, tw);
    for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
        psi[q + n * S] = Cvt<R, K>::out(sm[n * TL::LP + l], salt, q + n * S);
}

// P7: x-pass forward on the half spectrum, multiply by -1/kappa^2 (0 at k=0),
// x-pass inverse.
template <typename R, typename K, int N>
__global__ void __launch_bounds__(Tile<R, K, N>::NT)
    k_fft_x_poisson(cx<R> *__restrict__ rhok, const TState *__restrict__ ts, const cx<K> *__restrict__ tw) {
    using TL = Tile<R, K, N>;
    using C = typename TL::C;
    constexpr int NH = N / 2 + 1;
    constexpr int NHP = half_pitch<R>(N);
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sm = reinterpret_cast<C *>(smraw);
    const int l = threadIdx.x % TL::L;
    const long q = long(blockIdx.x) * TL::L + l;  // column = y*NHP + kz
    const int y = int(q / NHP), kz = int(q % NHP);
    const bool valid = kz < NH;
    const size_t S = size_t(N) * NHP;
    const uint32_t salt = pass_salt(ts, 7);
    for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
        sm[n * TL::LP + l] = valid ? cin<K>(rhok[q + n * S]) : mkc(K(0), K(0));
    __syncthreads();
    fft_tile<C, N, TL::E, -1, TL::L, TL::LP>(sm, tw);
    const int ky = kappa(y, N), kzz = kappa(kz, N);
    const int k2yz = ky * ky + kzz * kzz;
    for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L) {
        const int kx = kappa(n, N);
        const int k2 = kx * kx + k2yz;
        const K m = k2 == 0 ? K(0) : K(-1) / K(k2);
        sm[n * TL::LP + l] = cscale(sm[n * TL::LP + l], m);
    }
    __syncthreads();
    fft_tile<C, N, TL::E, +1, TL::L, TL::LP>(sm, tw);
    if (valid)
        for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
            rhok[q + n * S] = Cvt<R, K>::out(sm[n * TL::LP + l], salt, q + n * S);
}

// x-pass of a slab-decomposed Poisson solve.  The data are a rank's y-slab
// [x][planes][N] of a complex field already transformed along z and y (the
// layout after the x <-> y transpose of the slab scheme), holding the global
// y-planes y0 .. y0 + planes - 1: forward FFT along x, multiply by
// -1/(kappa^2 N^3) (0 at kappa = 0; the 1/N^3 of the three inverse
// transforms folded in), inverse FFT along x.
template <typename R, typename K, int N>
__global__ void __launch_bounds__(Tile<R, K, N>::NT)
    k_fft_x_poisson_slab(cx<R> *__restrict__ data, int planes, int y0, const cx<K> *__restrict__ tw) {
    using TL = Tile<R, K, N>;
    using C = typename TL::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sm = reinterpret_cast<C *>(smraw);
    const int l = threadIdx.x % TL::L;
    const long q = long(blockIdx.x) * TL::L + l;  // column = y_local * N + z
    const int y = y0 + int(q / N), z = int(q % N);
    const size_t S = size_t(N) * planes;
    for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L) sm[n * TL::LP + l] = cin<K>(data[q + n * S]);
    __syncthreads();
    fft_tile<C, N, TL::E, -1, TL::L, TL::LP>(sm, tw);
    const int ky = kappa(y, N), kz = kappa(z, N);
    const int k2yz = ky * ky + kz * kz;
    const double inv3 = 1.0 / ((double)N * N * N);
    for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L) {
        const int kx = kappa(n, N);
        const int k2 = kx * kx + k2yz;
        sm[n * TL::LP + l] = cscale(sm[n * TL::LP + l], k2 == 0 ? K(0) : K(-inv3 / k2));
    }
    __syncthreads();
    fft_tile<C, N, TL::E, +1, TL::L, TL::LP>(sm, tw);
    for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
        data[q + n * S] = Cvt<R, K>::out(sm[n * TL::LP + l], 0x6a09e667u, q + n * S);
}

// ------------------------------------------------------- state transfer ---
// out = S * psi_s * exp(-i (cP phi_s + cQ |psi_s|^2)) as complex128; the
// coefficients are read from the TState field pair selected by `which`
// (0: none, 1: snapshot kick, 2: pending kick).
template <typename R>
__global__ void k_psi_out(const cx<R> *__restrict__ psi, const R *__restrict__ phi, const TState *__restrict__ ts,
                          int which, double S, double2 *__restrict__ out, size_t n) {
    const double cp = which == 1 ? ts->snapP : (which == 2 ? ts->pendP : 0.0);
    const double cq = which == 1 ? ts->snapQ : (which == 2 ? ts->pendQ : 0.0);
    // undo the accumulated dither phase (psi is stored as exp(-i g) psi)
    const double g = which == 1 ? ts->gphase_prev : ts->gphase;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const cx<R> v = psi[i];
        double2 w = make_double2((double)v.x, (double)v.y);
        if (which || g != 0.0) {
            const double p = cp * (double)phi[i] + cq * (w.x * w.x + w.y * w.y) - g;
            double s, c;
            sincos(p, &s, &c);
            w = make_double2(w.x * c + w.y * s, w.y * c - w.x * s);
        }
        out[i] = make_double2(w.x * S, w.y * S);
    }
}

template <typename R>
__global__ void k_psi_in(const double2 *__restrict__ in, cx<R> *__restrict__ psi, double invS, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double2 v = in[i];
        psi[i] = mkc((R)(v.x * invS), (R)(v.y * invS));
    }
}

template <typename R>
__global__ void k_phi_out(const R *__restrict__ phi, double Phi0, double *__restrict__ out, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = (double)phi[i] * Phi0;
}

}  // namespace ifdm
