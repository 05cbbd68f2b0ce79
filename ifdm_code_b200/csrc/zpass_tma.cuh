// zpass_tma.cuh -- persistent z passes fed by bulk copies (FP32 and FP64, N >= 256).
//
// The z passes work on whole rows (z fastest), which are contiguous in HBM.
// Each CTA keeps a ring of ST slots; thread 0 keeps ST-1 tiles of rows in
// flight with one untiled cp.async.bulk per row (completion on one mbarrier
// per slot), so the bytes in flight no longer depend on registers, while the
// CTA transforms the current tile with the register-resident Stockham chain
// of the y/x passes.  Rows land at a pitch padded by 16 bytes: the first
// stage reads element n of row l with the row index fastest across a warp,
// and the pad puts those rows in different banks.  Later stages exchange
// through the same slot laid out [n][l] (the swizzled 8-line tile of the
// narrow x passes).  The twiddle table is staged in shared memory once per
// CTA.  Every mbarrier wait is bounded (error bit in TState).
//
//   k_kick_fft_z_tma      P1: kick with the merged coefficients, remove the
//                         offset c, forward FFT along z.
//   k_density_r2c_z_tma   P5: inverse FFT along z, add c -> psi, density
//                         rho = |psi|^2 - mu, max |psi|^2, and the real-to-
//                         half-complex FFT of rho: rows l and l+4 of the tile
//                         packed as one complex line rho_l + i rho_{l+4},
//                         one N-point complex FFT, then
//                         X_l = (Z_k + conj Z_{N-k})/2,
//                         X_{l+4} = -i (Z_k - conj Z_{N-k})/2   (k = 0..N/2).
//   k_c2r_z_tma           P9: the inverse of that packing: half rows l and
//                         l+8 of a 16-row tile become Z = X_l + i X_{l+8}
//                         on the full circle (X_{N-k} = conj X_k), one
//                         N-point inverse FFT gives N phi_l + i N phi_{l+8};
//                         scale by 1/N^3, store, max|phi| over the
//                         reference's scan window.
// The packed transforms need no post-twiddle (the half-length method of
// k_density_r2c_z / k_c2r_z_phi does): the same N-point plan and table as
// the complex passes.
#pragma once

#include "step_kernels.cuh"
#include "tma.cuh"

namespace ifdm {

// Tile geometry of the z passes: L complex rows per tile (NT threads), 64
// bytes of the [n][l] exchange tile per element index: 8 FP32 rows or 4 FP64
// rows.  Landed rows are padded by 2 elements (16 bytes FP32, 32 bytes FP64),
// which puts the rows of a tile in different banks for the row-fastest first
// stage.
template <int N, typename R = float> struct ZT {
    using C = cx<R>;
    static constexpr int L = sizeof(R) == 4 ? 8 : 4;
    static constexpr int E = Plan<N>::E;
    static constexpr int T = N / E;
    static constexpr int NT = L * T;
    static constexpr int R0 = Plan<N>::R[0];
    static constexpr int RL = Plan<N>::R[Plan<N>::NST - 1];
    static constexpr int PP = N + 2;  // complex elements per landed psi row
    static constexpr int PF = N + 4;  // reals per landed phi row
    static constexpr int NHP = half_pitch<R>(N);
    static constexpr int PH = NHP + 2;  // complex elements per landed half row
    static constexpr size_t XCH = size_t(N) * L * sizeof(C);  // [n][l] exchange tile
    // P1 slot: L psi rows, then L phi rows
    static constexpr size_t PSI_B = size_t(L) * PP * sizeof(C);
    static constexpr size_t SLOT1 = (PSI_B + size_t(L) * PF * sizeof(R) + 127) / 128 * 128;
    // P5 slot: L psi rows
    static constexpr size_t SLOT5 = (PSI_B + 127) / 128 * 128;
    // P9 slot: 2L half rows
    static constexpr size_t SLOT9 = (size_t(2 * L) * PH * sizeof(C) + 127) / 128 * 128;
    static_assert(XCH <= PSI_B && XCH <= SLOT9, "the exchange tile fits the landed rows");
    static_assert(E % R0 == 0 && E % RL == 0 && R0 == RL, "register chain: equal first and last radix");
    static_assert((N * sizeof(C)) % 16 == 0 && (NHP * sizeof(C)) % 16 == 0 && (PP * sizeof(C)) % 16 == 0 &&
                      (PF * sizeof(R)) % 16 == 0 && (PH * sizeof(C)) % 16 == 0,
                  "bulk copies need 16-byte sizes and destinations");
};

template <int ST> __device__ __forceinline__ void ring_init(uint64_t *bar) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) mbar_init(&bar[s], 1);
        mbar_init_fence();
    }
    __syncthreads();
}

// Bounded wait for tile i of the ring; on failure waits (bounded) for the
// copies still in flight and returns false for the whole CTA.
template <int ST> __device__ __forceinline__ bool ring_wait(uint64_t *bar, int i, int my_n, int *err) {
    const bool ok = mbar_wait(&bar[i % ST], (uint32_t)((i / ST) & 1), err, 2);
    if (__syncthreads_and(ok)) return true;
    if (threadIdx.x == 0)
        for (int j = i; j < my_n && j <= i + ST - 1; ++j) mbar_wait(&bar[j % ST], (uint32_t)((j / ST) & 1), err, 2);
    __syncthreads();
    return false;
}

__device__ __forceinline__ int ztiles_of_block(int ntiles) {
    return (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
}

// ------------------------------------------------------------------- P1 ---
template <int N, int ST, int MINB, typename R = float>
__global__ void __launch_bounds__(ZT<N, R>::NT, MINB)
    k_kick_fft_z_tma(cx<R> *__restrict__ psi, const R *__restrict__ phi, TState *__restrict__ ts,
                     const cx<R> *__restrict__ tw, int ntiles) {
    using Z = ZT<N, R>;
    using C = cx<R>;
    constexpr int L = Z::L, T = Z::T, E = Z::E, R0 = Z::R0, RL = Z::RL;
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + ST * Z::SLOT1);
    const int tid = threadIdx.x, l = tid % L, t = tid / L;
    C *stw = reinterpret_cast<C *>(smraw + ST * Z::SLOT1 + 64);
    stage_twiddles(stw, tw, N);
    const SmemTw<C> tws{stw};
    ring_init<ST>(bar);
    const int my_n = ztiles_of_block(ntiles);
    auto issue = [&](int i) {
        const size_t row0 = size_t(blockIdx.x + (long)i * gridDim.x) * L;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT1;
        uint64_t *b = &bar[i % ST];
        mbar_arrive_expect_tx(b, (uint32_t)(L * N * (sizeof(C) + sizeof(R))));
#pragma unroll 1
        for (int r = 0; r < L; ++r) {
            bulk_load(slot + size_t(r) * Z::PP * sizeof(C), psi + (row0 + r) * N, N * sizeof(C), b);
            bulk_load(slot + Z::PSI_B + size_t(r) * Z::PF * sizeof(R), phi + (row0 + r) * N, N * sizeof(R),
                      b);
        }
    };
    if (tid == 0)
        for (int i = 0; i < ST - 1 && i < my_n; ++i) issue(i);
    const double cp = ts->coefP, cq = ts->coefQ, alpha = ts->alpha;
    const C c0 = mkc((R)ts->cre, (R)ts->cim);
    for (int i = 0; i < my_n; ++i) {
        if (tid == 0 && i + ST - 1 < my_n) issue(i + ST - 1);
        if (!ring_wait<ST>(bar, i, my_n, &ts->err)) return;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT1;
        const C *lp = reinterpret_cast<const C *>(slot) + l * Z::PP;
        const R *lf = reinterpret_cast<const R *>(slot + Z::PSI_B) + l * Z::PF;
        C v[E];
#pragma unroll
        for (int b = 0; b < E / R0; ++b)
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int n = t + T * b + r * (N / R0);
                const C g = lp[n];
                const double p = cp * (double)lf[n] + cq * (double)cnorm2(g) + alpha;
                v[b * R0 + r] = cmul(g, expmi<R>(p)) - c0;
            }
        stage_compute<C, N, E, -1, R0, 1>(v, tws, t);
        RegChain<C, N, E, -1, L, L, 1, R0, 1>::run(reinterpret_cast<C *>(slot), v, tws, l, t, true);
        C *out = psi + (size_t(blockIdx.x + (long)i * gridDim.x) * L + l) * N;
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) out[t + T * b + r * (N / RL)] = v[b * RL + r];
        fence_proxy_async_smem();
        __syncthreads();
    }
}

// P1 with half the threads (256 per 8-row tile at 512), two rows per thread
// (the kick of both rows, then the paired transform: fft_engine.cuh,
// *_pair).  Same slots, arithmetic and outputs as k_kick_fft_z_tma.
template <int N, int ST, int MINB>
__global__ void __launch_bounds__(ZT<N>::NT / 2, MINB)
    k_kick_fft_z_pair(float2 *__restrict__ psi, const float *__restrict__ phi, TState *__restrict__ ts,
                      const float2 *__restrict__ tw, int ntiles) {
    using Z = ZT<N>;
    using C = float2;
    constexpr int L = Z::L, LH = L / 2, T = Z::T, E = Z::E, R0 = Z::R0, RL = Z::RL;
    static_assert(Z::NT / 2 == LH * T, "one thread per row pair");
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + ST * Z::SLOT1);
    const int tid = threadIdx.x, lp = tid % LH, t = tid / LH;
    float4 *stw = reinterpret_cast<float4 *>(smraw + ST * Z::SLOT1 + 64);
    stage_twiddles_staged<N>(stw, tw);
    const StagedTw<N> tws{stw};
    ring_init<ST>(bar);
    const int my_n = ztiles_of_block(ntiles);
    auto issue = [&](int i) {
        const size_t row0 = size_t(blockIdx.x + (long)i * gridDim.x) * L;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT1;
        uint64_t *b = &bar[i % ST];
        mbar_arrive_expect_tx(b, (uint32_t)(L * N * (sizeof(float2) + sizeof(float))));
#pragma unroll 1
        for (int r = 0; r < L; ++r) {
            bulk_load(slot + size_t(r) * Z::PP * sizeof(float2), psi + (row0 + r) * N, N * sizeof(float2), b);
            bulk_load(slot + Z::PSI_B + size_t(r) * Z::PF * sizeof(float), phi + (row0 + r) * N, N * sizeof(float),
                      b);
        }
    };
    if (tid == 0)
        for (int i = 0; i < ST - 1 && i < my_n; ++i) issue(i);
    const double cp = ts->coefP, cq = ts->coefQ, alpha = ts->alpha;
    const C c0 = mkc((float)ts->cre, (float)ts->cim);
    for (int i = 0; i < my_n; ++i) {
        if (tid == 0 && i + ST - 1 < my_n) issue(i + ST - 1);
        if (!ring_wait<ST>(bar, i, my_n, &ts->err)) return;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT1;
        const C *pa = reinterpret_cast<const C *>(slot) + (2 * lp) * Z::PP, *pb = pa + Z::PP;
        const float *fa = reinterpret_cast<const float *>(slot + Z::PSI_B) + (2 * lp) * Z::PF, *fb = fa + Z::PF;
        C va[E], vb[E];
#pragma unroll
        for (int b = 0; b < E / R0; ++b)
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int n = t + T * b + r * (N / R0);
                const C ga = pa[n], gb = pb[n];
                const double qa = cp * (double)fa[n] + cq * (double)cnorm2(ga) + alpha;
                const double qb = cp * (double)fb[n] + cq * (double)cnorm2(gb) + alpha;
                va[b * R0 + r] = cmul(ga, expmi<float>(qa)) - c0;
                vb[b * R0 + r] = cmul(gb, expmi<float>(qb)) - c0;
            }
        stage_compute_pair<N, E, -1, R0, 1>(va, vb, tws, t);
        RegChainPair<N, E, -1, LH, 1, R0, 1>::run(reinterpret_cast<float4 *>(slot), va, vb, tws, lp, t);
        C *oa = psi + (size_t(blockIdx.x + (long)i * gridDim.x) * L + 2 * lp) * N, *ob = oa + N;
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const int n = t + T * b + r * (N / RL);
                oa[n] = va[b * RL + r];
                ob[n] = vb[b * RL + r];
            }
        fence_proxy_async_smem();
        __syncthreads();
    }
}

// ------------------------------------------------------------------- P5 ---
template <int N, int ST, int MINB, typename R = float>
__global__ void __launch_bounds__(ZT<N, R>::NT, MINB)
    k_density_r2c_z_tma(cx<R> *__restrict__ psi, cx<R> *__restrict__ rhok, TState *__restrict__ ts,
                        const cx<R> *__restrict__ tw, int ntiles) {
    using Z = ZT<N, R>;
    using C = cx<R>;
    constexpr int L = Z::L, T = Z::T, E = Z::E, R0 = Z::R0, RL = Z::RL, NT = Z::NT;
    constexpr int M = N / 2, NHP = Z::NHP;
    constexpr int LH = L / 2;  // packed complex lines of the density transform
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + ST * Z::SLOT5);
    const int tid = threadIdx.x, l = tid % L, t = tid / L;
    C *stw = reinterpret_cast<C *>(smraw + ST * Z::SLOT5 + 64);
    stage_twiddles(stw, tw, N);
    const SmemTw<C> tws{stw};
    // the density transform: 4 lines, T threads each (whole warps: threads < LH * T)
    const bool act = tid < LH * T;
    const int p = tid % LH, tq = tid / LH;
    ring_init<ST>(bar);
    const int my_n = ztiles_of_block(ntiles);
    auto issue = [&](int i) {
        const size_t row0 = size_t(blockIdx.x + (long)i * gridDim.x) * L;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT5;
        uint64_t *b = &bar[i % ST];
        mbar_arrive_expect_tx(b, (uint32_t)(L * N * sizeof(C)));
#pragma unroll 1
        for (int r = 0; r < L; ++r)
            bulk_load(slot + size_t(r) * Z::PP * sizeof(C), psi + (row0 + r) * N, N * sizeof(C), b);
    };
    if (tid == 0)
        for (int i = 0; i < ST - 1 && i < my_n; ++i) issue(i);
    const double mu = ts->mu;
    const C c0 = mkc((R)ts->cre, (R)ts->cim);
    double mx = 0.0;
    for (int i = 0; i < my_n; ++i) {
        if (tid == 0 && i + ST - 1 < my_n) issue(i + ST - 1);
        if (!ring_wait<ST>(bar, i, my_n, &ts->err)) return;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT5;
        C *wk = reinterpret_cast<C *>(slot);
        const size_t row0 = size_t(blockIdx.x + (long)i * gridDim.x) * L;
        // inverse FFT of psi along z, stage 0 from the landed rows
        C v[E];
        const C *lp = reinterpret_cast<const C *>(slot) + l * Z::PP;
#pragma unroll
        for (int b = 0; b < E / R0; ++b)
#pragma unroll
            for (int r = 0; r < R0; ++r) v[b * R0 + r] = lp[t + T * b + r * (N / R0)];
        stage_compute<C, N, E, +1, R0, 1>(v, tws, t);
        RegChain<C, N, E, +1, L, L, 1, R0, 1>::run(wk, v, tws, l, t, true);
        // psi = IFFT + c; rho = |psi|^2 - mu into a real tile that pairs rows
        // p and p+LH of element n: rt[(n*LH + p)*2 + h] holds row p + h*LH
        // (conflict-free stores of the [l, t] layout and complex loads of the
        // packed layout)
        R rho[E];
        C *out = psi + (row0 + l) * N;
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const C g = v[b * RL + r] + c0;
                out[t + T * b + r * (N / RL)] = g;
                const double n2 = (double)cnorm2(g);
                mx = fmax(mx, n2);
                rho[b * RL + r] = (R)(n2 - mu);
            }
        R *rt = reinterpret_cast<R *>(slot);
        __syncthreads();  // every thread is done with the exchange tile
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r)
                rt[((t + T * b + r * (N / RL)) * LH + l % LH) * 2 + l / LH] = rho[b * RL + r];
        __syncthreads();
        // packed lines rho_p + i rho_{p+4}, forward FFT (threads < LH*T)
        if (act) {
            const C *rp = reinterpret_cast<const C *>(rt);
#pragma unroll
            for (int b = 0; b < E / R0; ++b)
#pragma unroll
                for (int r = 0; r < R0; ++r) v[b * R0 + r] = rp[(tq + T * b + r * (N / R0)) * LH + p];
            stage_compute<C, N, E, -1, R0, 1>(v, tws, tq);
        }
        RegChain<C, N, E, -1, LH, LH, 1, R0, 3>::run(wk, v, tws, p, tq, act);
        // Z_k in an [k][p] tile, then the two half spectra of each line
        __syncthreads();
        if (act) {
#pragma unroll
            for (int b = 0; b < E / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) wk[(tq + T * b + r * (N / RL)) * LH + p] = v[b * RL + r];
        }
        __syncthreads();
        for (int q = tid; q < LH * (M + 1); q += NT) {
            const int pp = q % LH, k = q / LH;
            const C zk = wk[k * LH + pp];
            const C zc = cconj(wk[((N - k) % N) * LH + pp]);
            const C s = cscale(zk + zc, R(0.5));
            const C d = cscale(zk - zc, R(0.5));
            rhok[(row0 + pp) * NHP + k] = s;
            rhok[(row0 + pp + LH) * NHP + k] = mkc(d.y, -d.x);
        }
        fence_proxy_async_smem();
        __syncthreads();
    }
    mx = warp_max(mx);
    if ((tid & 31) == 0 && my_n > 0) atomic_max_nonneg(&ts->maxrho_bits, mx);
}

// P5 with half the threads (256 per 8-row tile at 512): the inverse transform
// of psi runs two rows per thread (fft_engine.cuh, *_pair: 128-bit exchanges,
// one twiddle load per two rows), the packed density transform of the tile's
// 4 complex lines one line per thread, so every thread works in both
// transforms (the one-line kernel above idles half of its threads in the
// second one).  The packed line of thread lp is rho_{2lp} + i rho_{2lp+1}, its
// own two rows, so the density goes from registers straight into the second
// transform.  Same slots and outputs as k_density_r2c_z_tma, the same
// arithmetic but for which rows share a packed line.
template <int N, int ST, int MINB>
__global__ void __launch_bounds__(ZT<N>::NT / 2, MINB)
    k_density_r2c_z_pair(float2 *__restrict__ psi, float2 *__restrict__ rhok, TState *__restrict__ ts,
                         const float2 *__restrict__ tw, int ntiles) {
    using Z = ZT<N>;
    using C = float2;
    constexpr int L = Z::L, T = Z::T, E = Z::E, R0 = Z::R0, RL = Z::RL, NT = Z::NT / 2;
    constexpr int M = N / 2, NHP = Z::NHP;
    constexpr int LH = L / 2;  // row pairs of the psi transform = packed lines of the density transform
    static_assert(NT == LH * T, "one thread per row pair and per packed line");
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + ST * Z::SLOT5);
    const int tid = threadIdx.x, lp = tid % LH, t = tid / LH;
    float4 *stw = reinterpret_cast<float4 *>(smraw + ST * Z::SLOT5 + 64);
    stage_twiddles_staged<N>(stw, tw);
    const StagedTw<N> tws{stw};
    ring_init<ST>(bar);
    const int my_n = ztiles_of_block(ntiles);
    auto issue = [&](int i) {
        const size_t row0 = size_t(blockIdx.x + (long)i * gridDim.x) * L;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT5;
        uint64_t *b = &bar[i % ST];
        mbar_arrive_expect_tx(b, (uint32_t)(L * N * sizeof(float2)));
#pragma unroll 1
        for (int r = 0; r < L; ++r)
            bulk_load(slot + size_t(r) * Z::PP * sizeof(float2), psi + (row0 + r) * N, N * sizeof(float2), b);
    };
    if (tid == 0)
        for (int i = 0; i < ST - 1 && i < my_n; ++i) issue(i);
    const double mu = ts->mu;
    const C c0 = mkc((float)ts->cre, (float)ts->cim);
    double mx = 0.0;
    for (int i = 0; i < my_n; ++i) {
        if (tid == 0 && i + ST - 1 < my_n) issue(i + ST - 1);
        if (!ring_wait<ST>(bar, i, my_n, &ts->err)) return;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT5;
        C *wk = reinterpret_cast<C *>(slot);
        const size_t row0 = size_t(blockIdx.x + (long)i * gridDim.x) * L;
        // inverse FFT of rows 2lp (va) and 2lp + 1 (vb), stage 0 from the landed rows
        C va[E], vb[E];
        const C *la = reinterpret_cast<const C *>(slot) + (2 * lp) * Z::PP, *lb = la + Z::PP;
#pragma unroll
        for (int b = 0; b < E / R0; ++b)
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int n = t + T * b + r * (N / R0);
                va[b * R0 + r] = la[n];
                vb[b * R0 + r] = lb[n];
            }
        stage_compute_pair<N, E, +1, R0, 1>(va, vb, tws, t);
        RegChainPair<N, E, +1, LH, 1, R0, 1>::run(reinterpret_cast<float4 *>(wk), va, vb, tws, lp, t);
        // psi = IFFT + c; rho = |psi|^2 - mu; the thread's two rows 2lp and
        // 2lp + 1 form the packed line rho_{2lp} + i rho_{2lp+1}, whose
        // elements are already the first-stage inputs of the next transform
        // (first radix = last radix): no exchange through shared memory
        const int p = lp;
        C v[E];
        C *oa = psi + (row0 + 2 * lp) * N, *ob = oa + N;
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const int n = t + T * b + r * (N / RL);
                const C ga = va[b * RL + r] + c0, gb = vb[b * RL + r] + c0;
                oa[n] = ga;
                ob[n] = gb;
                const double na = (double)cnorm2(ga), nb = (double)cnorm2(gb);
                mx = fmax(mx, fmax(na, nb));
                v[b * RL + r] = mkc((float)(na - mu), (float)(nb - mu));
            }
        // forward FFT of the packed line, one line per thread
        stage_compute<C, N, E, -1, R0, 1>(v, tws, t);
        RegChain<C, N, E, -1, LH, LH, 1, R0, 3>::run(wk, v, tws, p, t, true);
        // Z_k in an [k][p] tile, then the two half spectra of each line
        __syncthreads();
#pragma unroll
        for (int b = 0; b < E / RL; ++b)
#pragma unroll
            for (int r = 0; r < RL; ++r) wk[(t + T * b + r * (N / RL)) * LH + p] = v[b * RL + r];
        __syncthreads();
        for (int q = tid; q < LH * (M + 1); q += NT) {
            const int pp = q % LH, k = q / LH;
            const C zk = wk[k * LH + pp];
            const C zc = cconj(wk[((N - k) % N) * LH + pp]);
            const C s = cscale(zk + zc, 0.5f);
            const C d = cscale(zk - zc, 0.5f);
            rhok[(row0 + 2 * pp) * NHP + k] = s;
            rhok[(row0 + 2 * pp + 1) * NHP + k] = mkc(d.y, -d.x);
        }
        fence_proxy_async_smem();
        __syncthreads();
    }
    mx = warp_max(mx);
    if ((tid & 31) == 0 && my_n > 0) atomic_max_nonneg(&ts->maxrho_bits, mx);
}

// ------------------------------------------------------------------- P9 ---
template <int N, int ST, int MINB, typename R = float>
__global__ void __launch_bounds__(ZT<N, R>::NT, MINB)
    k_c2r_z_tma(const cx<R> *__restrict__ rhok, R *__restrict__ phi, TState *__restrict__ ts, long win_rows,
                int win_tail, const cx<R> *__restrict__ tw, int ntiles) {
    using Z = ZT<N, R>;
    using C = cx<R>;
    constexpr int L = Z::L, T = Z::T, E = Z::E, R0 = Z::R0, RL = Z::RL;
    constexpr int M = N / 2, NHP = Z::NHP, ROWS = 2 * L;
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + ST * Z::SLOT9);
    const int tid = threadIdx.x, l = tid % L, t = tid / L;
    C *stw = reinterpret_cast<C *>(smraw + ST * Z::SLOT9 + 64);
    stage_twiddles(stw, tw, N);
    const SmemTw<C> tws{stw};
    ring_init<ST>(bar);
    const int my_n = ztiles_of_block(ntiles);
    auto issue = [&](int i) {
        const size_t row0 = size_t(blockIdx.x + (long)i * gridDim.x) * ROWS;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT9;
        uint64_t *b = &bar[i % ST];
        mbar_arrive_expect_tx(b, (uint32_t)(ROWS * NHP * sizeof(C)));
#pragma unroll 1
        for (int r = 0; r < ROWS; ++r)
            bulk_load(slot + size_t(r) * Z::PH * sizeof(C), rhok + (row0 + r) * NHP, NHP * sizeof(C), b);
    };
    if (tid == 0)
        for (int i = 0; i < ST - 1 && i < my_n; ++i) issue(i);
    constexpr KSplit<R> inv(1.0 / ((double)N * N * N));
    double mx = 0.0;  // the running max on the FP64 pipe, which this pass leaves idle
    for (int i = 0; i < my_n; ++i) {
        if (tid == 0 && i + ST - 1 < my_n) issue(i + ST - 1);
        if (!ring_wait<ST>(bar, i, my_n, &ts->err)) return;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT9;
        const C *xa = reinterpret_cast<const C *>(slot) + l * Z::PH;
        const C *xb = xa + L * Z::PH;
        C v[E];
#pragma unroll
        for (int bb = 0; bb < E / R0; ++bb)
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int n = t + T * bb + r * (N / R0);
                const int m = n <= M ? n : N - n;
                C a = xa[m], b = xb[m];
                if (m == 0 || m == M) {  // c2r ignores these imaginary parts
                    a.y = R(0);
                    b.y = R(0);
                }
                v[bb * R0 + r] = n <= M ? mkc(a.x - b.y, a.y + b.x) : mkc(a.x + b.y, b.x - a.y);
            }
        stage_compute<C, N, E, +1, R0, 1>(v, tws, t);
        RegChain<C, N, E, +1, L, L, 1, R0, 1>::run(reinterpret_cast<C *>(slot), v, tws, l, t, true);
        const long ra = long(blockIdx.x + (long)i * gridDim.x) * ROWS + l, rb = ra + L;
        // elements of rows below win_rows, and the first win_tail of row win_rows, are in the window
        const int lima = ra < win_rows ? N : (ra == win_rows ? win_tail : 0);
        const int limb = rb < win_rows ? N : (rb == win_rows ? win_tail : 0);
        R *oa = phi + size_t(ra) * N, *ob = phi + size_t(rb) * N;
#pragma unroll
        for (int bb = 0; bb < E / RL; ++bb)
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const int n = t + T * bb + r * (N / RL);
                const C z = v[bb * RL + r];
                const R fa = mulk(z.x, inv.hi, inv.lo), fb = mulk(z.y, inv.hi, inv.lo);
                oa[n] = fa;
                ob[n] = fb;
                if (n < lima) mx = fmax(mx, fabs((double)fa));
                if (n < limb) mx = fmax(mx, fabs((double)fb));
            }
        fence_proxy_async_smem();
        __syncthreads();
    }
    const double m = warp_max(mx);
    if ((tid & 31) == 0) atomic_max_nonneg(&ts->maxphi_bits, m);
}

// P9 with half the threads (256 per 16-row tile at 512): packed lines 2lp and
// 2lp + 1 (rows 2lp, 2lp + 8 and 2lp + 1, 2lp + 9) per thread, the paired
// inverse transform (fft_engine.cuh, *_pair).  Same slots, arithmetic and
// outputs as k_c2r_z_tma.
template <int N, int ST, int MINB>
__global__ void __launch_bounds__(ZT<N>::NT / 2, MINB)
    k_c2r_z_pair(const float2 *__restrict__ rhok, float *__restrict__ phi, TState *__restrict__ ts, long win_rows,
                 int win_tail, const float2 *__restrict__ tw, int ntiles) {
    using Z = ZT<N>;
    using C = float2;
    constexpr int L = Z::L, LH = L / 2, T = Z::T, E = Z::E, R0 = Z::R0, RL = Z::RL;
    constexpr int M = N / 2, NHP = Z::NHP, ROWS = 2 * L;
    static_assert(Z::NT / 2 == LH * T, "one thread per line pair");
    extern __shared__ __align__(128) unsigned char smraw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + ST * Z::SLOT9);
    const int tid = threadIdx.x, lp = tid % LH, t = tid / LH;
    float4 *stw = reinterpret_cast<float4 *>(smraw + ST * Z::SLOT9 + 64);
    stage_twiddles_staged<N>(stw, tw);
    const StagedTw<N> tws{stw};
    ring_init<ST>(bar);
    const int my_n = ztiles_of_block(ntiles);
    auto issue = [&](int i) {
        const size_t row0 = size_t(blockIdx.x + (long)i * gridDim.x) * ROWS;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT9;
        uint64_t *b = &bar[i % ST];
        mbar_arrive_expect_tx(b, (uint32_t)(ROWS * NHP * sizeof(float2)));
#pragma unroll 1
        for (int r = 0; r < ROWS; ++r)
            bulk_load(slot + size_t(r) * Z::PH * sizeof(float2), rhok + (row0 + r) * NHP, NHP * sizeof(float2), b);
    };
    if (tid == 0)
        for (int i = 0; i < ST - 1 && i < my_n; ++i) issue(i);
    constexpr KSplit<float> inv(1.0 / ((double)N * N * N));
    double mx = 0.0;  // the running max on the FP64 pipe, which this pass leaves idle
    // line l of the tile: Z = X_l + i X_{l+8} on the full circle (X_{N-k} = conj X_k)
    auto packed = [&](const C *xa, const C *xb, int n) {
        const int m = n <= M ? n : N - n;
        C a = xa[m], b = xb[m];
        if (m == 0 || m == M) {  // c2r ignores these imaginary parts
            a.y = 0.f;
            b.y = 0.f;
        }
        return n <= M ? mkc(a.x - b.y, a.y + b.x) : mkc(a.x + b.y, b.x - a.y);
    };
    for (int i = 0; i < my_n; ++i) {
        if (tid == 0 && i + ST - 1 < my_n) issue(i + ST - 1);
        if (!ring_wait<ST>(bar, i, my_n, &ts->err)) return;
        unsigned char *slot = smraw + size_t(i % ST) * Z::SLOT9;
        const C *xa0 = reinterpret_cast<const C *>(slot) + (2 * lp) * Z::PH, *xb0 = xa0 + L * Z::PH;
        const C *xa1 = xa0 + Z::PH, *xb1 = xb0 + Z::PH;
        C va[E], vb[E];
#pragma unroll
        for (int bb = 0; bb < E / R0; ++bb)
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int n = t + T * bb + r * (N / R0);
                va[bb * R0 + r] = packed(xa0, xb0, n);
                vb[bb * R0 + r] = packed(xa1, xb1, n);
            }
        stage_compute_pair<N, E, +1, R0, 1>(va, vb, tws, t);
        RegChainPair<N, E, +1, LH, 1, R0, 1>::run(reinterpret_cast<float4 *>(slot), va, vb, tws, lp, t);
        // line 2lp writes rows ra, ra + 8; line 2lp + 1 rows ra + 1, ra + 9
        const long ra = long(blockIdx.x + (long)i * gridDim.x) * ROWS + 2 * lp;
        const long rows[4] = {ra, ra + L, ra + 1, ra + 1 + L};
        int lim[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)  // elements of rows below win_rows, and the first win_tail of row win_rows
            lim[q] = rows[q] < win_rows ? N : (rows[q] == win_rows ? win_tail : 0);
        float *o0 = phi + size_t(rows[0]) * N, *o1 = phi + size_t(rows[1]) * N;
        float *o2 = phi + size_t(rows[2]) * N, *o3 = phi + size_t(rows[3]) * N;
#pragma unroll
        for (int bb = 0; bb < E / RL; ++bb)
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const int n = t + T * bb + r * (N / RL);
                const C za = va[bb * RL + r], zb = vb[bb * RL + r];
                const float f0 = mulk(za.x, inv.hi, inv.lo), f1 = mulk(za.y, inv.hi, inv.lo);
                const float f2 = mulk(zb.x, inv.hi, inv.lo), f3 = mulk(zb.y, inv.hi, inv.lo);
                o0[n] = f0;
                o1[n] = f1;
                o2[n] = f2;
                o3[n] = f3;
                if (n < lim[0]) mx = fmax(mx, (double)fabsf(f0));
                if (n < lim[1]) mx = fmax(mx, (double)fabsf(f1));
                if (n < lim[2]) mx = fmax(mx, (double)fabsf(f2));
                if (n < lim[3]) mx = fmax(mx, (double)fabsf(f3));
            }
        fence_proxy_async_smem();
        __syncthreads();
    }
    const double m = warp_max(mx);
    if ((tid & 31) == 0) atomic_max_nonneg(&ts->maxphi_bits, m);
}

}  // namespace ifdm
