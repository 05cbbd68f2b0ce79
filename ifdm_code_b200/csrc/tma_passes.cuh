// tma_passes.cuh -- persistent, TMA-pipelined y- and x-axis passes.
//
// Each CTA owns a ring of STAGES tile buffers in shared memory.  Thread 0
// keeps STAGES-1 tile loads in flight (cp.async.bulk.tensor into the ring,
// completion on one mbarrier per slot) while the whole CTA transforms the
// current tile in place and writes it back with coalesced stores.  The tile
// is N rows (the transform axis) by L consecutive lines (128-byte rows), laid
// out [n][l] exactly as the copy engine writes it, so butterfly accesses of
// consecutive threads hit consecutive shared-memory words.
//
// MODE 0: one FFT in direction DIR.  MODE 1 (x-pass on psi): forward FFT,
// drift exp(-i s kappa^2)/N^3 from the separable tables, inverse FFT.
// MODE 2 (x-pass on the half spectrum): forward FFT, -1/kappa^2, inverse FFT.
#pragma once

#include "step_kernels.cuh"
#include "tma.cuh"

#include <type_traits>

namespace ifdm {

// R: element type in HBM (TMA landing ring), K: arithmetic type.  When they
// differ (mixed mode) the landing slot is converted into a separate FP64
// compute tile and freed before the transform.
// AXIS 2 tiles carry the x passes (two transforms each), AXIS 1 the y passes.
template <typename R, typename K, int N, int AXIS = 1> struct TmaTile {
    using G = cx<R>;
    using C = cx<K>;
    static constexpr bool SPLIT = !std::is_same<R, K>::value;
    // lines per tile: 128-byte rows, except for FP32 at N = 512: 8 lines (512
    // threads) capped at 64 registers so that two blocks share an SM (y
    // passes measured: P2/P4 0.531 -> 0.49 ms, P6/P8 0.30 -> 0.27 ms against
    // 16 lines, one block per SM).
    // 4-line x tiles, two blocks per SM at the same 128 registers (32-byte
    // TMA rows), measured slower: P3 0.92 -> 1.31 ms, P7 0.52 -> 0.59 ms.
    static constexpr bool NARROW = !SPLIT && sizeof(G) == 8 && N >= 512;
    // FP64 y passes at N = 512: 4 lines (64-byte rows, 256 threads) so that
    // two blocks share an SM at the same 128 registers (measured: P2/P4
    // 0.89 -> 0.85 ms, P6/P8 0.50 -> 0.45 ms; the FP64 x passes measured
    // slower that way: P3 1.39 -> 1.93 ms, P7 0.71 -> 0.78 ms)
    static constexpr bool NARROW64 = !SPLIT && sizeof(G) == 16 && AXIS == 1 && N >= 512;
    // N = 1024 (128 threads per line): one block per SM holds the ring; the
    // FP64 x tiles (two chained transforms) take half the y tiles' lines, 2,
    // which keeps them within the registers of their block size.  FP32 x
    // tiles take 8 lines like the y tiles: the two-lines-per-thread kernel
    // (k_yx_tma_pair, 512 threads) runs them; this one-line kernel (1024
    // threads, which spill 344 bytes a thread at 64 registers) only when
    // IFDM_NO_PAIR asks for it
    static constexpr bool BIG = N >= 1024;
    // resident blocks the registers must allow: two for the narrow tiles (the
    // FP32 x passes too since their twiddles come from shared memory: no
    // spills at 64 registers; measured at 512^3: P3 0.895 -> 0.877 ms, P7
    // 0.457 -> 0.433 ms)
    static constexpr int MINB = BIG ? 1 : (NARROW || NARROW64) ? 2 : 1;
    static constexpr int L = BIG ? (sizeof(G) == 16 ? 4 / (AXIS == 2 ? 2 : 1) : 8)
                                 : NARROW64 ? 4 : (SPLIT || NARROW) ? 8 : 128 / (int)sizeof(G);
    static constexpr bool SWZ = NARROW || NARROW64;  // slot swizzle of the exchange tile
    static constexpr int E = Plan<N>::E;
    static constexpr int T = N / E;
    static constexpr int NT = L * T;
    static constexpr int STAGES = 3;
    static constexpr int BOXR = N < 256 ? N : 256;               // rows per TMA box (limit 256)
    static constexpr size_t TILE_BYTES = size_t(N) * L * sizeof(G);
    // exchange tile between stages: the landing slot itself, or (mixed) a
    // separate FP64 tile.  (A separate tile with rows padded to L + 1 for the
    // narrow FP32 tiles, against their 2-way bank conflicts, measured slower:
    // P3 0.94 -> 0.99 ms at 512^3.)
    static constexpr bool OWN_WORK = SPLIT;
    static constexpr int LPW = L;
    static constexpr size_t WORK_BYTES = OWN_WORK ? size_t(N) * LPW * sizeof(C) : 0;
    // the N-point twiddle table, staged in shared memory once per CTA
    static constexpr size_t TWOFF = STAGES * TILE_BYTES + WORK_BYTES + 64;
    static constexpr size_t SMEM = TWOFF + tw_bytes<C>(N);
    static_assert(NT <= 1024, "block size");
    static_assert(SMEM <= 227 * 1024, "shared memory per block");
    static_assert(TWOFF % 16 == 0, "twiddle table alignment");
};

template <typename R, typename K, int N, int AXIS, int MODE, int DIR>
__global__ void __launch_bounds__(TmaTile<R, K, N, AXIS>::NT, TmaTile<R, K, N, AXIS>::MINB)
    k_yx_tma(const __grid_constant__ CUtensorMap map, cx<R> *__restrict__ data, int W, int VW, int ntiles,
             TState *__restrict__ ts, int pass, const cx<K> *__restrict__ drift, const cx<K> *__restrict__ tw) {
    using TL = TmaTile<R, K, N, AXIS>;
    using G = cx<R>;
    using C = cx<K>;
    constexpr int L = TL::L, T = TL::T, ST = TL::STAGES;
    extern __shared__ __align__(128) unsigned char smraw[];
    G *bufs = reinterpret_cast<G *>(smraw);
    C *work = reinterpret_cast<C *>(smraw + ST * TL::TILE_BYTES);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + ST * TL::TILE_BYTES + TL::WORK_BYTES);
    const int tid = threadIdx.x;
    const int l = tid % L;
    int *err = ts ? &ts->err : nullptr;
    if (tid == 0) {
        for (int s = 0; s < ST; ++s) mbar_init(&bar[s], 1);
        mbar_init_fence();
        prefetch_tmap(&map);
    }
    C *stw = reinterpret_cast<C *>(smraw + TL::TWOFF);
    stage_twiddles(stw, tw, N);
    const SmemTw<C> tws{stw};
    __syncthreads();
    const int my_n = blockIdx.x < (unsigned)ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto issue = [&](int i) {
        const long t = (long)blockIdx.x + (long)i * gridDim.x;
        const int s = i % ST;
        G *dst = bufs + (size_t)s * N * L;
        const long g0 = t * L;
        mbar_arrive_expect_tx(&bar[s], (uint32_t)TL::TILE_BYTES);
#pragma unroll
        for (int h = 0; h < N; h += TL::BOXR) {
            if (AXIS == 1) tma_load_3d(dst + (size_t)h * L, &map, 2 * int(g0 % W), h, int(g0 / W), &bar[s]);
            else tma_load_2d(dst + (size_t)h * L, &map, 2 * int(g0), h, &bar[s]);
        }
    };
    if (tid == 0)
        for (int i = 0; i < ST - 1 && i < my_n; ++i) issue(i);
    const uint32_t salt = ts ? pass_salt(ts, pass) : 0x2545f491u;
    const size_t S = AXIS == 1 ? size_t(W) : size_t(N) * W;
    for (int i = 0; i < my_n; ++i) {
        const int s = i % ST;
        if (tid == 0 && i + ST - 1 < my_n) issue(i + ST - 1);
        const bool ok = mbar_wait(&bar[s], (uint32_t)((i / ST) & 1), err, 2);
        if (!__syncthreads_and(ok)) {
            // a load never completed: wait (bounded) for the copies still in flight, then leave
            if (tid == 0)
                for (int j = i; j < my_n && j <= i + ST - 1; ++j)
                    mbar_wait(&bar[j % ST], (uint32_t)((j / ST) & 1), err, 2);
            __syncthreads();
            return;
        }
        const long g = ((long)blockIdx.x + (long)i * gridDim.x) * L + l;
        const int t = tid / L;
        constexpr int R0 = Plan<N>::R[0];
        constexpr int RL = Plan<N>::R[Plan<N>::NST - 1];
        constexpr int E = TL::E;
        C v[E];
        const G *land = bufs + (size_t)s * N * L;
        C *wk = TL::OWN_WORK ? work : reinterpret_cast<C *>(bufs + (size_t)s * N * L);
        constexpr int LPW = TL::LPW;
        // stage 0 straight from the landing slot
        stage_load<C, N, E, L, L, R0>(land, v, l, t);
        if constexpr (TL::OWN_WORK) fence_proxy_async_smem();  // slot is released at the next barrier
        stage_compute<C, N, E, (MODE == 0 ? DIR : -1), R0, 1>(v, tws, t);
        RegChain<C, N, E, (MODE == 0 ? DIR : -1), L, LPW, 1, R0, TL::SWZ>::run(wk, v, tws, l, t, true);
        if (MODE != 0) {
            // v[b*RL + r] holds element n = (t + T*b) + r*N/RL of the forward transform
            if (MODE == 1) {
                if (g == 0 && tid == 0) {
                    const double inv = 1.0 / ((double)N * N * N);
                    ts->cnext_re = ts->cre + (double)v[0].x * inv;
                    ts->cnext_im = ts->cim + (double)v[0].y * inv;
                }
                // drift factor d_x d_y d_z / N^3 and its product with psi in
                // FP64 whatever the storage type, rounded once: in FP32 the
                // three complex products of the factor and psi rounded three
                // times (measured at 256^3, g = 0, 1000 steps: density error
                // against FP64 1.055e-5 -> 9.97e-6; P3 +0.04 ms at 512^3)
                const int y = int(g / N), z = int(g % N);
                const C dy_ = __ldg(drift + y), dz_ = __ldg(drift + z);
                const double2 dyz = cmul(make_double2(dy_.x, dy_.y), make_double2(dz_.x, dz_.y));
                const double inv = 1.0 / ((double)N * N * N);
#pragma unroll
                for (int b = 0; b < E / RL; ++b)
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const int n = t + T * b + r * (N / RL);
                        const C dn_ = __ldg(drift + n);
                        const double2 f = cmul(dyz, make_double2(dn_.x * inv, dn_.y * inv));
                        const C vv = v[b * RL + r];
                        const double2 w = cmul(make_double2(vv.x, vv.y), f);
                        v[b * RL + r] = mkc((decltype(vv.x))w.x, (decltype(vv.x))w.y);
                    }
            } else {
                const int y = int(g / W), kz = int(g % W);
                const int ky = kappa(y, N), kzz = kappa(kz, N);
                const int k2yz = ky * ky + kzz * kzz;
#pragma unroll
                for (int b = 0; b < E / RL; ++b)
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const int kx = kappa(t + T * b + r * (N / RL), N);
                        const int k2 = kx * kx + k2yz;
                        v[b * RL + r] = cscale(v[b * RL + r], k2 == 0 ? K(0) : K(-1) / K(k2));
                    }
            }
            fft_regs_chained<C, N, E, +1, L, LPW, TL::SWZ>(wk, v, tws, l, t, true);
        }
        if ((g % W) < VW) {
            const size_t b0 = AXIS == 1 ? size_t(g / W) * N * W + size_t(g % W) : size_t(g);
#pragma unroll
            for (int b = 0; b < E / RL; ++b)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const size_t gi = b0 + size_t(t + T * b + r * (N / RL)) * S;
                    data[gi] = Cvt<R, K>::out(v[b * RL + r], salt, gi);
                }
        }
        fence_proxy_async_smem();
        __syncthreads();
    }
}

// FP32 y/x passes with two lines per thread (fft_engine.cuh, *_pair): the
// same 8-line tiles, tensor maps, modes and arithmetic as k_yx_tma<float,
// float, N>, with 256 threads per tile and 128-bit exchanges, twiddle loads
// shared by two lines and 16-byte global stores.  ST ring slots, MINB
// resident blocks per SM.
template <int N, int ST, int MINB> struct TmaPair {
    static constexpr int L = 8, LH = L / 2;
    static constexpr int E = Plan<N>::E, T = N / E, NT = LH * T;
    static constexpr int BOXR = N < 256 ? N : 256;
    static constexpr size_t TILE_BYTES = size_t(N) * L * sizeof(float2);
    static constexpr size_t TWOFF = ST * TILE_BYTES + 64;
    static constexpr size_t SMEM = TWOFF + tw_bytes<float2>(N);  // room for either table
    static_assert(staged_tw_bytes<N>() <= tw_bytes<float2>(N), "per-stage tables fit the flat table's room");
    static_assert(Plan<N>::R[0] == Plan<N>::R[Plan<N>::NST - 1], "chained transforms need equal first/last radix");
    static_assert(SMEM <= 227 * 1024, "shared memory per block");
};

template <int N, int AXIS, int MODE, int DIR, int ST, int MINB>
__global__ void __launch_bounds__(TmaPair<N, ST, MINB>::NT, MINB)
    k_yx_tma_pair(const __grid_constant__ CUtensorMap map, float2 *__restrict__ data, int W, int VW, int ntiles,
                  TState *__restrict__ ts, const float2 *__restrict__ drift, const float2 *__restrict__ tw) {
    using TP = TmaPair<N, ST, MINB>;
    constexpr int L = TP::L, LH = TP::LH, T = TP::T, E = TP::E;
    constexpr int R0 = Plan<N>::R[0];
    constexpr int SW = 1;  // the slot swizzle of the 8-line FP32 exchange tile (fft_engine.cuh)
    extern __shared__ __align__(128) unsigned char smraw[];
    float2 *bufs = reinterpret_cast<float2 *>(smraw);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + ST * TP::TILE_BYTES);
    const int tid = threadIdx.x;
    const int lp = tid % LH, t = tid / LH;
    int *err = ts ? &ts->err : nullptr;
    if (tid == 0) {
        for (int s = 0; s < ST; ++s) mbar_init(&bar[s], 1);
        mbar_init_fence();
        prefetch_tmap(&map);
    }
    // x passes: per-stage twiddle tables; y passes: the flat table (measured
    // at 512^3 with per-stage tables: P3 0.754 -> 0.704 ms, P7 0.363 -> 0.338
    // ms, but P2/P4 0.392 -> 0.43 ms, P6/P8 0.211 -> 0.22 ms)
    using TWT = std::conditional_t<AXIS == 2, StagedTw<N>, SmemTw<float2>>;
    unsigned char *stw = smraw + TP::TWOFF;
    if constexpr (AXIS == 2) stage_twiddles_staged<N>(reinterpret_cast<float4 *>(stw), tw);
    else stage_twiddles(reinterpret_cast<float2 *>(stw), tw, N);
    const TWT tws{reinterpret_cast<decltype(TWT::p)>(stw)};
    __syncthreads();
    const int my_n = blockIdx.x < (unsigned)ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto issue = [&](int i) {
        const long tile = (long)blockIdx.x + (long)i * gridDim.x;
        const int s = i % ST;
        float2 *dst = bufs + (size_t)s * N * L;
        const long g0 = tile * L;
        mbar_arrive_expect_tx(&bar[s], (uint32_t)TP::TILE_BYTES);
#pragma unroll
        for (int h = 0; h < N; h += TP::BOXR) {
            if (AXIS == 1) tma_load_3d(dst + (size_t)h * L, &map, 2 * int(g0 % W), h, int(g0 / W), &bar[s]);
            else tma_load_2d(dst + (size_t)h * L, &map, 2 * int(g0), h, &bar[s]);
        }
    };
    if (tid == 0)
        for (int i = 0; i < ST - 1 && i < my_n; ++i) issue(i);
    const size_t S = AXIS == 1 ? size_t(W) : size_t(N) * W;
    for (int i = 0; i < my_n; ++i) {
        const int s = i % ST;
        if (tid == 0 && i + ST - 1 < my_n) issue(i + ST - 1);
        const bool ok = mbar_wait(&bar[s], (uint32_t)((i / ST) & 1), err, 2);
        if (!__syncthreads_and(ok)) {
            // a load never completed: wait (bounded) for the copies still in flight, then leave
            if (tid == 0)
                for (int j = i; j < my_n && j <= i + ST - 1; ++j)
                    mbar_wait(&bar[j % ST], (uint32_t)((j / ST) & 1), err, 2);
            __syncthreads();
            return;
        }
        // line g holds va, line g + 1 vb: W and L are even, so both lie in one row
        const long g = ((long)blockIdx.x + (long)i * gridDim.x) * L + 2 * lp;
        float2 va[E], vb[E];
        float4 *wk = reinterpret_cast<float4 *>(bufs + (size_t)s * N * L);
        stage_load_pair<N, E, LH, R0>(wk, va, vb, lp, t);
        stage_compute_pair<N, E, (MODE == 0 ? DIR : -1), R0, 1>(va, vb, tws, t);
        RegChainPair<N, E, (MODE == 0 ? DIR : -1), LH, 1, R0, SW>::run(wk, va, vb, tws, lp, t);
        if (MODE != 0) {
            // va[b*R0 + r] holds element n = (t + T*b) + r*N/R0 of the forward transform
            if (MODE == 1) {
                if (g == 0 && tid == 0) {
                    const double inv = 1.0 / ((double)N * N * N);
                    ts->cnext_re = ts->cre + (double)va[0].x * inv;
                    ts->cnext_im = ts->cim + (double)va[0].y * inv;
                }
                // the drift factor and its product with psi in FP64 (as k_yx_tma)
                const int y = int(g / N), z = int(g % N);
                const double inv = 1.0 / ((double)N * N * N);
                const float2 dyf = __ldg(drift + y), dza = __ldg(drift + z), dzb = __ldg(drift + z + 1);
                const double2 dy2 = make_double2(dyf.x * inv, dyf.y * inv);
                const double2 lfa = cmul(dy2, make_double2(dza.x, dza.y)), lfb = cmul(dy2, make_double2(dzb.x, dzb.y));
#pragma unroll
                for (int b = 0; b < E / R0; ++b)
#pragma unroll
                    for (int r = 0; r < R0; ++r) {
                        const int n = t + T * b + r * (N / R0);
                        const float2 dn = __ldg(drift + n);
                        const double2 dd = make_double2(dn.x, dn.y);
                        const double2 fa = cmul(lfa, dd), fb = cmul(lfb, dd);
                        const float2 xa = va[b * R0 + r], xb = vb[b * R0 + r];
                        const double2 wa = cmul(make_double2(xa.x, xa.y), fa), wb = cmul(make_double2(xb.x, xb.y), fb);
                        va[b * R0 + r] = make_float2((float)wa.x, (float)wa.y);
                        vb[b * R0 + r] = make_float2((float)wb.x, (float)wb.y);
                    }
            } else {
                const int y = int(g / W), kz = int(g % W);
                const int ky = kappa(y, N), ka = kappa(kz, N), kb = kappa(kz + 1, N);
                const int k2a = ky * ky + ka * ka, k2b = ky * ky + kb * kb;
#pragma unroll
                for (int b = 0; b < E / R0; ++b)
#pragma unroll
                    for (int r = 0; r < R0; ++r) {
                        const int kx = kappa(t + T * b + r * (N / R0), N);
                        const int ea = kx * kx + k2a, eb = kx * kx + k2b;
                        va[b * R0 + r] = cscale(va[b * R0 + r], ea == 0 ? 0.0f : -1.0f / float(ea));
                        vb[b * R0 + r] = cscale(vb[b * R0 + r], eb == 0 ? 0.0f : -1.0f / float(eb));
                    }
            }
            stage_compute_pair<N, E, +1, R0, 1>(va, vb, tws, t);
            RegChainPair<N, E, +1, LH, 1, R0, SW>::run(wk, va, vb, tws, lp, t);
        }
        const int ca = int(g % W);
        if (ca < VW) {
            const size_t b0 = AXIS == 1 ? size_t(g / W) * N * W + size_t(ca) : size_t(g);
            const bool both = ca + 1 < VW;
#pragma unroll
            for (int b = 0; b < E / R0; ++b)
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const size_t gi = b0 + size_t(t + T * b + r * (N / R0)) * S;
                    const float2 a = va[b * R0 + r], c = vb[b * R0 + r];
                    if (both) *reinterpret_cast<float4 *>(data + gi) = make_float4(a.x, a.y, c.x, c.y);
                    else data[gi] = a;
                }
        }
        fence_proxy_async_smem();
        __syncthreads();
    }
}

}  // namespace ifdm
