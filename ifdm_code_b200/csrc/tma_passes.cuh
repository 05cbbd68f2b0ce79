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

namespace ifdm {

template <typename R, int N> struct TmaTile {
    using C = cx<R>;
    static constexpr int L = 128 / (int)sizeof(C);   // 8 complex doubles or 16 complex floats
    static constexpr int E = Plan<N>::E;
    static constexpr int T = N / E;
    static constexpr int NT = L * T;
    static constexpr int STAGES = 3;
    static constexpr int BOXR = N < 256 ? N : 256;    // rows per TMA box (limit 256)
    static constexpr size_t TILE_BYTES = size_t(N) * L * sizeof(C);
    static constexpr size_t SMEM = STAGES * TILE_BYTES + 64;
    static_assert(NT <= 1024, "block size");
};

template <typename R, int N, int AXIS, int MODE, int DIR>
__global__ void __launch_bounds__(TmaTile<R, N>::NT, 1)
    k_yx_tma(const __grid_constant__ CUtensorMap map, cx<R> *__restrict__ data, int W, int VW, int ntiles,
             TState *__restrict__ ts, int pass, const cx<R> *__restrict__ drift, const cx<R> *__restrict__ tw) {
    using TL = TmaTile<R, N>;
    using C = cx<R>;
    constexpr int L = TL::L, T = TL::T, ST = TL::STAGES;
    extern __shared__ __align__(128) unsigned char smraw[];
    C *bufs = reinterpret_cast<C *>(smraw);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + ST * TL::TILE_BYTES);
    const int tid = threadIdx.x;
    const int l = tid % L;
    int *err = ts ? &ts->err : nullptr;
    if (tid == 0) {
        for (int s = 0; s < ST; ++s) mbar_init(&bar[s], 1);
        mbar_init_fence();
        prefetch_tmap(&map);
    }
    __syncthreads();
    const int my_n = blockIdx.x < (unsigned)ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto issue = [&](int i) {
        const long t = (long)blockIdx.x + (long)i * gridDim.x;
        const int s = i % ST;
        C *dst = bufs + (size_t)s * N * L;
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
    (void)pass;
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
        C *sm = bufs + (size_t)s * N * L;
        const long g = ((long)blockIdx.x + (long)i * gridDim.x) * L + l;
        if (MODE == 0) {
            fft_tile<C, N, TL::E, DIR, L, L>(sm, tw);
        } else {
            fft_tile<C, N, TL::E, -1, L, L>(sm, tw);
            if (MODE == 1) {
                if (g == 0 && tid == 0) {
                    const double inv = 1.0 / ((double)N * N * N);
                    ts->cnext_re = ts->cre + (double)sm[0].x * inv;
                    ts->cnext_im = ts->cim + (double)sm[0].y * inv;
                }
                const int y = int(g / N), z = int(g % N);
                const C lf = cscale(cmul(__ldg(drift + y), __ldg(drift + z)), R(1.0 / ((double)N * N * N)));
                for (int n = tid / L; n < N; n += T) sm[n * L + l] = cmul(sm[n * L + l], cmul(lf, __ldg(drift + n)));
            } else {
                const int y = int(g / W), kz = int(g % W);
                const int ky = kappa(y, N), kzz = kappa(kz, N);
                const int k2yz = ky * ky + kzz * kzz;
                for (int n = tid / L; n < N; n += T) {
                    const int kx = kappa(n, N);
                    const int k2 = kx * kx + k2yz;
                    sm[n * L + l] = cscale(sm[n * L + l], k2 == 0 ? R(0) : R(-1) / R(k2));
                }
            }
            __syncthreads();
            fft_tile<C, N, TL::E, +1, L, L>(sm, tw);
        }
        if ((g % W) < VW) {
            const size_t b = AXIS == 1 ? size_t(g / W) * N * W + size_t(g % W) : size_t(g);
            for (int n = tid / L; n < N; n += T) data[b + n * S] = sm[n * L + l];
        }
        fence_proxy_async_smem();
        __syncthreads();
    }
}

}  // namespace ifdm
