// zpass_pipe.cuh -- persistent P5 z-pass with a two-slot cp.async pipeline.
//
// Same transform as k_density_r2c_z of step_kernels.cuh (inverse FFT along z,
// density, real-to-half FFT), for R == K and N >= 128.  Each CTA loops over
// its tiles; while it transforms tile i, every thread's asynchronous copies of
// tile i+1 are in flight into the other slot, landing directly in the padded,
// transposed [n][l] layout.  cp.async.wait_group waits in hardware (no spin in
// this code).
#pragma once

#include "step_kernels.cuh"
#include "tma.cuh"

namespace ifdm {

// The tile of the y/x passes (16 FP32 lines, 1024 threads, one block per SM).
// Half the lines under a 64-register cap (two blocks per SM, as the FP32 y
// passes use) spilled and measured slower at 512^3: 1.03 -> 1.46 ms.
template <typename R, int N> struct ZPipe {
    using TL = Tile<R, R, N>;
    using C = cx<R>;
    static constexpr int L = TL::L, LP = TL::LP, E = TL::E, NT = TL::NT, EH = TL::EH;
    static constexpr size_t TILE = size_t(N) * LP * sizeof(C);  // one slot
    static constexpr size_t SMEM5 = 2 * TILE;
    static_assert(SMEM5 <= 227 * 1024, "shared memory per block");
};

__device__ __forceinline__ int tiles_of_block(int ntiles) {
    return (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
}

// P5: inverse FFT z, psi = IFFT + c, rho = |psi|^2 - mu, max |psi|^2, r2c along z.
template <typename R, int N>
__global__ void __launch_bounds__(ZPipe<R, N>::NT, 1)
    k_density_r2c_z_pipe(cx<R> *__restrict__ psi, cx<R> *__restrict__ rhok, TState *__restrict__ ts,
                         const cx<R> *__restrict__ tw, const cx<R> *__restrict__ twh, int ntiles) {
    using ZP = ZPipe<R, N>;
    using C = cx<R>;
    constexpr int L = ZP::L, LP = ZP::LP, NT = ZP::NT;
    constexpr int NH = N / 2 + 1, NHP = half_pitch<R>(N), M = N / 2;
    extern __shared__ __align__(128) unsigned char smraw[];
    C *buf = reinterpret_cast<C *>(smraw);
    const int tid = threadIdx.x;
    const int my_n = tiles_of_block(ntiles);
    auto issue = [&](int i) {
        const size_t base = size_t(blockIdx.x + (long)i * gridDim.x) * L * N;
        C *dst = buf + (size_t)(i & 1) * N * LP;
        for (int f = tid; f < L * N; f += NT) cp_async<sizeof(C)>(&dst[(f % N) * LP + f / N], &psi[base + f]);
    };
    if (my_n > 0) issue(0);
    cp_async_commit();
    const double mu = ts->mu;
    const C c0 = mkc((R)ts->cre, (R)ts->cim);
    double mx = 0.0;
    for (int i = 0; i < my_n; ++i) {
        if (i + 1 < my_n) issue(i + 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        C *sm = buf + (size_t)(i & 1) * N * LP;
        const size_t row0 = size_t(blockIdx.x + (long)i * gridDim.x) * L;
        const size_t base = row0 * N;
        fft_tile<C, N, ZP::E, +1, L, LP>(sm, tw);
        R rho[ZP::E];
#pragma unroll
        for (int e = 0; e < ZP::E; ++e) {
            const int f = tid + e * NT;
            const C v = sm[(f % N) * LP + f / N] + c0;
            psi[base + f] = v;
            const double n2 = (double)cnorm2(v);
            mx = fmax(mx, n2);
            rho[e] = (R)(n2 - mu);
        }
        __syncthreads();
        R *smr = reinterpret_cast<R *>(sm);
#pragma unroll
        for (int e = 0; e < ZP::E; ++e) {
            const int f = tid + e * NT;
            const int l = f / N, n = f % N;
            smr[2 * ((n >> 1) * LP + l) + (n & 1)] = rho[e];
        }
        __syncthreads();
        fft_tile<C, M, ZP::EH, -1, L, LP, typename ZP::TL::HP>(sm, twh);
        constexpr int TPR = NT / L;  // threads per row: no division by N/2+1
        static_assert(TPR * L == NT, "whole rows per thread block");
        const int l = tid / TPR;
        for (int k = tid % TPR; k < NH; k += TPR) {
            const C zk = sm[(k % M) * LP + l];
            const C zc = cconj(sm[((M - k) % M) * LP + l]);
            const C e = cscale(zk + zc, R(0.5));
            const C o = cscale(zk - zc, R(0.5));
            const C wo = post_tw<-1, N>(tw, k % N, o);
            rhok[(row0 + l) * NHP + k] = mkc(e.x + wo.y, e.y - wo.x);
        }
        __syncthreads();
    }
    mx = warp_max(mx);
    if ((tid & 31) == 0 && my_n > 0) atomic_max_nonneg(&ts->maxrho_bits, mx);
}

}  // namespace ifdm
