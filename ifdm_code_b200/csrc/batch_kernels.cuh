// batch_kernels.cuh -- many independent boxes advanced by one persistent kernel.
//
// The work of a step of box b is a list of items: the timestep (one item),
// then the tiles of passes P1..P9 (the same fused passes as step_kernels.cuh,
// with the same tile shapes, so each box's arithmetic is that of a one-box
// run).  A batch step is the concatenation of all boxes' items in an order
// chosen on the host (segments of (box, phase) tiles).  Persistent CTAs claim
// items in that global order from one atomic counter; an item of box b in
// phase p of step s may start once box b has completed every item of its
// earlier phases and steps, which is one counter per box:
//   done[b] >= s * step_items[b] + prefix[b][p].
// Each box size has its own launch, item list and counters.
// Items are claimed in increasing order and only wait for items of smaller
// index, which are held by CTAs already running, so the wait always ends.
// Waits are bounded anyway: a wait that gives up sets *status, after which no
// item waits or computes (the host reports a device error).
//
// Everything one item writes (psi, phi, the half spectrum, the TState, the
// drift tables) is read by later items of the same launch on other SMs, so
// those reads use plain coherent loads: no read-only cache (__ldg) and no
// const __restrict__ on produced data.  The producing CTA releases with a
// fence and a release add after a block barrier; the consumer's thread 0
// acquires the counter before a block barrier.
#pragma once

#include "step_kernels.cuh"
#include "timestep.cuh"
#include "tma.cuh"

namespace ifdm {

constexpr int kBatchThreads = 256;
constexpr int kBatchPhases = 10;  // timestep, P1..P9

struct BatchBox {
    int N;           // grid size
    int win_tail;    // max|phi| scan window (see k_c2r_z_phi)
    int step_items;  // items of one step of this box
    long win_rows;
    void *psi, *phi, *rhok;  // storage type R
    const void *tw, *twh;    // twiddles, arithmetic type K (N and N/2)
    TState *ts;
    double2 *drift64;
    float2 *drift32;
    Phys ph;                          // constants of the timestep (dt_scale included)
    int prefix[kBatchPhases + 1];     // items of this box before phase p within a step
};

// A run of consecutive items: `count` tiles of phase `phase` of box `box`,
// starting at item `first` of a step.
struct BatchSeg {
    int box, phase, first, count;
};

struct BatchArgs {
    const BatchBox *boxes;
    const BatchSeg *segs;
    int nsegs;
    long long step_items;      // items of one step of all boxes
    long long total;           // step_items * steps of this launch
    unsigned long long *next;  // claim counter (0 at launch)
    unsigned long long *done;  // completed items per box (0 at launch)
    int *status;               // 0 ok, 1 a dependency wait gave up
};

// Items of phase p of one box: 1 for the timestep, else the tiles of the pass.
template <typename R, typename K, int N> __host__ __device__ constexpr int batch_items(int p) {
    using TL = Tile<R, K, N>;
    using TZ = TileZ<R, K, N>;
    constexpr int NHP = half_pitch<R>(N);
    switch (p) {
        case 0: return 1;
        case 1: case 5: case 9: return N * N / TZ::L;
        case 2: case 3: case 4: return N * N / TL::L;
        default: return N * NHP / TL::L;  // 6, 7, 8: half spectrum
    }
}

// Largest dynamic shared memory of any pass of an N-box.
template <typename R, typename K, int N> __host__ __device__ constexpr size_t batch_smem() {
    return TileZ<R, K, N>::SMEM9 > Tile<R, K, N>::SMEM ? TileZ<R, K, N>::SMEM9 : Tile<R, K, N>::SMEM;
}

__device__ __forceinline__ int batch_wait(unsigned long long *ctr, unsigned long long need, int *status) {
    for (uint32_t i = 0; i < kMaxSpins; ++i) {
        unsigned long long v;
        asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(ctr) : "memory");
        if (v >= need) return 1;
        if (*(volatile int *)status) return 0;
        if (i > 32) __nanosleep(i > 4096 ? 256 : 64);
    }
    atomicExch(status, 1);
    return 0;
}

__device__ __forceinline__ void batch_release(unsigned long long *ctr) {
    __threadfence();
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(ctr), "l"(1ull) : "memory");
}

// The passes of one N-box on one tile; P: radix plan of the full-length transforms.
template <typename R, typename K, int N, class P> struct BatchOps {
    using TL = Tile<R, K, N>;
    using TZ = TileZ<R, K, N>;
    using C = cx<K>;
    using G = cx<R>;
    static constexpr int NH = N / 2 + 1, NHP = half_pitch<R>(N), M = N / 2;
    static_assert(TL::NT == kBatchThreads && TZ::NT == kBatchThreads, "batch tiles use the batch block size");
    static_assert(P::E == Plan<N>::E, "plan variants keep the elements per thread");

    // P1: kick with the merged coefficients, remove the offset c, FFT along z
    __device__ __forceinline__ static void kick_fft_z(C *sm, const BatchBox &bx, int tile) {
        G *psi = (G *)bx.psi;
        const R *phi = (const R *)bx.phi;
        const TState *ts = bx.ts;
        const C *tw = (const C *)bx.tw;
        const double cp = ts->coefP, cq = ts->coefQ, alpha = ts->alpha;
        const C c0 = mkc((K)ts->cre, (K)ts->cim);
        const uint32_t salt = pass_salt(ts, 1);
        const size_t base = size_t(tile) * TZ::L * N;
        for (int f = threadIdx.x; f < TZ::L * N; f += TZ::NT) {
            const C v = cin<K>(psi[base + f]);
            const double p = cp * (double)phi[base + f] + cq * (double)cnorm2(v) + alpha;
            sm[(f % N) * TZ::LP + f / N] = cmul(v, expmi<K>(p)) - c0;
        }
        __syncthreads();
        fft_tile<C, N, TZ::E, -1, TZ::L, TZ::LP, P>(sm, tw);
        for (int f = threadIdx.x; f < TZ::L * N; f += TZ::NT)
            psi[base + f] = Cvt<R, K>::out(sm[(f % N) * TZ::LP + f / N], salt, base + f);
    }

    // P2/P4 (W = VW = N) and P6/P8 (half spectrum, W = NHP, VW = NH): FFT along y
    template <int DIR>
    __device__ __forceinline__ static void fft_y(C *sm, G *data, int W, int VW, const TState *ts, int pass, const C *tw, int tile) {
        const int l = threadIdx.x % TL::L;
        const long g = long(tile) * TL::L + l;
        const bool valid = (g % W) < VW;
        const size_t b = size_t(g / W) * N * W + size_t(g % W);
        const size_t S = size_t(W);
        const uint32_t salt = pass_salt(ts, pass);
        for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
            sm[n * TL::LP + l] = valid ? cin<K>(data[b + n * S]) : mkc(K(0), K(0));
        __syncthreads();
        fft_tile<C, N, TL::E, DIR, TL::L, TL::LP, P>(sm, tw);
        if (valid)
            for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
                data[b + n * S] = Cvt<R, K>::out(sm[n * TL::LP + l], salt, b + n * S);
    }

    // P3: FFT along x, drift exp(-i s kappa^2) / N^3, inverse FFT along x
    __device__ __forceinline__ static void fft_x_drift(C *sm, const BatchBox &bx, int tile) {
        G *psi = (G *)bx.psi;
        TState *ts = bx.ts;
        const C *tw = (const C *)bx.tw;
        const C *drift = sizeof(K) == 8 ? (const C *)(const void *)bx.drift64 : (const C *)(const void *)bx.drift32;
        const int l = threadIdx.x % TL::L;
        const long q = long(tile) * TL::L + l;
        const size_t S = size_t(N) * N;
        const uint32_t salt = pass_salt(ts, 3);
        for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L) sm[n * TL::LP + l] = cin<K>(psi[q + n * S]);
        __syncthreads();
        fft_tile<C, N, TL::E, -1, TL::L, TL::LP, P>(sm, tw);
        if (q == 0 && threadIdx.x == 0) {
            const double inv = 1.0 / ((double)N * N * N);
            ts->cnext_re = ts->cre + (double)sm[0].x * inv;
            ts->cnext_im = ts->cim + (double)sm[0].y * inv;
        }
        const int y = int(q / N), z = int(q % N);
        constexpr KSplit<K> inv3(1.0 / ((double)N * N * N));
        const C dyz = cmul(drift[y], drift[z]);
        const C lf = mkc(mulk(dyz.x, inv3.hi, inv3.lo), mulk(dyz.y, inv3.hi, inv3.lo));
        for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
            sm[n * TL::LP + l] = cmul(sm[n * TL::LP + l], cmul(lf, drift[n]));
        __syncthreads();
        fft_tile<C, N, TL::E, +1, TL::L, TL::LP, P>(sm, tw);
        for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
            psi[q + n * S] = Cvt<R, K>::out(sm[n * TL::LP + l], salt, q + n * S);
    }

    // P5: inverse FFT along z, + c, density, max, real-to-half FFT along z
    __device__ __forceinline__ static void density_r2c_z(C *sm, const BatchBox &bx, int tile) {
        G *psi = (G *)bx.psi;
        G *rhok = (G *)bx.rhok;
        TState *ts = bx.ts;
        const C *tw = (const C *)bx.tw;
        const C *twh = (const C *)bx.twh;
        const size_t row0 = size_t(tile) * TZ::L;
        const size_t base = row0 * N;
        const uint32_t salt = pass_salt(ts, 5), salt2 = pass_salt(ts, 10);
        for (int f = threadIdx.x; f < TZ::L * N; f += TZ::NT) sm[(f % N) * TZ::LP + f / N] = cin<K>(psi[base + f]);
        __syncthreads();
        fft_tile<C, N, TZ::E, +1, TZ::L, TZ::LP, P>(sm, tw);
        K rho[TZ::E];
        double mx = 0.0;
        const double mu = ts->mu;
        const C c0 = mkc((K)ts->cre, (K)ts->cim);
#pragma unroll
        for (int i = 0; i < TZ::E; ++i) {
            const int f = threadIdx.x + i * TZ::NT;
            const G g = Cvt<R, K>::out(sm[(f % N) * TZ::LP + f / N] + c0, salt, base + f);
            psi[base + f] = g;
            const C v = cin<K>(g);
            const double n2 = (double)cnorm2(v);
            mx = fmax(mx, n2);
            rho[i] = (K)(n2 - mu);
        }
        mx = warp_max(mx);
        if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&ts->maxrho_bits, mx);
        __syncthreads();
        K *smr = reinterpret_cast<K *>(sm);
#pragma unroll
        for (int i = 0; i < TZ::E; ++i) {
            const int f = threadIdx.x + i * TZ::NT;
            const int l = f / N, n = f % N;
            smr[2 * ((n >> 1) * TZ::LP + l) + (n & 1)] = rho[i];
        }
        __syncthreads();
        fft_tile<C, M, TZ::EH, -1, TZ::L, TZ::LP, typename TZ::HP>(sm, twh);
        constexpr int TPR = TZ::NT / TZ::L;  // threads per row: no division by N/2+1
        static_assert(TPR * TZ::L == TZ::NT, "whole rows per thread block");
        const int l = threadIdx.x / TPR;
        for (int k = threadIdx.x % TPR; k < NH; k += TPR) {
            const C zk = sm[(k % M) * TZ::LP + l];
            const C zc = cconj(sm[((M - k) % M) * TZ::LP + l]);
            const C e = cscale(zk + zc, K(0.5));
            const C o = cscale(zk - zc, K(0.5));
            const C wo = post_tw<-1, N>(tw, k % N, o);
            const size_t gi = (row0 + l) * NHP + k;
            rhok[gi] = Cvt<R, K>::out(mkc(e.x + wo.y, e.y - wo.x), salt2, gi);
        }
    }

    // P7: FFT along x on the half spectrum, -1/kappa^2, inverse FFT along x
    __device__ __forceinline__ static void fft_x_poisson(C *sm, const BatchBox &bx, int tile) {
        G *rhok = (G *)bx.rhok;
        const TState *ts = bx.ts;
        const C *tw = (const C *)bx.tw;
        const int l = threadIdx.x % TL::L;
        const long q = long(tile) * TL::L + l;
        const int y = int(q / NHP), kz = int(q % NHP);
        const bool valid = kz < NH;
        const size_t S = size_t(N) * NHP;
        const uint32_t salt = pass_salt(ts, 7);
        for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
            sm[n * TL::LP + l] = valid ? cin<K>(rhok[q + n * S]) : mkc(K(0), K(0));
        __syncthreads();
        fft_tile<C, N, TL::E, -1, TL::L, TL::LP, P>(sm, tw);
        const int ky = kappa(y, N), kzz = kappa(kz, N);
        const int k2yz = ky * ky + kzz * kzz;
        for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L) {
            const int kx = kappa(n, N);
            const int k2 = kx * kx + k2yz;
            const K m = k2 == 0 ? K(0) : K(-1) / K(k2);
            sm[n * TL::LP + l] = cscale(sm[n * TL::LP + l], m);
        }
        __syncthreads();
        fft_tile<C, N, TL::E, +1, TL::L, TL::LP, P>(sm, tw);
        if (valid)
            for (int n = threadIdx.x / TL::L; n < N; n += TL::NT / TL::L)
                rhok[q + n * S] = Cvt<R, K>::out(sm[n * TL::LP + l], salt, q + n * S);
    }

    // P9: half-complex-to-real FFT along z, /N^3 -> phi, max|phi| over the scan window
    __device__ __forceinline__ static void c2r_z_phi(C *sm, const BatchBox &bx, int tile) {
        const G *rhok = (const G *)bx.rhok;
        R *phi = (R *)bx.phi;
        TState *ts = bx.ts;
        const C *tw = (const C *)bx.tw;
        const C *twh = (const C *)bx.twh;
        C *xs = sm + M * TZ::LP;
        const size_t row0 = size_t(tile) * TZ::L;
        const uint32_t salt = pass_salt(ts, 9);
        {
            constexpr int TPR = TZ::NT / TZ::L;  // threads per row
            const int l = threadIdx.x / TPR;
            for (int k = threadIdx.x % TPR; k <= M; k += TPR) {
                C x = cin<K>(rhok[(row0 + l) * NHP + k]);
                if (k == 0 || k == M) x.y = K(0);
                xs[k * TZ::LP + l] = x;
            }
        }
        __syncthreads();
        for (int f = threadIdx.x; f < TZ::L * M; f += TZ::NT) {
            const int l = f % TZ::L, k = f / TZ::L;
            const C xk = xs[k * TZ::LP + l];
            const C xc = cconj(xs[(M - k) * TZ::LP + l]);
            const C e = xk + xc;
            const C d = post_tw<+1, N>(tw, k, xk - xc);
            sm[k * TZ::LP + l] = mkc(e.x - d.y, e.y + d.x);
        }
        __syncthreads();
        fft_tile<C, M, TZ::EHD, +1, TZ::L, TZ::LP>(sm, twh);
        const K *smr = reinterpret_cast<const K *>(sm);
        constexpr KSplit<K> inv(1.0 / ((double)N * N * N));
        // the scan window as one limit per tile, the running max on the pipe
        // the pass leaves idle (as in the one-box c2r pass)
        R *out = phi + row0 * N;
        const bool inside = (long)(row0 + TZ::L) <= bx.win_rows;
        const int lim =
            inside ? TZ::L * N : (int)max(0L, min((long)TZ::L * N, (bx.win_rows - (long)row0) * N + bx.win_tail));
        using MX = std::conditional_t<sizeof(K) == 4, double, R>;
        MX mx = MX(0);
        for (int f = threadIdx.x; f < TZ::L * N; f += TZ::NT) {
            const int l = f / N, n = f % N;
            const R v = Cvt<R, K>::outr(mulk(smr[2 * ((n >> 1) * TZ::LP + l) + (n & 1)], inv.hi, inv.lo), salt,
                                        row0 * N + f);
            out[f] = v;
            if (f < lim) mx = fmax(mx, (MX)fabs(v));
        }
        const double m = warp_max((double)mx);
        if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&ts->maxphi_bits, m);
    }

    // one phase of one tile, chosen at compile time
    template <int PH> __device__ __forceinline__ static void phase(unsigned char *smraw, const BatchBox &bx, int tile) {
        C *sm = reinterpret_cast<C *>(smraw);
        const TState *ts = bx.ts;
        if constexpr (PH == 0) timestep_body(bx.ts, bx.ph, bx.drift64, bx.drift32);
        else if constexpr (PH == 1) kick_fft_z(sm, bx, tile);
        else if constexpr (PH == 2) fft_y<-1>(sm, (G *)bx.psi, N, N, ts, 2, (const C *)bx.tw, tile);
        else if constexpr (PH == 3) fft_x_drift(sm, bx, tile);
        else if constexpr (PH == 4) fft_y<+1>(sm, (G *)bx.psi, N, N, ts, 4, (const C *)bx.tw, tile);
        else if constexpr (PH == 5) density_r2c_z(sm, bx, tile);
        else if constexpr (PH == 6) fft_y<-1>(sm, (G *)bx.rhok, NHP, NH, ts, 6, (const C *)bx.tw, tile);
        else if constexpr (PH == 7) fft_x_poisson(sm, bx, tile);
        else if constexpr (PH == 8) fft_y<+1>(sm, (G *)bx.rhok, NHP, NH, ts, 8, (const C *)bx.tw, tile);
        else if constexpr (PH == 9) c2r_z_phi(sm, bx, tile);
    }

    // The persistent kernel reaches the phases through calls: inlining all ten
    // bodies into one loop makes the register allocator spill kilobytes per
    // thread, while each body alone fits in ~64 registers.
    template <int PH> __device__ __noinline__ static void phase_call(unsigned char *smraw, const BatchBox &bx, int tile) {
        phase<PH>(smraw, bx, tile);
    }

    __device__ __forceinline__ static void run(unsigned char *smraw, const BatchBox &bx, int ph, int tile) {
        switch (ph) {
            case 0: phase_call<0>(smraw, bx, tile); break;
            case 1: phase_call<1>(smraw, bx, tile); break;
            case 2: phase_call<2>(smraw, bx, tile); break;
            case 3: phase_call<3>(smraw, bx, tile); break;
            case 4: phase_call<4>(smraw, bx, tile); break;
            case 5: phase_call<5>(smraw, bx, tile); break;
            case 6: phase_call<6>(smraw, bx, tile); break;
            case 7: phase_call<7>(smraw, bx, tile); break;
            case 8: phase_call<8>(smraw, bx, tile); break;
            case 9: phase_call<9>(smraw, bx, tile); break;
            default: break;
        }
    }
};

// One persistent kernel per (precision, grid size, radix plan): every box of
// the launch has size N.  Launches of different sizes run side by side.
template <typename R, typename K, int N, int V>
__global__ void __launch_bounds__(kBatchThreads, 2) k_batch(BatchArgs a) {
    using Ops = BatchOps<R, K, N, PlanV<N, V>>;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ long long s_item;
    __shared__ int s_ok;
    for (;;) {
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(a.next, 1ull);
        __syncthreads();
        const long long it = s_item;
        if (it >= a.total) return;
        const long long step = it / a.step_items;
        const int r = int(it - step * a.step_items);
        int lo = 0, hi = a.nsegs - 1;  // last segment with first <= r
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(&a.segs[mid].first) <= r) lo = mid;
            else hi = mid - 1;
        }
        const int box = __ldg(&a.segs[lo].box), phase = __ldg(&a.segs[lo].phase);
        const int tile = r - __ldg(&a.segs[lo].first);
        const BatchBox &bx = a.boxes[box];
        if (threadIdx.x == 0) {
            const unsigned long long need =
                (unsigned long long)step * (unsigned long long)bx.step_items + (unsigned long long)bx.prefix[phase];
            s_ok = batch_wait(&a.done[box], need, a.status);
        }
        __syncthreads();
        if (s_ok) Ops::run(smraw, bx, phase, tile);
        __syncthreads();
        if (threadIdx.x == 0) batch_release(&a.done[box]);
    }
}

// The same phases as one launch per (phase, box size) over all boxes of that
// size (blockIdx.y = box, blockIdx.x = tile): the other batch schedule, a
// CUDA graph of such launches, which the autotuner weighs against the
// persistent kernel.
template <typename R, typename K, int N, int V, int PH>
__global__ void __launch_bounds__(kBatchThreads) k_batch_phase(const BatchBox *boxes) {
    extern __shared__ __align__(16) unsigned char smraw[];
    BatchOps<R, K, N, PlanV<N, V>>::template phase<PH>(smraw, boxes[blockIdx.y], (int)blockIdx.x);
}

}  // namespace ifdm
