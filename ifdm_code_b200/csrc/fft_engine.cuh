// fft_engine.cuh -- shared-memory Stockham FFT over a tile of lines, sm_100a.
//
// A tile holds L independent lines of length N in shared memory, element
// (line l, index n) at sm[n * LP + l] with LP = L + 1.  The line index is the
// fastest-varying one, so the 8 (FP64) or 16 (FP32) threads of one
// shared-memory phase always touch consecutive words: butterfly reads and
// writes are conflict-free whatever the stage stride, and the odd pitch also
// makes the transposing copies of contiguous z-lines conflict-free.
//
// Thread (l = tid % L, t = tid / L) owns E = N / T elements of line l; a
// radix-R stage runs E / R butterflies per thread (Stockham autosort, so no
// bit reversal pass).  Twiddles come from a per-size table of
// exp(-2 pi i m / N) built on the host in long double and rounded once (FP32
// tables also carry the rounding remainders, see twmul).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ifdm {

// ---------------------------------------------------------------- complex --
template <typename R> struct CxT;
template <> struct CxT<double> { using T = double2; };
template <> struct CxT<float> { using T = float2; };
template <typename R> using cx = typename CxT<R>::T;

__device__ __forceinline__ double2 mkc(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 mkc(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return mkc(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return mkc(a.x - b.x, a.y - b.y); }
// FP32 complex sums on the paired FP32 pipe of sm_100 (one instruction per
// complex add; each component rounds exactly like the scalar add)
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C, typename S> __device__ __forceinline__ C cscale(C a, S s) { return mkc(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
template <typename C> __device__ __forceinline__ C cconj(C a) { return mkc(a.x, -a.y); }
// multiply by -i (DIR = -1) or +i (DIR = +1)
template <int DIR, typename C> __device__ __forceinline__ C mul_i(C a) {
    return DIR < 0 ? mkc(a.y, -a.x) : mkc(-a.y, a.x);
}
template <typename C> __device__ __forceinline__ auto cnorm2(C a) { return a.x * a.x + a.y * a.y; }

// ------------------------------------------------------------- radix plans --
// Radix sequence per transform length; every radix divides E (elements per
// thread), so a stage is E/R whole butterflies per thread.  Where possible the
// first and last radix are equal: the last stage then leaves each thread
// holding exactly the elements the first stage of the next transform reads.
template <int N> struct Plan;
template <> struct Plan<8> { static constexpr int E = 8, NST = 1; static constexpr int R[1] = {8}; };
template <> struct Plan<16> { static constexpr int E = 8, NST = 2; static constexpr int R[2] = {8, 2}; };
template <> struct Plan<24> { static constexpr int E = 12, NST = 3; static constexpr int R[3] = {4, 3, 2}; };
template <> struct Plan<32> { static constexpr int E = 8, NST = 2; static constexpr int R[2] = {8, 4}; };
template <> struct Plan<48> { static constexpr int E = 12, NST = 3; static constexpr int R[3] = {4, 3, 4}; };
template <> struct Plan<64> { static constexpr int E = 8, NST = 2; static constexpr int R[2] = {8, 8}; };
template <> struct Plan<96> { static constexpr int E = 12, NST = 4; static constexpr int R[4] = {4, 3, 2, 4}; };
template <> struct Plan<128> { static constexpr int E = 8, NST = 3; static constexpr int R[3] = {8, 2, 8}; };
template <> struct Plan<256> { static constexpr int E = 8, NST = 3; static constexpr int R[3] = {8, 4, 8}; };
template <> struct Plan<512> { static constexpr int E = 8, NST = 3; static constexpr int R[3] = {8, 8, 8}; };
// 1024 = 4 * 8 * 8 * 4: radix-4 ends keep the first and last radix equal
// (chained transforms) with 8 elements per thread
template <> struct Plan<1024> { static constexpr int E = 8, NST = 4; static constexpr int R[4] = {4, 8, 8, 4}; };

// Alternative radix orders with the same elements per thread (V = 1), for the
// batch autotuner; V = 0 and sizes without an alternative are Plan<N>.
template <int N, int V> struct PlanV : Plan<N> {};
template <> struct PlanV<32, 1> { static constexpr int E = 8, NST = 2; static constexpr int R[2] = {4, 8}; };
template <> struct PlanV<48, 1> { static constexpr int E = 12, NST = 3; static constexpr int R[3] = {3, 4, 4}; };
template <> struct PlanV<64, 1> { static constexpr int E = 8, NST = 3; static constexpr int R[3] = {4, 4, 4}; };
template <> struct PlanV<96, 1> { static constexpr int E = 12, NST = 4; static constexpr int R[4] = {3, 4, 2, 4}; };

// ------------------------------------------------------------- butterflies --
template <int RAD, int DIR> struct Bfly;

template <int DIR> struct Bfly<2, DIR> {
    template <typename C> __device__ __forceinline__ static void run(C *v) {
        C a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};

template <int DIR> struct Bfly<4, DIR> {
    template <typename C> __device__ __forceinline__ static void run(C *v) {
        C s02 = v[0] + v[2], d02 = v[0] - v[2];
        C s13 = v[1] + v[3], d13 = mul_i<DIR>(v[1] - v[3]);
        v[0] = s02 + s13;
        v[2] = s02 - s13;
        v[1] = d02 + d13;
        v[3] = d02 - d13;
    }
};

// x * c for a real constant c = hi + lo.  FP32 adds the product with the
// rounding remainder lo of the constant: a constant rounded to FP32 would
// scale every butterfly output the same way at every step (a systematic bias
// of ~1e-8 per stage, e.g. a steady loss of norm), while the remaining product
// roundings vary with the data.  In FP64 lo is 0 and this is x * hi.
__device__ __forceinline__ double mulk(double x, double hi, double) { return x * hi; }
__device__ __forceinline__ float mulk(float x, float hi, float lo) { return fmaf(x, hi, x * lo); }
template <typename R> struct KSplit {
    R hi, lo;
    __host__ __device__ constexpr KSplit(double c) : hi(R(c)), lo(R(c - double(R(c)))) {}
};

template <int DIR> struct Bfly<3, DIR> {
    template <typename C> __device__ __forceinline__ static void run(C *v) {
        using R = decltype(v[0].x);
        const R h = R(0.5);
        constexpr KSplit<R> s3(0.86602540378443864676372317075294);  // sqrt(3)/2
        C t1 = v[1] + v[2];
        C t2 = v[0] - cscale(t1, h);
        const C d = mul_i<DIR>(v[1] - v[2]);
        C t3 = mkc(mulk(d.x, s3.hi, s3.lo), mulk(d.y, s3.hi, s3.lo));
        v[0] = v[0] + t1;
        v[1] = t2 + t3;
        v[2] = t2 - t3;
    }
};

template <int DIR> struct Bfly<8, DIR> {
    template <typename C> __device__ __forceinline__ static void run(C *v) {
        using R = decltype(v[0].x);
        constexpr KSplit<R> q(0.70710678118654752440084436210485);  // 1/sqrt(2)
        C a0 = v[0] + v[4], a1 = v[0] - v[4];
        C a2 = v[2] + v[6], a3 = mul_i<DIR>(v[2] - v[6]);
        C a4 = v[1] + v[5], a5 = v[1] - v[5];
        C a6 = v[3] + v[7], a7 = mul_i<DIR>(v[3] - v[7]);
        C b0 = a0 + a2, b2 = a0 - a2, b1 = a1 + a3, b3 = a1 - a3;
        C c0 = a4 + a6, c2 = a4 - a6, c1 = a5 + a7, c3 = a5 - a7;
        // c1 *= w8, c2 *= w8^2 = -/+i, c3 *= w8^3 ; w8 = (1 -/+ i)/sqrt2
        C w1, w3;
        if (DIR < 0) {
            w1 = mkc(mulk(c1.x + c1.y, q.hi, q.lo), mulk(c1.y - c1.x, q.hi, q.lo));
            w3 = mkc(mulk(c3.y - c3.x, q.hi, q.lo), -mulk(c3.x + c3.y, q.hi, q.lo));
        } else {
            w1 = mkc(mulk(c1.x - c1.y, q.hi, q.lo), mulk(c1.x + c1.y, q.hi, q.lo));
            w3 = mkc(-mulk(c3.x + c3.y, q.hi, q.lo), mulk(c3.x - c3.y, q.hi, q.lo));
        }
        C w2 = mul_i<DIR>(c2);
        v[0] = b0 + c0;
        v[4] = b0 - c0;
        v[1] = b1 + w1;
        v[5] = b1 - w1;
        v[2] = b2 + w2;
        v[6] = b2 - w2;
        v[3] = b3 + w3;
        v[7] = b3 - w3;
    }
};

// twiddle exp(DIR * 2 pi i m / N) from the forward table
template <int DIR, typename C> __device__ __forceinline__ C twiddle(const C *__restrict__ tw, int m) {
    C w = __ldg(tw + m);
    return DIR < 0 ? w : cconj(w);
}

// a * exp(DIR * 2 pi i m / TN).  FP64 tables hold one double2 per m.  FP32
// tables hold two float2 per m, the rounded twiddle and its rounding
// remainder (one 16-byte load), and the remainder is folded into the product,
// so the transform is the exact DFT up to the product's own rounding (a
// twiddle table rounded to FP32 alone is a fixed operator error that every
// step repeats).
template <int DIR, int TN> __device__ __forceinline__ double2 twmul(double2 a, const double2 *__restrict__ tw, int m) {
    return cmul(a, twiddle<DIR>(tw, m));
}
template <int DIR, int TN> __device__ __forceinline__ float2 twmul(float2 a, const float2 *__restrict__ tw, int m) {
    const float4 q = __ldg(reinterpret_cast<const float4 *>(tw) + m);
    const float2 h = make_float2(q.x, q.y), r = make_float2(q.z, q.w);
    const float hy = DIR < 0 ? h.y : -h.y, ry = DIR < 0 ? r.y : -r.y;
    const float cr = fmaf(a.x, r.x, -a.y * ry), ci = fmaf(a.x, ry, a.y * r.x);
    return make_float2(fmaf(a.x, h.x, fmaf(-a.y, hy, cr)), fmaf(a.x, hy, fmaf(a.y, h.x, ci)));
}

// The same table staged in shared memory by a persistent kernel (one copy per
// CTA, read with shared-memory loads): the chain then needs no registers to
// hide global-load latency of its twiddles (a two-transform chain with global
// twiddles spills at 64 registers, with staged twiddles it does not).
template <typename C> struct SmemTw {
    const C *p;
};
template <int DIR, int TN> __device__ __forceinline__ double2 twmul(double2 a, SmemTw<double2> tw, int m) {
    const double2 w = tw.p[m];
    return cmul(a, DIR < 0 ? w : cconj(w));
}
template <int DIR, int TN> __device__ __forceinline__ float2 twmul(float2 a, SmemTw<float2> tw, int m) {
    const float4 q = reinterpret_cast<const float4 *>(tw.p)[m];
    const float2 h = make_float2(q.x, q.y), r = make_float2(q.z, q.w);
    const float hy = DIR < 0 ? h.y : -h.y, ry = DIR < 0 ? r.y : -r.y;
    const float cr = fmaf(a.x, r.x, -a.y * ry), ci = fmaf(a.x, ry, a.y * r.x);
    return make_float2(fmaf(a.x, h.x, fmaf(-a.y, hy, cr)), fmaf(a.x, hy, fmaf(a.y, h.x, ci)));
}
// bytes of a twiddle table of length N (FP32 tables pair each entry with its remainder)
template <typename C> __host__ __device__ constexpr size_t tw_bytes(int n) { return size_t(n) * 16; }
// Copy a table into shared memory (all threads of the block; caller syncs).
template <typename C> __device__ __forceinline__ void stage_twiddles(C *dst, const C *__restrict__ src, int n) {
    const float4 *s = reinterpret_cast<const float4 *>(src);
    float4 *d = reinterpret_cast<float4 *>(dst);
    for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = __ldg(s + i);
}

// One Stockham stage: radix RAD, NS = product of the previous radices.
template <typename C, int N, int E, int DIR, int L, int LP, int RAD, int NS>
__device__ __forceinline__ void stockham_stage(C *sm, const C *__restrict__ tw, int l, int t, bool active) {
    constexpr int T = N / E;
    constexpr int NB = E / RAD;
    constexpr int STRIDE = N / RAD;
    constexpr int TWSTEP = N / (NS * RAD);
    C v[E];
    if (active) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + T * b;
            const int k = j % NS;
#pragma unroll
            for (int r = 0; r < RAD; ++r) {
                C a = sm[(j + r * STRIDE) * LP + l];
                if (NS > 1 && r > 0) a = twmul<DIR, N>(a, tw, k * r * TWSTEP);
                v[b * RAD + r] = a;
            }
            Bfly<RAD, DIR>::run(&v[b * RAD]);
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + T * b;
            const int k = j % NS;
            const int base = (j / NS) * NS * RAD + k;
#pragma unroll
            for (int r = 0; r < RAD; ++r) sm[(base + r * NS) * LP + l] = v[b * RAD + r];
        }
    }
    __syncthreads();
}

template <typename C, int N, int E, int DIR, int L, int LP, int S, int NS, class P = Plan<N>>
struct StageLoop {
    __device__ __forceinline__ static void run(C *sm, const C *__restrict__ tw, int l, int t, bool active) {
        if constexpr (S < P::NST) {
            constexpr int RAD = P::R[S];
            static_assert(E % RAD == 0, "elements per thread must be a multiple of every radix");
            stockham_stage<C, N, E, DIR, L, LP, RAD, NS>(sm, tw, l, t, active);
            StageLoop<C, N, E, DIR, L, LP, S + 1, NS * RAD, P>::run(sm, tw, l, t, active);
        }
    }
};

// Elements per thread for a length-N line when T threads serve each line:
// N / T when every radix divides it, else the plan's minimum.
template <int N, class P = Plan<N>> __host__ __device__ constexpr bool divides_all(int e) {
    for (int s = 0; s < P::NST; ++s)
        if (e % P::R[s]) return false;
    return true;
}
template <int N, int T, class P = Plan<N>> __host__ __device__ constexpr int elems_for(int) {
    return (N % T == 0 && N / T >= P::E && divides_all<N, P>(N / T)) ? N / T : P::E;
}

// Plans of the half-length transforms of the real-to-complex passes: 256
// points in radix 4 (4 elements per thread), so the 64 threads that serve a
// 512-point line in the same block all take part (radix 8 would idle half).
template <int M> struct HalfPlan : Plan<M> {};
template <> struct HalfPlan<256> { static constexpr int E = 4, NST = 4; static constexpr int R[4] = {4, 4, 4, 4}; };

// Transform all L lines of the tile in place, E elements per thread (threads
// tid < L * (N / E) work; the rest only join the barriers).  Caller must
// __syncthreads() before (tile written); the tile is synced on return.
template <typename C, int N, int E, int DIR, int L, int LP, class P = Plan<N>>
__device__ __forceinline__ void fft_tile(C *sm, const C *__restrict__ tw) {
    constexpr int T = N / E;
    const int tid = threadIdx.x;
    const int l = tid % L;
    const int t = tid / L;
    StageLoop<C, N, E, DIR, L, LP, 0, 1, P>::run(sm, tw, l, t, t < T);
}

// ------------------------------------------------ register-resident chain --
// The same Stockham stages with the stage inputs held in registers v[E]:
// v[b*RAD + r] is element j + r*N/RAD of line l, j = t + T*b.
//
// SW: element n of a line sits in slot n ^ ((n >> 3) & SW) of the exchange
// tile (SW = 0: no swizzle).  With 8 unpadded float2 lines (the narrow FP32
// x tiles) the first radix-8 stage stores element 8j + r of lines l = 0..7
// for two consecutive j in one half-warp, and both land in the same banks
// (2-way conflicts on every such store); SW = 1 swaps odd and even slots where
// bit 3 is set, which moves one of the two to the other half of the banks,
// and the other store and load patterns of the 8 x 8 x 8 chain stay
// conflict-free (measured at 512^3: P3 0.936 -> 0.917 ms, P7 0.521 -> 0.519
// ms).  With 4 lines a half-warp stores for four consecutive j (4-way); SW = 3
// spreads them over four slots.
template <int SW> __device__ __forceinline__ int slot(int n) { return SW ? (n ^ ((n >> 3) & SW)) : n; }

template <typename C, int N, int E, int L, int LP, int RAD, typename SrcT, int SW = 0>
__device__ __forceinline__ void stage_load(const SrcT *src, C *v, int l, int t) {
    constexpr int T = N / E, NB = E / RAD, STRIDE = N / RAD;
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int r = 0; r < RAD; ++r) {
            const auto g = src[slot<SW>(t + T * b + r * STRIDE) * LP + l];
            v[b * RAD + r] = mkc((decltype(v[0].x))g.x, (decltype(v[0].x))g.y);
        }
}

// twiddle r of butterfly k in the stage (NS, RAD) from a flat table (the
// per-stage tables of the paired kernels add an overload further down)
template <int DIR, int N, int RAD, int NS, typename C, typename TW>
__device__ __forceinline__ C tw_apply(C a, TW tw, int k, int r) {
    return twmul<DIR, N>(a, tw, k * r * (N / (NS * RAD)));
}

template <typename C, int N, int E, int DIR, int RAD, int NS, typename TW>
__device__ __forceinline__ void stage_compute(C *v, TW tw, int t) {
    constexpr int T = N / E, NB = E / RAD;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int k = (t + T * b) % NS;
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < RAD; ++r) v[b * RAD + r] = tw_apply<DIR, N, RAD, NS>(v[b * RAD + r], tw, k, r);
        }
        Bfly<RAD, DIR>::run(&v[b * RAD]);
    }
}

template <typename C, int N, int E, int L, int LP, int RAD, int NS, int SW = 0>
__device__ __forceinline__ void stage_store(C *dst, const C *v, int l, int t) {
    constexpr int T = N / E, NB = E / RAD;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int j = t + T * b;
        const int base = (j / NS) * NS * RAD + j % NS;
#pragma unroll
        for (int r = 0; r < RAD; ++r) dst[slot<SW>(base + r * NS) * LP + l] = v[b * RAD + r];
    }
}

// Stages S.. of a transform whose stage S-1 outputs are in v: round trip
// through `work` (barrier, store, barrier, load) then compute stage S.
template <typename C, int N, int E, int DIR, int L, int LP, int S, int NS, int SW = 0>
struct RegChain {
    template <typename TW> __device__ __forceinline__ static void run(C *work, C *v, TW tw, int l, int t, bool active) {
        if constexpr (S < Plan<N>::NST) {
            constexpr int RP = Plan<N>::R[S - 1];
            constexpr int RAD = Plan<N>::R[S];
            __syncthreads();
            if (active) stage_store<C, N, E, L, LP, RP, NS / RP, SW>(work, v, l, t);
            __syncthreads();
            if (active) {
                stage_load<C, N, E, L, LP, RAD, C, SW>(work, v, l, t);
                stage_compute<C, N, E, DIR, RAD, NS>(v, tw, t);
            }
            RegChain<C, N, E, DIR, L, LP, S + 1, NS * RAD, SW>::run(work, v, tw, l, t, active);
        }
    }
};

// Full transform: stage 0 reads `src` (any element type), later stages go
// through `work`; on return v holds the outputs, v[b*R + r] = element
// j + r*N/R (R the last radix, j = t + T*b).  `src` may alias `work`.
template <typename C, int N, int E, int DIR, int L, int LP, typename SrcT, typename TW>
__device__ __forceinline__ void fft_regs(const SrcT *src, C *work, C *v, TW tw, int l, int t, bool active) {
    constexpr int R0 = Plan<N>::R[0];
    if (active) {
        stage_load<C, N, E, L, LP, R0>(src, v, l, t);
        stage_compute<C, N, E, DIR, R0, 1>(v, tw, t);
    }
    RegChain<C, N, E, DIR, L, LP, 1, R0>::run(work, v, tw, l, t, active);
}

// ------------------------------------------- two lines per thread (FP32) --
// Thread (lp, t) of an FP32 tile [n][L] owns element n of lines 2lp and
// 2lp + 1, which share one 16-byte word: each exchange moves the pair with
// one 128-bit shared-memory access and each twiddle load serves both lines
// (half the shared-memory instructions and twiddle wavefronts of one line per
// thread).  va holds line 2lp, vb line 2lp + 1, in the RegChain order.
//
// StagedTw: the FP32 twiddles as per-stage tables in shared memory, which the
// paired x and z passes use: the stage with NS = product of the earlier radices and
// radix RAD keeps w^(k r N/(NS RAD)) at [(r-1) NS + k] (k < NS, r = 1 ..
// RAD-1).  The threads of a warp hold consecutive k, so their loads hit
// consecutive 16-byte entries, where the flat table's entries k r N/(NS RAD)
// lie r N/(NS RAD) entries apart (for the radix-8 stages of 512 points 128 r
// bytes: the same banks).  Same values as the flat table, so the same results.
template <int N, class P = Plan<N>> struct StagedTw {
    const float4 *p;
    // first entry of the stage whose earlier radices multiply to ns
    static constexpr int offset(int ns) {
        int o = 0, q = 1;
        for (int s = 0; s < P::NST; ++s) {
            if (q == ns) return o;
            if (q > 1) o += (P::R[s] - 1) * q;
            q *= P::R[s];
        }
        return o;
    }
    static constexpr int entries() { return offset(N); }
};
template <int N, class P = Plan<N>> __host__ __device__ constexpr size_t staged_tw_bytes() {
    return size_t(StagedTw<N, P>::entries()) * 16;
}
// 512 = 8 * 8 * 8: stage NS = 8 at [0, 56), NS = 64 at [56, 504)
static_assert(StagedTw<512>::offset(8) == 0 && StagedTw<512>::offset(64) == 56 && StagedTw<512>::entries() == 504,
              "per-stage table layout");
// 1024 = 4 * 8 * 8 * 4: NS = 4, 32, 256 at 0, 28, 252; 1020 entries
static_assert(StagedTw<1024>::offset(4) == 0 && StagedTw<1024>::offset(32) == 28 &&
                  StagedTw<1024>::offset(256) == 252 && StagedTw<1024>::entries() == 1020,
              "per-stage table layout");
// Flat-table index of per-stage entry i (stages S.., Q = product of the
// radices before S, O = first entry of stage S).
template <int N, class P, int S = 0, int Q = 1, int O = 0>
__device__ __forceinline__ int staged_src(int i) {
    if constexpr (S >= P::NST) {
        return 0;
    } else {
        constexpr int RAD = P::R[S];
        constexpr int CNT = Q > 1 ? (RAD - 1) * Q : 0;
        if (i >= O && i < O + CNT) {
            const int j = i - O;
            return (j % Q) * (j / Q + 1) * (N / (Q * RAD));
        }
        return staged_src<N, P, S + 1, Q * RAD, O + CNT>(i);
    }
}
// Fill the per-stage tables from the flat FP32 table (hi, remainder pairs);
// all threads of the block, the caller syncs.
template <int N, class P = Plan<N>> __device__ __forceinline__ void stage_twiddles_staged(float4 *dst, const float2 *src) {
    const float4 *s4 = reinterpret_cast<const float4 *>(src);
    for (int i = threadIdx.x; i < StagedTw<N, P>::entries(); i += blockDim.x) dst[i] = __ldg(s4 + staged_src<N, P>(i));
}

__device__ __forceinline__ void twmul_pair_q(float2 &a, float2 &b, float4 q, int dir) {
    const float hy = dir < 0 ? q.y : -q.y, ry = dir < 0 ? q.w : -q.w;
    float cr = fmaf(a.x, q.z, -a.y * ry), ci = fmaf(a.x, ry, a.y * q.z);
    a = make_float2(fmaf(a.x, q.x, fmaf(-a.y, hy, cr)), fmaf(a.x, hy, fmaf(a.y, q.x, ci)));
    cr = fmaf(b.x, q.z, -b.y * ry);
    ci = fmaf(b.x, ry, b.y * q.z);
    b = make_float2(fmaf(b.x, q.x, fmaf(-b.y, hy, cr)), fmaf(b.x, hy, fmaf(b.y, q.x, ci)));
}
// twiddle r of butterfly k in the stage (NS, RAD), from either table
template <int DIR, int N, int RAD, int NS>
__device__ __forceinline__ void twmul_pair(float2 &a, float2 &b, SmemTw<float2> tw, int k, int r) {
    twmul_pair_q(a, b, reinterpret_cast<const float4 *>(tw.p)[k * r * (N / (NS * RAD))], DIR);
}
template <int DIR, int N, int RAD, int NS, class P>
__device__ __forceinline__ void twmul_pair(float2 &a, float2 &b, StagedTw<N, P> tw, int k, int r) {
    twmul_pair_q(a, b, tw.p[StagedTw<N, P>::offset(NS) + (r - 1) * NS + k], DIR);
}
// one line from the per-stage tables (the single-line stages of the paired kernels)
template <int DIR, int N, int RAD, int NS, typename C, class P>
__device__ __forceinline__ C tw_apply(C a, StagedTw<N, P> tw, int k, int r) {
    static_assert(sizeof(C) == 8, "per-stage tables hold FP32 twiddles");
    const float4 q = tw.p[StagedTw<N, P>::offset(NS) + (r - 1) * NS + k];
    const float hy = DIR < 0 ? q.y : -q.y, ry = DIR < 0 ? q.w : -q.w;
    const float cr = fmaf(a.x, q.z, -a.y * ry), ci = fmaf(a.x, ry, a.y * q.z);
    return make_float2(fmaf(a.x, q.x, fmaf(-a.y, hy, cr)), fmaf(a.x, hy, fmaf(a.y, q.x, ci)));
}

template <int N, int E, int LH, int RAD, int SW = 0>
__device__ __forceinline__ void stage_load_pair(const float4 *src, float2 *va, float2 *vb, int lp, int t) {
    constexpr int T = N / E, NB = E / RAD, STRIDE = N / RAD;
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int r = 0; r < RAD; ++r) {
            const float4 q = src[slot<SW>(t + T * b + r * STRIDE) * LH + lp];
            va[b * RAD + r] = make_float2(q.x, q.y);
            vb[b * RAD + r] = make_float2(q.z, q.w);
        }
}

template <int N, int E, int DIR, int RAD, int NS, typename TW>
__device__ __forceinline__ void stage_compute_pair(float2 *va, float2 *vb, TW tw, int t) {
    constexpr int T = N / E, NB = E / RAD;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int k = (t + T * b) % NS;
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < RAD; ++r) twmul_pair<DIR, N, RAD, NS>(va[b * RAD + r], vb[b * RAD + r], tw, k, r);
        }
        Bfly<RAD, DIR>::run(&va[b * RAD]);
        Bfly<RAD, DIR>::run(&vb[b * RAD]);
    }
}

template <int N, int E, int LH, int RAD, int NS, int SW = 0>
__device__ __forceinline__ void stage_store_pair(float4 *dst, const float2 *va, const float2 *vb, int lp, int t) {
    constexpr int T = N / E, NB = E / RAD;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int j = t + T * b;
        const int base = (j / NS) * NS * RAD + j % NS;
#pragma unroll
        for (int r = 0; r < RAD; ++r)
            dst[slot<SW>(base + r * NS) * LH + lp] =
                make_float4(va[b * RAD + r].x, va[b * RAD + r].y, vb[b * RAD + r].x, vb[b * RAD + r].y);
    }
}

// RegChain for line pairs (same stage order and barriers)
template <int N, int E, int DIR, int LH, int S, int NS, int SW = 0> struct RegChainPair {
    template <typename TW>
    __device__ __forceinline__ static void run(float4 *work, float2 *va, float2 *vb, TW tw, int lp, int t) {
        if constexpr (S < Plan<N>::NST) {
            constexpr int RP = Plan<N>::R[S - 1];
            constexpr int RAD = Plan<N>::R[S];
            __syncthreads();
            stage_store_pair<N, E, LH, RP, NS / RP, SW>(work, va, vb, lp, t);
            __syncthreads();
            stage_load_pair<N, E, LH, RAD, SW>(work, va, vb, lp, t);
            stage_compute_pair<N, E, DIR, RAD, NS>(va, vb, tw, t);
            RegChainPair<N, E, DIR, LH, S + 1, NS * RAD, SW>::run(work, va, vb, tw, lp, t);
        }
    }
};

// Second transform straight from the registers of a first one (requires the
// plan's first and last radix to be equal).
template <typename C, int N, int E, int DIR, int L, int LP, int SW = 0, typename TW>
__device__ __forceinline__ void fft_regs_chained(C *work, C *v, TW tw, int l, int t, bool active) {
    constexpr int R0 = Plan<N>::R[0];
    static_assert(Plan<N>::R[0] == Plan<N>::R[Plan<N>::NST - 1], "chained transform needs equal first/last radix");
    if (active) stage_compute<C, N, E, DIR, R0, 1>(v, tw, t);
    RegChain<C, N, E, DIR, L, LP, 1, R0, SW>::run(work, v, tw, l, t, active);
}

}  // namespace ifdm
