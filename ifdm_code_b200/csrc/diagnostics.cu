// diagnostics.cu -- power spectrum of the density contrast on the device.
//
// P(k) of delta = rho / <rho> - 1, rho = |psi|^2, estimated on the full FFT
// grid: P(k_b) = <|delta_k|^2>_b L^3 / N^6 averaged over the modes of
// bin b, with integer wave numbers kappa (|kappa| in [edge_b, edge_{b+1}),
// k = 2 pi kappa / L).  The reference has no such output; it is the measure
// the precision comparisons of the step use, so it runs where psi lives.
//
//   1. rho into a complex128 work array (imaginary part 0) and its sum
//      (fixed-order block sums);
//   2. the 3-D c2c FFT of this project (fft3d);
//   3. one block per group of 16 (x, y) lines: for every bin present in a
//      line, a fixed-order block reduction of |rho_k|^2, |kappa| and the mode
//      count; thread 0 adds the line sums in line order -> per-group partials;
//   4. one block per bin adds the group partials in order.
// Every sum has a fixed order, so the result does not change between runs.
#include "diagnostics.hpp"
#include "step_engine.hpp"

#include <cmath>
#include <vector>

namespace ifdm {

#define DG_TRY(expr)                                                                     \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) return std::string(#expr) + ": " + cudaGetErrorString(e_); \
    } while (0)

namespace {

constexpr int kSumBlocks = 592, kSumThreads = 256;  // 4 blocks per SM
constexpr int kLinesPerBlock = 16, kBinThreads = 128;

__device__ __forceinline__ double block_sum(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < nw; ++i) t += red[i];  // every thread, same order
    return t;
}

// rho = |psi|^2 (in place: psi -> (rho, 0)); part[block] = sum over the block's elements
__global__ void k_rho_sum(double2 *__restrict__ d, size_t n, double *__restrict__ part) {
    __shared__ double red[32];
    double s = 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double2 v = d[i];
        const double r = v.x * v.x + v.y * v.y;
        d[i] = make_double2(r, 0.0);
        s += r;
    }
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_sum_parts(const double *__restrict__ part, int n, double *__restrict__ out) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) *out = t;
}

struct BinEdges {
    double e[kMaxBins + 1];
};

__device__ __forceinline__ int bin_of(double kk, const BinEdges &ed, int nb) {
    if (!(kk >= ed.e[0]) || !(kk < ed.e[nb])) return -1;
    int lo = 0, hi = nb;  // ed.e[lo] <= kk < ed.e[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (kk >= ed.e[mid]) lo = mid;
        else hi = mid;
    }
    return lo;
}

// part[(group * nb + b) * 3 + {0,1,2}] = sum |rho_k|^2, sum |kappa|, modes
template <int PER>
__global__ void __launch_bounds__(kBinThreads)
    k_bin_lines(const double2 *__restrict__ rk, int N, int nb, BinEdges ed, double *__restrict__ part) {
    __shared__ double red[32];
    __shared__ double acc[3 * kMaxBins];
    __shared__ int brange[2];
    for (int i = threadIdx.x; i < 3 * nb; i += blockDim.x) acc[i] = 0.0;
    const size_t lines = size_t(N) * N;
    for (int q = 0; q < kLinesPerBlock; ++q) {
        const size_t line = size_t(blockIdx.x) * kLinesPerBlock + q;
        if (line >= lines) break;
        const int ix = int(line / N), iy = int(line % N);
        const double kx = ix < N / 2 ? ix : ix - N, ky = iy < N / 2 ? iy : iy - N;
        double p[PER], kk[PER];
        int b[PER];
        int bmin = kMaxBins, bmax = -1;
#pragma unroll
        for (int e = 0; e < PER; ++e) {
            const int iz = threadIdx.x + e * kBinThreads;
            b[e] = -1;
            p[e] = 0.0;
            kk[e] = 0.0;
            if (iz < N) {
                const double kz = iz < N / 2 ? iz : iz - N;
                kk[e] = sqrt(kx * kx + ky * ky + kz * kz);
                b[e] = bin_of(kk[e], ed, nb);
                const double2 v = rk[line * N + iz];
                p[e] = kk[e] > 0.0 ? v.x * v.x + v.y * v.y : 0.0;  // delta_0 = 0
                if (b[e] >= 0) {
                    bmin = min(bmin, b[e]);
                    bmax = max(bmax, b[e]);
                }
            }
        }
        if (threadIdx.x == 0) {
            brange[0] = kMaxBins;
            brange[1] = -1;
        }
        __syncthreads();
        if (bmax >= 0) {
            atomicMin(&brange[0], bmin);
            atomicMax(&brange[1], bmax);
        }
        __syncthreads();
        const int b0 = brange[0], b1 = brange[1];
        for (int bb = b0; bb <= b1; ++bb) {
            double sp = 0.0, sk = 0.0, sc = 0.0;
#pragma unroll
            for (int e = 0; e < PER; ++e)
                if (b[e] == bb) {
                    sp += p[e];
                    sk += kk[e];
                    sc += 1.0;
                }
            sp = block_sum(sp, red);
            sk = block_sum(sk, red);
            sc = block_sum(sc, red);
            if (threadIdx.x == 0) {
                acc[3 * bb] += sp;
                acc[3 * bb + 1] += sk;
                acc[3 * bb + 2] += sc;
            }
        }
        __syncthreads();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * nb; i += blockDim.x) part[size_t(blockIdx.x) * 3 * nb + i] = acc[i];
}

// out[b * 3 + c] = sum over groups of part[(group * nb + b) * 3 + c]
__global__ void k_bin_total(const double *__restrict__ part, int groups, int nb, double *__restrict__ out) {
    __shared__ double red[32];
    const int b = blockIdx.x;
    for (int c = 0; c < 3; ++c) {
        double s = 0.0;
        for (int g = threadIdx.x; g < groups; g += blockDim.x) s += part[(size_t(g) * nb + b) * 3 + c];
        const double t = block_sum(s, red);
        if (threadIdx.x == 0) out[b * 3 + c] = t;
    }
}

template <int PER>
void launch_bins(const double2 *rk, int N, int nb, const BinEdges &ed, double *part, int groups, cudaStream_t s) {
    k_bin_lines<PER><<<groups, kBinThreads, 0, s>>>(rk, N, nb, ed, part);
}

}  // namespace

std::string power_spectrum(double2 *work, int N, double L, int nbins, const double *edges, double *k_out,
                           double *pk_out, long long *modes_out, double *mean_rho, cudaStream_t s) {
    if (nbins < 1 || nbins > kMaxBins) return "nbins must be 1.." + std::to_string(kMaxBins);
    if (N < 2 || N > 1024) return "unsupported grid";
    const size_t n3 = size_t(N) * N * N;
    BinEdges ed{};
    if (edges) {
        for (int i = 0; i <= nbins; ++i) {
            ed.e[i] = edges[i];
            if (i > 0 && !(edges[i] > edges[i - 1])) return "bin edges must increase";
        }
    } else {
        // log-spaced |kappa| edges from 1 to N/2
        const double top = std::log10(N / 2.0);
        for (int i = 0; i <= nbins; ++i) ed.e[i] = std::pow(10.0, i * (top / nbins));
        ed.e[0] = 1.0;
        ed.e[nbins] = N / 2.0;
    }
    const int groups = int((size_t(N) * N + kLinesPerBlock - 1) / kLinesPerBlock);
    double *d_part = nullptr, *d_out = nullptr;
    std::string err;
    auto run = [&]() -> std::string {
        DG_TRY(cudaMalloc(&d_part, sizeof(double) * std::max<size_t>(kSumBlocks, size_t(groups) * 3 * nbins)));
        DG_TRY(cudaMalloc(&d_out, sizeof(double) * (3 * kMaxBins + 1)));
        k_rho_sum<<<kSumBlocks, kSumThreads, 0, s>>>(work, n3, d_part);
        k_sum_parts<<<1, 1024, 0, s>>>(d_part, kSumBlocks, d_out + 3 * kMaxBins);
        DG_TRY(cudaGetLastError());
        const std::string e = fft3d(work, N, 0, -1, s);
        if (!e.empty()) return e;
        const int per = (N + kBinThreads - 1) / kBinThreads;
        if (per <= 1) launch_bins<1>(work, N, nbins, ed, d_part, groups, s);
        else if (per <= 2) launch_bins<2>(work, N, nbins, ed, d_part, groups, s);
        else if (per <= 4) launch_bins<4>(work, N, nbins, ed, d_part, groups, s);
        else launch_bins<8>(work, N, nbins, ed, d_part, groups, s);
        DG_TRY(cudaGetLastError());
        k_bin_total<<<nbins, 256, 0, s>>>(d_part, groups, nbins, d_out);
        DG_TRY(cudaGetLastError());
        std::vector<double> h(3 * kMaxBins + 1);
        DG_TRY(cudaMemcpyAsync(h.data(), d_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
        DG_TRY(cudaStreamSynchronize(s));
        const double sum = h[3 * kMaxBins], mean = sum / double(n3);
        if (mean_rho) *mean_rho = mean;
        // delta_k = rho_k / mean for kappa != 0 (the bins exclude kappa = 0)
        const double twopi = 6.283185307179586476925286766559;
        const double norm = (L * L * L) / (double(n3) * double(n3)) / (mean * mean);
        for (int b = 0; b < nbins; ++b) {
            const double cnt = h[3 * b + 2];
            if (modes_out) modes_out[b] = (long long)cnt;
            if (pk_out) pk_out[b] = cnt > 0 ? h[3 * b] / cnt * norm : 0.0;
            if (k_out) k_out[b] = cnt > 0 ? h[3 * b + 1] / cnt * twopi / L : 0.0;
        }
        return "";
    };
    err = run();
    cudaFree(d_part);
    cudaFree(d_out);
    return err;
}

}  // namespace ifdm
