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

// sums over x of |psi|^2, |psi|^4 and phi |psi|^2: part[3 * block + {0, 1, 2}]
__global__ void k_xsums(const double2 *__restrict__ psi, const double *__restrict__ phi, size_t n,
                        double *__restrict__ part) {
    __shared__ double red[32];
    double a = 0.0, b = 0.0, c = 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double2 v = psi[i];
        const double r = v.x * v.x + v.y * v.y;
        a += r;
        b += r * r;
        c += phi[i] * r;
    }
    a = block_sum(a, red);
    b = block_sum(b, red);
    c = block_sum(c, red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = a;
        part[3 * blockIdx.x + 1] = b;
        part[3 * blockIdx.x + 2] = c;
    }
}

// sum over k of |kappa|^2 |psi_k|^2 (kappa per axis in -N/2 .. N/2-1): part[block]
__global__ void k_ksum(const double2 *__restrict__ pk, int N, double *__restrict__ part) {
    __shared__ double red[32];
    const size_t n3 = size_t(N) * N * N;
    double a = 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n3; i += size_t(gridDim.x) * blockDim.x) {
        const int ix = int(i / (size_t(N) * N)), iy = int((i / N) % N), iz = int(i % N);
        const double kx = ix < N / 2 ? ix : ix - N, ky = iy < N / 2 ? iy : iy - N, kz = iz < N / 2 ? iz : iz - N;
        const double2 v = pk[i];
        a += (kx * kx + ky * ky + kz * kz) * (v.x * v.x + v.y * v.y);
    }
    a = block_sum(a, red);
    if (threadIdx.x == 0) part[blockIdx.x] = a;
}

// out[c] = sum over blocks b (in order) of part[nv * b + c], c < nv
__global__ void k_sum_cols(const double *__restrict__ part, int nb, int nv, double *__restrict__ out) {
    __shared__ double red[32];
    for (int c = 0; c < nv; ++c) {
        double a = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) a += part[size_t(nv) * b + c];
        a = block_sum(a, red);
        if (threadIdx.x == 0) out[c] = a;
    }
}

}  // namespace

std::string field_means(double2 *psi_work, const double *phi, int N, double xmax, double out[4], cudaStream_t s) {
    if (N < 2 || N > 1024) return "unsupported grid";
    const size_t n3 = size_t(N) * N * N;
    double *d_part = nullptr;
    std::string err;
    auto run = [&]() -> std::string {
        DG_TRY(cudaMalloc(&d_part, sizeof(double) * (4 * kSumBlocks + 4)));
        double *d_tot = d_part + 4 * kSumBlocks;
        k_xsums<<<kSumBlocks, kSumThreads, 0, s>>>(psi_work, phi, n3, d_part);
        k_sum_cols<<<1, 1024, 0, s>>>(d_part, kSumBlocks, 3, d_tot);
        DG_TRY(cudaGetLastError());
        const std::string e = fft3d(psi_work, N, 0, -1, s);
        if (!e.empty()) return e;
        k_ksum<<<kSumBlocks, kSumThreads, 0, s>>>(psi_work, N, d_part + 3 * kSumBlocks);
        k_sum_cols<<<1, 1024, 0, s>>>(d_part + 3 * kSumBlocks, kSumBlocks, 1, d_tot + 3);
        DG_TRY(cudaGetLastError());
        double h[4];
        DG_TRY(cudaMemcpyAsync(h, d_tot, sizeof(h), cudaMemcpyDeviceToHost, s));
        DG_TRY(cudaStreamSynchronize(s));
        const double inv = 1.0 / double(n3), kf = 3.14159265358979323846 / xmax;  // k = pi kappa / xmax
        out[0] = h[0] * inv;
        out[1] = h[3] * inv * inv * kf * kf;  // Parseval: sum_x |grad psi|^2 = sum_k k^2 |psi_k|^2 / N^3
        out[2] = h[2] * inv;
        out[3] = h[1] * inv;
        return "";
    };
    err = run();
    cudaFree(d_part);
    return err;
}

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
