// ic_pipeline.cu -- Gadget IC pre-processing on the device (read_gadget,
// src/gadget_IC.h:573-672).  Compiled with --fmad=false: every product and
// sum below rounds exactly where the reference's does.
//
// CIC deposit as a deterministic sort-by-cell segmented reduction:
//   1. each particle s (in the reference's processing order) emits one
//      (cell, s) pair per corner it deposits to (CIC_scheme,
//      src/gadget_IC.h:45-156), in s-major order;
//   2. the pairs are radix-sorted by cell alone (32-bit keys, only the bits a
//      cell index needs); the sort is stable, so every cell's contributions
//      sit together in particle order;
//   3. one thread per cell folds them in that order: density in FP64,
//      velocities in FP32 with the reference's float += double rounding, so
//      the result is bit-identical to the reference's sequential loop.
// Then mass weighting (:645-651), the central-difference divergence of the
// velocity in FP32 (:190-219), the spectral inverse Laplacian -a^{3/2}/k^2
// with this project's FFT (:222-244), and psi = 1.225 sqrt(rho h^2 1e9 / m)
// exp(i m/(c^2 hbar) theta) (:659-670).
#include "ic_pipeline.hpp"
#include "step_engine.hpp"
#include "fft_engine.cuh"

#include <cub/cub.cuh>

#include <cmath>

namespace ifdm {

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) return std::string(#expr) + ": " + cudaGetErrorString(e_); \
    } while (0)

struct CicGeo {
    int N;
    double Lg, box, pmass, L3;
};

struct CicCell {
    int gi, gj, gk, gii, gjj, gkk;
    double dx, dy, dz, tx, ty, tz;
};

// CIC_scheme's index and weight arithmetic (src/gadget_IC.h:60-99), one rank
__device__ __forceinline__ CicCell cic_cell(const CicGeo &g, float xp, float yp, float zp) {
    CicCell c;
    const int Ng = g.N;
    c.gi = (int)floor(((double)xp - 0.5 * g.Lg) / g.Lg);
    c.gj = (int)floor(((double)yp - 0.5 * g.Lg) / g.Lg);
    c.gk = (int)floor(((double)zp - 0.5 * g.Lg) / g.Lg);
    if (c.gi == -1) { c.gi = Ng - 1; xp = (float)((double)xp + g.box); }
    if (c.gj < 0) { c.gj = Ng - 1; yp = (float)((double)yp + g.box); }
    if (c.gk < 0) { c.gk = Ng - 1; zp = (float)((double)zp + g.box); }
    const double xgi = c.gi * g.Lg + 0.5 * g.Lg;
    const double xgj = c.gj * g.Lg + 0.5 * g.Lg;
    const double xgk = c.gk * g.Lg + 0.5 * g.Lg;
    c.dx = fabs((double)xp - xgi) / g.Lg;
    c.dy = fabs((double)yp - xgj) / g.Lg;
    c.dz = fabs((double)zp - xgk) / g.Lg;
    c.tx = 1. - c.dx;
    c.ty = 1. - c.dy;
    c.tz = 1. - c.dz;
    c.gii = c.gi + 1;
    c.gjj = c.gj + 1;
    c.gkk = c.gk + 1;
    if (c.gii == Ng) c.gii = 0;
    if (c.gjj == Ng) c.gjj = 0;
    if (c.gkk == Ng) c.gkk = 0;
    return c;
}

__device__ __forceinline__ bool cell_ok(const CicCell &c, int N) {
    return c.gi >= 0 && c.gi < N && c.gj >= 0 && c.gj < N && c.gk >= 0 && c.gk < N;
}

// cells of the 8 corners of particle s at keys[8s..8s+7], s at vals[8s..8s+7]
__global__ void k_cic_keys(const float *__restrict__ pos, long np, CicGeo g, unsigned *__restrict__ keys,
                           unsigned *__restrict__ vals, int *__restrict__ bad) {
    const long s = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= np) return;
    const CicCell c = cic_cell(g, pos[3 * s], pos[3 * s + 1], pos[3 * s + 2]);
    unsigned *k = keys + 8 * s, *v = vals + 8 * s;
    const long N = g.N;
    if (!cell_ok(c, g.N)) {
        // outside [0, box): the reference indexes out of its arrays here; refuse
        atomicOr(bad, 1);
        for (int q = 0; q < 8; ++q) {
            k[q] = unsigned(N * N * N);  // past every cell
            v[q] = unsigned(s);
        }
        return;
    }
    const int ii[2] = {c.gi, c.gii}, jj[2] = {c.gj, c.gjj}, kk[2] = {c.gk, c.gkk};
    for (int q = 0; q < 8; ++q) {
        k[q] = unsigned(kk[q & 1] + N * (jj[(q >> 1) & 1] + N * ii[q >> 2]));
        v[q] = unsigned(s);
    }
}

__global__ void k_cell_bounds(const unsigned *__restrict__ keys, long nk, long ncell, int *__restrict__ start,
                              int *__restrict__ end) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nk) return;
    const long c = (long)keys[i];
    if (c >= ncell) return;
    const long cp = i > 0 ? (long)keys[i - 1] : -1;
    const long cn = i + 1 < nk ? (long)keys[i + 1] : -1;
    if (c != cp) start[c] = (int)i;
    if (c != cn) end[c] = (int)(i + 1);
}

// one thread per cell: contributions in particle order
__global__ void k_cic_fold(const unsigned *__restrict__ vals, const int *__restrict__ start,
                           const int *__restrict__ end, const float *__restrict__ pos, const float *__restrict__ vel,
                           CicGeo g, double *__restrict__ rho, float *__restrict__ vx, float *__restrict__ vy,
                           float *__restrict__ vz) {
    const long N = g.N;
    const long cell = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (cell >= N * N * N) return;
    const int ci = int(cell / (N * N)), cj = int((cell / N) % N), ck = int(cell % N);
    double r = 0.0;
    float ax = 0.f, ay = 0.f, az = 0.f;
    for (int i = start[cell]; i < end[cell]; ++i) {
        const long s = (long)vals[i];
        const CicCell c = cic_cell(g, pos[3 * s], pos[3 * s + 1], pos[3 * s + 2]);
        const double X = (ci == c.gi) ? c.tx : c.dx;
        const double Y = (cj == c.gj) ? c.ty : c.dy;
        const double Z = (ck == c.gk) ? c.tz : c.dz;
        const double w = X * Y * Z;
        r = r + w * g.pmass / g.L3;
        ax = (float)((double)ax + w * (double)vel[3 * s] / g.L3);
        ay = (float)((double)ay + w * (double)vel[3 * s + 1] / g.L3);
        az = (float)((double)az + w * (double)vel[3 * s + 2] / g.L3);
    }
    // volume -> mass weighted velocity (src/gadget_IC.h:645-651)
    if (r != 0) {
        ax = (float)((double)ax * (g.pmass / r));
        ay = (float)((double)ay * (g.pmass / r));
        az = (float)((double)az * (g.pmass / r));
    }
    rho[cell] = r;
    vx[cell] = ax;
    vy[cell] = ay;
    vz[cell] = az;
}

// 0.5 (dvx + dvy + dvz) * uc / dx with periodic central differences
// (src/gadget_IC.h:190-219; one rank: the ghost planes are the periodic
// neighbours)
__global__ void k_divergence(const float *__restrict__ vx, const float *__restrict__ vy, const float *__restrict__ vz,
                             int N, double uc, double dx, double2 *__restrict__ out) {
    const long n = N;
    const long idx = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= n * n * n) return;
    const int i = int(idx / (n * n)), j = int((idx / n) % n), k = int(idx % n);
    const int ip = i == N - 1 ? 0 : i + 1, im = i == 0 ? N - 1 : i - 1;
    const int jp = j == N - 1 ? 0 : j + 1, jm = j == 0 ? N - 1 : j - 1;
    const int kp = k == N - 1 ? 0 : k + 1, km = k == 0 ? N - 1 : k - 1;
    const float dvx = vx[k + n * (j + n * ip)] - vx[k + n * (j + n * im)];
    const float dvy = vy[k + n * (jp + n * i)] - vy[k + n * (jm + n * i)];
    const float dvz = vz[kp + n * (j + n * i)] - vz[km + n * (j + n * i)];
    const float sum = (dvx + dvy) + dvz;
    out[idx] = make_double2(0.5 * (double)sum * uc / dx, 0.0);
}

// theta_k *= -a^{3/2} / k^2 (k = 0 -> 0), k as src/struct3D.h:76-85 builds it
__device__ __forceinline__ double kvec(int i, int N, double xmax) {
    return i < N / 2 ? i * M_PI / xmax : ((double)i - N) * M_PI / xmax;
}
__global__ void k_inv_laplace(double2 *__restrict__ th, int N, double a32, double xmax) {
    const long n = N;
    const long idx = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= n * n * n) return;
    const int i = int(idx / (n * n)), j = int((idx / n) % n), k = int(idx % n);
    const double kx = kvec(i, N, xmax), ky = kvec(j, N, xmax), kz = kvec(k, N, xmax);
    const double k2 = kx * kx + ky * ky + kz * kz;
    double2 v = th[idx];
    if (k2 == 0) v = make_double2(0.0, 0.0);
    else v = make_double2(-a32 * v.x / k2, -a32 * v.y / k2);
    th[idx] = v;
}

// psi = 1.225 sqrt(rho uc / m) exp(i kf theta / N^3) as complex128
__global__ void k_build_psi(const double *__restrict__ rho, const double2 *__restrict__ th, long n3, double uc_rho,
                            double mfdm_solar, double kf, double n3d, double2 *__restrict__ psi) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const double amp = 1.225 * sqrt(rho[i] * uc_rho / mfdm_solar);
    const double tr = th[i].x / n3d, ti = th[i].y / n3d;
    const double mag = exp(-(kf * ti));
    double s, c;
    sincos(kf * tr, &s, &c);
    psi[i] = make_double2(amp * (mag * c), amp * (mag * s));
}

std::string ic_pipeline(const IcInput &in, double *d_psi_out, std::vector<float> *vx_out) {
    const int N = in.N;
    const long n3 = long(N) * N * N;
    const long np = in.np;
    const long nk = 8 * np;
    if (nk >= (1L << 31) - 1 || n3 >= (1L << 31)) return "too many particles or cells";
    CicGeo g{N, in.Lg, in.box, in.pmass, in.L3};
    const float *d_pos = in.d_pos, *d_vel = in.d_vel;
    unsigned *d_keys = nullptr, *d_keys2 = nullptr, *d_vals = nullptr, *d_vals2 = nullptr;
    int *d_start = nullptr, *d_end = nullptr, *d_bad = nullptr;
    double *d_rho = nullptr;
    float *d_v = nullptr;
    double2 *d_th = nullptr;
    void *d_tmp = nullptr;
    size_t tmp_bytes = 0;
    std::string err;
    auto cleanup = [&]() {
        cudaFree(d_keys); cudaFree(d_keys2); cudaFree(d_vals); cudaFree(d_vals2); cudaFree(d_start);
        cudaFree(d_end); cudaFree(d_bad); cudaFree(d_rho); cudaFree(d_v); cudaFree(d_th); cudaFree(d_tmp);
    };
    auto run = [&]() -> std::string {
        cudaStream_t s = in.stream;
        CUDA_TRY(cudaMalloc(&d_keys, sizeof(unsigned) * nk));
        CUDA_TRY(cudaMalloc(&d_keys2, sizeof(unsigned) * nk));
        CUDA_TRY(cudaMalloc(&d_vals, sizeof(unsigned) * nk));
        CUDA_TRY(cudaMalloc(&d_vals2, sizeof(unsigned) * nk));
        CUDA_TRY(cudaMalloc(&d_bad, sizeof(int)));
        CUDA_TRY(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
        k_cic_keys<<<unsigned((np + 255) / 256), 256, 0, s>>>(d_pos, np, g, d_keys, d_vals, d_bad);
        CUDA_TRY(cudaGetLastError());
        int end_bit = 1;  // keys 0..n3 (n3 marks a refused particle)
        while ((1L << end_bit) <= n3) ++end_bit;
        cub::DoubleBuffer<unsigned> kb(d_keys, d_keys2), vb(d_vals, d_vals2);
        CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, (int)nk, 0, end_bit, s));
        CUDA_TRY(cudaMalloc(&d_tmp, tmp_bytes));
        CUDA_TRY(cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, kb, vb, (int)nk, 0, end_bit, s));
        const unsigned *sk = kb.Current(), *sv = vb.Current();
        CUDA_TRY(cudaMalloc(&d_start, sizeof(int) * n3));
        CUDA_TRY(cudaMalloc(&d_end, sizeof(int) * n3));
        CUDA_TRY(cudaMemsetAsync(d_start, 0, sizeof(int) * n3, s));
        CUDA_TRY(cudaMemsetAsync(d_end, 0, sizeof(int) * n3, s));
        k_cell_bounds<<<unsigned((nk + 255) / 256), 256, 0, s>>>(sk, nk, n3, d_start, d_end);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMalloc(&d_rho, sizeof(double) * n3));
        CUDA_TRY(cudaMalloc(&d_v, sizeof(float) * 3 * n3));
        float *vx = d_v, *vy = d_v + n3, *vz = d_v + 2 * n3;
        k_cic_fold<<<unsigned((n3 + 127) / 128), 128, 0, s>>>(sv, d_start, d_end, d_pos, d_vel, g, d_rho, vx, vy, vz);
        CUDA_TRY(cudaGetLastError());
        int bad = 0;
        CUDA_TRY(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        if (bad) return "IC particle outside [0, BoxSize)";
        cudaFree(d_keys); d_keys = nullptr;
        cudaFree(d_keys2); d_keys2 = nullptr;
        cudaFree(d_vals); d_vals = nullptr;
        cudaFree(d_vals2); d_vals2 = nullptr;
        cudaFree(d_tmp); d_tmp = nullptr;
        // velocity phase
        CUDA_TRY(cudaMalloc(&d_th, sizeof(double2) * n3));
        const unsigned gb = unsigned((n3 + 255) / 256);
        k_divergence<<<gb, 256, 0, s>>>(vx, vy, vz, N, in.uc_vel, in.dx, d_th);
        CUDA_TRY(cudaGetLastError());
        std::string e = fft3d(d_th, N, 0, -1, s);
        if (!e.empty()) return e;
        k_inv_laplace<<<gb, 256, 0, s>>>(d_th, N, pow(in.a, 3. / 2), in.xmax);
        CUDA_TRY(cudaGetLastError());
        e = fft3d(d_th, N, 0, +1, s);
        if (!e.empty()) return e;
        k_build_psi<<<gb, 256, 0, s>>>(d_rho, d_th, n3, in.uc_rho, in.mfdm_solar, in.kf, (double)(N * N * N),
                                       (double2 *)d_psi_out);
        CUDA_TRY(cudaGetLastError());
        vx_out->resize(n3);
        CUDA_TRY(cudaMemcpyAsync(vx_out->data(), vx, sizeof(float) * n3, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        return "";
    };
    err = run();
    cleanup();
    return err;
}

}  // namespace ifdm
