// static_poisson.cu -- the potential of a wave function with no device
// allocation: ifdm_poisson_static (include/ifdm.h).
//
// The same kernels as a context's Poisson passes (density + real-to-half
// FFT along z, FFTs along y and x with -1/kappa^2, half-to-real FFT along z)
// run with their scratch -- the half spectrum, the reduction state, partial
// sums and twiddle tables -- in one file-scope __device__ array of
// kStaticScratchBytes.  Every GPU that loads the library holds that array
// until the process exits.
//
// Host code must not pass the array's name to a kernel: on the host that name
// is only a stand-in for the device symbol.  The first call on each device
// looks up the array's device address with cudaGetSymbolAddress while that
// device is current, and sets the shared-memory attributes of the kernels of
// every supported size; later calls on that device reuse both.
#include "../../include/ifdm.h"
#include "physics.hpp"
#include "step_kernels.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

namespace ifdm {

constexpr size_t kStaticScratchBytes = IFDM_STATIC_SCRATCH_BYTES;
constexpr int kStaticMaxRes = IFDM_STATIC_MAX_RES;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// scratch layout (byte offsets)
constexpr size_t kOffState = 0;       // TState (zeroed every call)
constexpr size_t kOffPart = 256;      // 3 doubles per z-tile
constexpr size_t kOffTw = 8192;       // twiddles: N then N/2 complex doubles
constexpr size_t kOffRho = 16384;     // half spectrum N x N x NHP complex doubles

static_assert(sizeof(TState) <= kOffPart, "TState must fit its slot");

__global__ void k_static_twiddles(double2 *tw, int n) {
    // exp(-2 pi i m / n) for the n-point and n/2-point tables
    for (int m = threadIdx.x; m < n + n / 2; m += blockDim.x) {
        const int len = m < n ? n : n / 2;
        const int j = m < n ? m : m - n;
        double s, c;
        sincospi(-2.0 * j / len, &s, &c);
        tw[m] = make_double2(c, s);
    }
}

__global__ void k_static_scale(double *phi, double f, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        phi[i] *= f;
}

template <int N> static size_t static_bytes_needed() {
    return kOffRho + size_t(N) * N * half_pitch<double>(N) * sizeof(double2);
}

template <int N>
static int static_poisson_n(unsigned char *base, const double2 *psi, double *phi, double phi0, cudaStream_t s) {
    using TL = Tile<double, double, N>;
    static_assert(TileZ<double, double, N>::L == TL::L && TileZ<double, double, N>::NT == TL::NT,
                  "FP64 row tiles equal the line tiles");
    constexpr int NH = N / 2 + 1;
    constexpr int NHP = half_pitch<double>(N);
    static_assert(kOffPart + 3 * sizeof(double) * (size_t(N) * N / TL::L) <= kOffTw, "partial sums must fit");
    if (static_bytes_needed<N>() > kStaticScratchBytes) return IFDM_ERR_UNSUPPORTED;
    TState *ts = reinterpret_cast<TState *>(base + kOffState);
    double *part = reinterpret_cast<double *>(base + kOffPart);
    double2 *tw = reinterpret_cast<double2 *>(base + kOffTw);
    double2 *twh = tw + N;
    double2 *rhok = reinterpret_cast<double2 *>(base + kOffRho);
    // the array keeps the previous call's contents: the reduction state starts at zero
    if (cudaMemsetAsync(ts, 0, sizeof(TState), s) != cudaSuccess) return IFDM_ERR_CUDA;
    k_static_twiddles<<<1, 64, 0, s>>>(tw, N);
    const unsigned zb = unsigned(size_t(N) * N / TL::L), hb = unsigned(size_t(N) * NHP / TL::L);
    k_density_r2c_z<double, double, N, false>
        <<<zb, TL::NT, TL::SMEM, s>>>(const_cast<double2 *>(psi), rhok, ts, part, tw, twh);
    k_fft_yx<double, double, N, -1, 1><<<hb, TL::NT, TL::SMEM, s>>>(rhok, NHP, NH, ts, 6, tw);
    k_fft_x_poisson<double, double, N><<<hb, TL::NT, TL::SMEM, s>>>(rhok, ts, tw);
    k_fft_yx<double, double, N, +1, 1><<<hb, TL::NT, TL::SMEM, s>>>(rhok, NHP, NH, ts, 8, tw);
    const long P = 2 * (N / 2 + 1), tot = long(N) * N * N;
    k_c2r_z_phi<double, double, N><<<zb, TL::NT, TL::SMEM9, s>>>(rhok, phi, ts, tot / P, int(tot - (tot / P) * P),
                                                                 tw, twh);
    k_static_scale<<<64, 256, 0, s>>>(phi, phi0, size_t(tot));
    return cudaGetLastError() == cudaSuccess ? IFDM_OK : IFDM_ERR_CUDA;
}

// kernels above 48 KB of shared memory need the attribute (no allocation)
template <int N> static cudaError_t static_attributes() {
    using TL = Tile<double, double, N>;
    cudaError_t e = cudaFuncSetAttribute(k_density_r2c_z<double, double, N, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TL::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fft_yx<double, double, N, -1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TL::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fft_yx<double, double, N, +1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TL::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fft_x_poisson<double, double, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TL::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_c2r_z_phi<double, double, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TL::SMEM9);
    return e;
}

// Once per device, with that device current: the device address of
// g_static_scratch and the kernel attributes of every supported size, so
// that no later call on that device does any set-up work.
static int static_setup(unsigned char **out) {
    constexpr int kMaxDevices = 64;
    static void *addr[kMaxDevices] = {};
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return IFDM_ERR_CUDA;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) return IFDM_ERR_CUDA;
        if (static_attributes<16>() != cudaSuccess || static_attributes<32>() != cudaSuccess ||
            static_attributes<48>() != cudaSuccess || static_attributes<64>() != cudaSuccess)
            return IFDM_ERR_CUDA;
        addr[dev] = p;
    }
    *out = static_cast<unsigned char *>(addr[dev]);
    return IFDM_OK;
}

}  // namespace ifdm

extern "C" int ifdm_poisson_static(const double *psi, double *phi, int res, double mfdm, double xmax, void *stream) {
    using namespace ifdm;
    if (!psi || !phi || res <= 0 || !(mfdm > 0) || !(xmax > 0)) return IFDM_ERR_ARGS;
    if (res > kStaticMaxRes) return IFDM_ERR_UNSUPPORTED;
    unsigned char *base = nullptr;
    int rc = static_setup(&base);
    if (rc != IFDM_OK) return rc;
    // phi = 4 pi G m_solar (xmax/pi)^2 * (-F^-1[F[|psi|^2] / kappa^2] / N^3)
    const double ms = mfdm * phys::kg2eV / phys::kg2solar;
    const double xm = xmax / phys::h_0;
    const double phi0 = 4.0 * M_PI * phys::bigG * ms * (xm / M_PI) * (xm / M_PI);
    const double2 *p2 = reinterpret_cast<const double2 *>(psi);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (res) {
        case 16: return static_poisson_n<16>(base, p2, phi, phi0, s);
        case 32: return static_poisson_n<32>(base, p2, phi, phi0, s);
        case 48: return static_poisson_n<48>(base, p2, phi, phi0, s);
        case 64: return static_poisson_n<64>(base, p2, phi, phi0, s);
        default: return IFDM_ERR_UNSUPPORTED;
    }
}
