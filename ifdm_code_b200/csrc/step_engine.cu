// step_engine.cu -- buffers, twiddle tables and launch sequence of the fused
// leap-frog step (kernels in step_kernels.cuh / timestep.cuh).
#include "physics.hpp"
#include "step_engine.hpp"
#include "timestep.cuh"
#include "tma_passes.cuh"
#include "zpass_pipe.cuh"
#include "zpass_tma.cuh"
#include "adjoint_kernels.cuh"

#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <algorithm>
#include <mutex>
#include <set>

namespace ifdm {

// guards this file's process-wide caches (kernel attributes per device, the
// twiddle tables, the tensor-map encoder): contexts may be driven from
// several host threads at once (the batched adjoint does)
static std::mutex &setup_mutex() {
    static std::mutex m;
    return m;
}

const char *const kPassNames[kNumPasses] = {
    "T_timestep", "P1_kick_fft_z", "P2_fft_y", "P3_fft_x_drift_ifft_x", "P4_ifft_y",
    "P5_ifft_z_density_r2c_z", "P6_fft_y_half", "P7_fft_x_poisson_ifft_x", "P8_ifft_y_half", "P9_c2r_z_phi"};

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) return std::string(#expr) + ": " + cudaGetErrorString(e_); \
    } while (0)

bool supported_n(int n) {
    switch (n) {
        case 16: case 32: case 48: case 64: case 96: case 128: case 256: case 512: case 1024: return true;
        default: return false;
    }
}

bool supported_n(int n, int precision) {
    if (precision == 2 && n >= 1024) return false;  // mixed: FP64 exchange tiles exceed shared memory
    return supported_n(n);
}

// ---------------------------------------------------------------- per-N ops --
template <typename R_, typename K_, int N> struct Box {
    using R = R_;
    using K = K_;
    using TL = Tile<R, K, N>;   // y/x passes (strided lines)
    using TZ = TileZ<R, K, N>;  // z passes (contiguous rows)
    using C = cx<K>;
    using G = cx<R>;
    static constexpr int NH = N / 2 + 1;
    static constexpr int NHP = half_pitch<R>(N);
    static constexpr size_t SM = TL::SMEM;
    static constexpr size_t SMZ = TZ::SMEM;
    static constexpr size_t SMZ9 = TZ::SMEM9;
    // every launch covers its array exactly: no partial tiles
    static_assert((N * N) % TL::L == 0 && (N * N) % TZ::L == 0, "z/y/x tiles must divide N^2 lines");
    static_assert((N * NHP) % TL::L == 0, "half-spectrum tiles must divide N*NHP lines");
    static_assert(NHP >= NH, "half-spectrum pitch");
    static_assert(TL::NT <= 1024 && TZ::NT <= 1024, "block size");
    static_assert(SM <= 227 * 1024 && SMZ9 <= 227 * 1024, "shared memory per block");

    template <typename Kern> static cudaError_t prep(Kern kern, size_t smem) {
        return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }

    static std::string configure() {
        // once per device (kernel attributes are per device), under the lock
        // that guards every process-wide cache of this file
        std::lock_guard<std::mutex> lk(setup_mutex());
        static std::set<int> done_on;
        int dev = 0;
        CUDA_TRY(cudaGetDevice(&dev));
        if (done_on.count(dev)) return "";
        CUDA_TRY(prep(k_kick_fft_z<R, K, N>, SMZ));
        CUDA_TRY(prep(k_fft_yx<R, K, N, -1, 1>, SM));
        CUDA_TRY(prep(k_fft_yx<R, K, N, +1, 1>, SM));
        CUDA_TRY(prep(k_fft_yx<R, K, N, -1, 2>, SM));
        CUDA_TRY(prep(k_fft_yx<R, K, N, +1, 2>, SM));
        CUDA_TRY(prep(k_fft_x_drift<R, K, N>, SM));
        CUDA_TRY(prep(k_density_r2c_z<R, K, N, true>, SMZ));
        CUDA_TRY(prep(k_density_r2c_z<R, K, N, false>, SMZ));
        CUDA_TRY(prep(k_fft_x_poisson<R, K, N>, SM));
        CUDA_TRY(prep(k_c2r_z_phi<R, K, N>, SMZ9));
        CUDA_TRY(prep(k_fft_z<R, K, N, -1>, SMZ));
        CUDA_TRY(prep(k_fft_z<R, K, N, +1>, SMZ));
        CUDA_TRY(prep(k_source_r2c_z<R, K, N>, SMZ));
        CUDA_TRY(prep(k_fft_x_poisson_slab<R, K, N>, SM));
        int sms = 0;
        CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if constexpr (kZPipe) {
            using ZP = ZPipe<R, N>;
            CUDA_TRY(prep(k_density_r2c_z_pipe<R, N>, ZP::SMEM5));
            int b5 = 0;
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b5, k_density_r2c_z_pipe<R, N>, ZP::NT, ZP::SMEM5));
            zgrid = sms * (b5 > 0 ? b5 : 1);
        }
        if constexpr (kZT) {
            using Z = ZT<N, R>;
            CUDA_TRY(prep(k_kick_fft_z_tma<N, ZST1, ZB1, R>, ZSM1));
            CUDA_TRY(prep(k_density_r2c_z_tma<N, ZST5, ZB5, R>, ZSM5));
            CUDA_TRY(prep(k_c2r_z_tma<N, ZST9, ZB9, R>, ZSM9));
            int b1 = 0, b5 = 0, b9 = 0;
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_kick_fft_z_tma<N, ZST1, ZB1, R>, Z::NT, ZSM1));
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b5, k_density_r2c_z_tma<N, ZST5, ZB5, R>, Z::NT, ZSM5));
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b9, k_c2r_z_tma<N, ZST9, ZB9, R>, Z::NT, ZSM9));
            zt1grid = sms * (b1 > 0 ? b1 : 1);
            zt5grid = sms * (b5 > 0 ? b5 : 1);
            zt9grid = sms * (b9 > 0 ? b9 : 1);
            if constexpr (kPairZ) {
                CUDA_TRY(prep(k_kick_fft_z_pair<N, ZST1P, ZB1P>, ZSM1P));
                CUDA_TRY(prep(k_density_r2c_z_pair<N, ZST5P, ZB5P>, ZSM5P));
                CUDA_TRY(prep(k_c2r_z_pair<N, ZST9P, ZB9P>, ZSM9P));
                int b1p = 0, b5p = 0, b9p = 0;
                CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1p, k_kick_fft_z_pair<N, ZST1P, ZB1P>,
                                                                       Z::NT / 2, ZSM1P));
                CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b5p, k_density_r2c_z_pair<N, ZST5P, ZB5P>,
                                                                       Z::NT / 2, ZSM5P));
                CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b9p, k_c2r_z_pair<N, ZST9P, ZB9P>,
                                                                       Z::NT / 2, ZSM9P));
                zt1pgrid = sms * (b1p > 0 ? b1p : 1);
                zt5pgrid = sms * (b5p > 0 ? b5p : 1);
                zt9pgrid = sms * (b9p > 0 ? b9p : 1);
            }
        }
        if constexpr (kTma) {
            CUDA_TRY(prep(k_yx_tma<R, K, N, 1, 0, -1>, TT::SMEM));
            CUDA_TRY(prep(k_yx_tma<R, K, N, 1, 0, +1>, TT::SMEM));
            CUDA_TRY(prep(k_yx_tma<R, K, N, 2, 1, 0>, TX::SMEM));
            CUDA_TRY(prep(k_yx_tma<R, K, N, 2, 2, 0>, TX::SMEM));
            // persistent grids: every block resident at once (one wave)
            int by = 0, bx = 0;
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&by, k_yx_tma<R, K, N, 1, 0, -1>, TT::NT, TT::SMEM));
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bx, k_yx_tma<R, K, N, 2, 1, 0>, TX::NT, TX::SMEM));
            ygrid = sms * (by > 0 ? by : 1);
            xgrid = sms * (bx > 0 ? bx : 1);
            if constexpr (kPair) {
                CUDA_TRY(prep(k_yx_tma_pair<N, 1, 0, -1, PSTY, PBY>, TPY::SMEM));
                CUDA_TRY(prep(k_yx_tma_pair<N, 1, 0, +1, PSTY, PBY>, TPY::SMEM));
                CUDA_TRY(prep(k_yx_tma_pair<N, 2, 1, 0, PSTX, PBX>, TPX::SMEM));
                CUDA_TRY(prep(k_yx_tma_pair<N, 2, 2, 0, PSTX, PBX>, TPX::SMEM));
                int py = 0, px = 0;
                CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&py, k_yx_tma_pair<N, 1, 0, -1, PSTY, PBY>,
                                                                       TPY::NT, TPY::SMEM));
                CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&px, k_yx_tma_pair<N, 2, 1, 0, PSTX, PBX>,
                                                                       TPX::NT, TPX::SMEM));
                pygrid = sms * (py > 0 ? py : 1);
                pxgrid = sms * (px > 0 ? px : 1);
            }
        }
        done_on.insert(dev);
        return "";
    }

    // TMA-pipelined y/x passes for N >= 128.  The cp.async-pipelined P5 is
    // used in FP32 only: measured at 512^3 it cut FP32 P5 from 1.42 to 1.02 ms
    // but slowed the FP64 z passes (one 2-slot block per SM hides less latency
    // than three plain blocks), and pipelined P1/P9 gained nothing.
    static constexpr bool kTma = N >= 128;
    static constexpr bool kZPipe = N >= 128 && N <= 512 && std::is_same<R, float>::value && std::is_same<K, float>::value;
    // z passes fed by bulk copies (zpass_tma.cuh) for N >= 256, FP32 and
    // FP64 (8 FP32 or 4 FP64 rows per tile); ring depth and resident blocks
    // per SM of P1, P5 and P9
    static constexpr bool kZT = N >= 256 && std::is_same<R, K>::value;
    static constexpr int ZST1 = 2, ZST5 = 3, ZST9 = 3, ZB1 = N >= 1024 ? 1 : 2, ZB5 = ZB1, ZB9 = ZB1;
    using ZG = ZT<(kZT ? N : 256), R>;
    // ring slots, the mbarriers (64 bytes) and the staged twiddle table
    static constexpr size_t ZSM1 = kZT ? ZST1 * ZG::SLOT1 + 64 + tw_bytes<C>(N) : 0;
    static constexpr size_t ZSM5 = kZT ? ZST5 * ZG::SLOT5 + 64 + tw_bytes<C>(N) : 0;
    static constexpr size_t ZSM9 = kZT ? ZST9 * ZG::SLOT9 + 64 + tw_bytes<C>(N) : 0;
    static inline int zt1grid = 0, zt5grid = 0, zt9grid = 0;  // persistent grids of the bulk-copy z passes
    // the paired z passes (two rows per thread, 256 threads at 512, 512 at
    // 1024; kPairZ below): ring slots, resident blocks per SM, shared memory
    // and persistent grids (at 512, P1 and P9 with one slot at three blocks
    // per SM measured 0.641 -> 0.593 ms and 0.273 -> 0.244 ms against two or
    // three slots at two blocks: the blocks overlap each other's loads; the y
    // passes at one slot and four blocks measured slower, 0.392 -> 0.43 ms;
    // at 1024 the slots leave room for one block)
    static constexpr int ZB = N >= 1024 ? 1 : 3;
    static constexpr int ZST1P = 1, ZB1P = ZB, ZST5P = 2, ZB5P = ZB, ZST9P = 1, ZB9P = ZB;
    static constexpr size_t ZSM1P = kZT ? ZST1P * ZG::SLOT1 + 64 + tw_bytes<C>(N) : 0;
    static constexpr size_t ZSM5P = kZT ? ZST5P * ZG::SLOT5 + 64 + tw_bytes<C>(N) : 0;
    static constexpr size_t ZSM9P = kZT ? ZST9P * ZG::SLOT9 + 64 + tw_bytes<C>(N) : 0;
    static inline int zt1pgrid = 0, zt5pgrid = 0, zt9pgrid = 0;
    using TT = TmaTile<R, K, N, 1>;
    using TX = TmaTile<R, K, N, 2>;
    // FP32 passes at N = 512 with two lines per thread: the y/x passes
    // (k_yx_tma_pair, the same tiles and maps as TT/TX; ring slots and resident
    // blocks per SM of the y and x passes below) and the z passes
    // (k_*_z_pair, ZST*P/ZB*P above).  IFDM_NO_PAIR selects the one-line kernels.
    // (512 and 1024; at 1024 a tile takes 512 threads, one block per SM:
    // measured at 1024^3, step 57.5 -> 44.6 ms, P3 14.8 -> 8.4 ms, P5 9.0 ->
    // 6.7 ms)
    static constexpr bool kPair = (N == 512 || N == 1024) && std::is_same<R, float>::value && std::is_same<K, float>::value;
    static constexpr bool kPairZ = kPair;  // the z passes
    static constexpr int PSTY = 2, PBY = N >= 1024 ? 1 : 3, PSTX = 2, PBX = PBY;
    using TPY = TmaPair<(kPair ? N : 512), PSTY, PBY>;
    using TPX = TmaPair<(kPair ? N : 512), PSTX, PBX>;
    static_assert(!kPair || (TT::L == TPY::L && TX::L == TPX::L), "pair kernels share the tensor maps");
    static inline int pygrid = 0, pxgrid = 0;
    static inline int zgrid = 0;             // persistent grid of the pipelined P5
    static inline int ygrid = 0, xgrid = 0;  // persistent grids of the TMA y and x passes

    // lines per TMA tile of the y and x passes (the inner box extent of their maps)
    static void tma_lines(int &ly, int &lx) {
        ly = TT::L;
        lx = TX::L;
    }

    static unsigned zblocks() { return unsigned(size_t(N) * N / TL::L); }  // y-pass tiles
    static unsigned zrows() { return unsigned(size_t(N) * N / TZ::L); }    // z-pass tiles
    static unsigned hblocks() { return unsigned(size_t(N) * NHP / TL::L); }

    // one pass by index 1..9; tm: TMA maps (psi y, psi x, rho y, rho x) or null
    static void pass(int p, cudaStream_t s, G *psi, R *phi, G *rhok, TState *ts, const C *drift, const C *tw,
                     const C *twh, long wr, int wt, const CUtensorMap *tm = nullptr) {
        const unsigned nt = TL::NT;
        if constexpr (kZT) {
            if (tm && (p == 1 || p == 5 || p == 9)) {
                using Z = ZT<N, R>;
                const int nz = int(size_t(N) * N / Z::L);
                if constexpr (kPairZ) {
                    if (std::getenv("IFDM_NO_PAIR") == nullptr) {
                        const unsigned q = Z::NT / 2;
                        if (p == 1)
                            k_kick_fft_z_pair<N, ZST1P, ZB1P><<<zt1pgrid, q, ZSM1P, s>>>(psi, phi, ts, tw, nz);
                        else if (p == 5)
                            k_density_r2c_z_pair<N, ZST5P, ZB5P><<<zt5pgrid, q, ZSM5P, s>>>(psi, rhok, ts, tw, nz);
                        else
                            k_c2r_z_pair<N, ZST9P, ZB9P><<<zt9pgrid, q, ZSM9P, s>>>(rhok, phi, ts, wr, wt, tw, nz / 2);
                        return;
                    }
                }
                if (p == 1)
                    k_kick_fft_z_tma<N, ZST1, ZB1, R><<<zt1grid, Z::NT, ZSM1, s>>>(psi, phi, ts, tw, nz);
                else if (p == 5)
                    k_density_r2c_z_tma<N, ZST5, ZB5, R><<<zt5grid, Z::NT, ZSM5, s>>>(psi, rhok, ts, tw, nz);
                else
                    k_c2r_z_tma<N, ZST9, ZB9, R><<<zt9grid, Z::NT, ZSM9, s>>>(rhok, phi, ts, wr, wt, tw, nz / 2);
                return;
            }
        }
        if constexpr (kZPipe) {
            if (tm && p == 5 && std::getenv("IFDM_NO_ZPIPE") == nullptr) {
                using ZP = ZPipe<R, N>;
                const int nz = int(size_t(N) * N / ZP::L);
                k_density_r2c_z_pipe<R, N><<<zgrid, ZP::NT, ZP::SMEM5, s>>>(psi, rhok, ts, tw, twh, nz);
                return;
            }
        }
        if constexpr (kTma) {
            if (tm && (p == 2 || p == 3 || p == 4 || p == 6 || p == 7 || p == 8)) {
                // y tiles (TT) and x tiles (TX) may differ in lines per tile
                const int tcy = int(size_t(N) * N / TT::L), thy = int(size_t(N) * NHP / TT::L);
                const int tcx = int(size_t(N) * N / TX::L), thx = int(size_t(N) * NHP / TX::L);
                const unsigned gy = unsigned(ygrid), gx = unsigned(xgrid), ny = TT::NT, nx = TX::NT;
                const size_t sy = TT::SMEM, sx = TX::SMEM;
                if constexpr (kPair) {
                    if (std::getenv("IFDM_NO_PAIR") == nullptr) {
                        const unsigned py = unsigned(pygrid), px = unsigned(pxgrid), qy = TPY::NT, qx = TPX::NT;
                        const size_t my = TPY::SMEM, mx = TPX::SMEM;
                        switch (p) {
                            case 2: k_yx_tma_pair<N, 1, 0, -1, PSTY, PBY><<<py, qy, my, s>>>(tm[0], psi, N, N, tcy, ts, drift, tw); break;
                            case 3: k_yx_tma_pair<N, 2, 1, 0, PSTX, PBX><<<px, qx, mx, s>>>(tm[1], psi, N, N, tcx, ts, drift, tw); break;
                            case 4: k_yx_tma_pair<N, 1, 0, +1, PSTY, PBY><<<py, qy, my, s>>>(tm[0], psi, N, N, tcy, ts, drift, tw); break;
                            case 6: k_yx_tma_pair<N, 1, 0, -1, PSTY, PBY><<<py, qy, my, s>>>(tm[2], rhok, NHP, NH, thy, ts, drift, tw); break;
                            case 7: k_yx_tma_pair<N, 2, 2, 0, PSTX, PBX><<<px, qx, mx, s>>>(tm[3], rhok, NHP, NH, thx, ts, drift, tw); break;
                            case 8: k_yx_tma_pair<N, 1, 0, +1, PSTY, PBY><<<py, qy, my, s>>>(tm[2], rhok, NHP, NH, thy, ts, drift, tw); break;
                        }
                        return;
                    }
                }
                switch (p) {
                    case 2: k_yx_tma<R, K, N, 1, 0, -1><<<gy, ny, sy, s>>>(tm[0], psi, N, N, tcy, ts, 2, drift, tw); break;
                    case 3: k_yx_tma<R, K, N, 2, 1, 0><<<gx, nx, sx, s>>>(tm[1], psi, N, N, tcx, ts, 3, drift, tw); break;
                    case 4: k_yx_tma<R, K, N, 1, 0, +1><<<gy, ny, sy, s>>>(tm[0], psi, N, N, tcy, ts, 4, drift, tw); break;
                    case 6: k_yx_tma<R, K, N, 1, 0, -1><<<gy, ny, sy, s>>>(tm[2], rhok, NHP, NH, thy, ts, 6, drift, tw); break;
                    case 7: k_yx_tma<R, K, N, 2, 2, 0><<<gx, nx, sx, s>>>(tm[3], rhok, NHP, NH, thx, ts, 7, drift, tw); break;
                    case 8: k_yx_tma<R, K, N, 1, 0, +1><<<gy, ny, sy, s>>>(tm[2], rhok, NHP, NH, thy, ts, 8, drift, tw); break;
                }
                return;
            }
        }
        switch (p) {
            case 1: k_kick_fft_z<R, K, N><<<zrows(), TZ::NT, SMZ, s>>>(psi, phi, ts, tw); break;
            case 2: k_fft_yx<R, K, N, -1, 1><<<zblocks(), nt, SM, s>>>(psi, N, N, ts, 2, tw); break;
            case 3: k_fft_x_drift<R, K, N><<<zblocks(), nt, SM, s>>>(psi, drift, ts, tw); break;
            case 4: k_fft_yx<R, K, N, +1, 1><<<zblocks(), nt, SM, s>>>(psi, N, N, ts, 4, tw); break;
            case 5:
                k_density_r2c_z<R, K, N, true><<<zrows(), TZ::NT, SMZ, s>>>(psi, rhok, ts, nullptr, tw, twh);
                break;
            case 6: k_fft_yx<R, K, N, -1, 1><<<hblocks(), nt, SM, s>>>(rhok, NHP, NH, ts, 6, tw); break;
            case 7: k_fft_x_poisson<R, K, N><<<hblocks(), nt, SM, s>>>(rhok, ts, tw); break;
            case 8: k_fft_yx<R, K, N, +1, 1><<<hblocks(), nt, SM, s>>>(rhok, NHP, NH, ts, 8, tw); break;
            case 9: k_c2r_z_phi<R, K, N><<<zrows(), TZ::NT, SMZ9, s>>>(rhok, phi, ts, wr, wt, tw, twh); break;
            default: break;
        }
    }

    static void initial_density(cudaStream_t s, G *psi, G *rhok, TState *ts, double *part, const C *tw,
                                const C *twh) {
        k_density_r2c_z<R, K, N, false><<<zrows(), TZ::NT, SMZ, s>>>(psi, rhok, ts, part, tw, twh);
        k_reduce_init<<<1, 256, 0, s>>>(ts, part, (int)zrows(), double(N) * N * N);
    }

    // g <- U^H g: forward FFT, drift with the conjugate tables, inverse FFT
    static void adj_drift(cudaStream_t s, G *g, TState *ts_adj, const C *drift_conj, const C *tw,
                          const CUtensorMap *tm, uint32_t salt) {
        k_fft_z<R, K, N, -1><<<zrows(), TZ::NT, SMZ, s>>>(g, tw, salt);
        pass(2, s, g, nullptr, nullptr, ts_adj, drift_conj, tw, nullptr, 0, 0, tm);
        pass(3, s, g, nullptr, nullptr, ts_adj, drift_conj, tw, nullptr, 0, 0, tm);
        pass(4, s, g, nullptr, nullptr, ts_adj, drift_conj, tw, nullptr, 0, 0, tm);
        k_fft_z<R, K, N, +1><<<zrows(), TZ::NT, SMZ, s>>>(g, tw, salt ^ 0x68e31da4u);
    }
    // pw = phi_s[w]: real source -> half spectrum -> -1/kappa^2 -> real
    static void poisson_of(cudaStream_t s, const R *w, R *pw, G *rhok, TState *ts_adj, const C *tw, const C *twh,
                           const CUtensorMap *tm) {
        k_source_r2c_z<R, K, N><<<zrows(), TZ::NT, SMZ, s>>>(w, rhok, ts_adj, tw, twh);
        for (int p = 6; p <= 9; ++p) pass(p, s, nullptr, pw, rhok, ts_adj, nullptr, tw, twh, 0, 0, tm);
    }

    // One axis of a slab's local FFT step (plain passes): axis 2 = z on the
    // x-slab [planes][N][N], axis 1 = y on the x-slab, axis 0 = x on the
    // transposed y-slab [N][planes][N] (op 1: forward, -1/(kappa^2 N^3) with
    // global y offset y0, inverse).
    static std::string fft_slab(G *data, int planes, int axis, int sign, int op, int y0, const C *tw, cudaStream_t s) {
        const size_t nl = size_t(planes) * N;
        if (nl % TL::L || nl % TZ::L) return "planes * n must be a multiple of the tile lines";
        const unsigned gz = unsigned(nl / TZ::L), gl = unsigned(nl / TL::L), nt = TL::NT;
        if (axis == 2) {
            if (sign < 0) k_fft_z<R, K, N, -1><<<gz, TZ::NT, SMZ, s>>>(data, tw, 0x2545f491u);
            else k_fft_z<R, K, N, +1><<<gz, TZ::NT, SMZ, s>>>(data, tw, 0x2545f491u);
        } else if (axis == 1) {
            if (sign < 0) k_fft_yx<R, K, N, -1, 1><<<gl, nt, SM, s>>>(data, N, N, nullptr, 0, tw);
            else k_fft_yx<R, K, N, +1, 1><<<gl, nt, SM, s>>>(data, N, N, nullptr, 0, tw);
        } else if (op == 1) {
            k_fft_x_poisson_slab<R, K, N><<<gl, nt, SM, s>>>(data, planes, y0, tw);
        } else {
            if (sign < 0) k_fft_yx<R, K, N, -1, 2><<<gl, nt, SM, s>>>(data, planes, planes, nullptr, 0, tw);
            else k_fft_yx<R, K, N, +1, 2><<<gl, nt, SM, s>>>(data, planes, planes, nullptr, 0, tw);
        }
        return "";
    }

    static void fft3d(G *data, int sign, const C *tw, cudaStream_t s) {
        const unsigned nt = TL::NT;
        if (sign < 0) {
            k_fft_z<R, K, N, -1><<<zrows(), TZ::NT, SMZ, s>>>(data, tw, 0x2545f491u);
            k_fft_yx<R, K, N, -1, 1><<<zblocks(), nt, SM, s>>>(data, N, N, nullptr, 0, tw);
            k_fft_yx<R, K, N, -1, 2><<<zblocks(), nt, SM, s>>>(data, N, N, nullptr, 0, tw);
        } else {
            k_fft_z<R, K, N, +1><<<zrows(), TZ::NT, SMZ, s>>>(data, tw, 0x2545f491u);
            k_fft_yx<R, K, N, +1, 1><<<zblocks(), nt, SM, s>>>(data, N, N, nullptr, 0, tw);
            k_fft_yx<R, K, N, +1, 2><<<zblocks(), nt, SM, s>>>(data, N, N, nullptr, 0, tw);
        }
    }
};

// Runtime (N, precision) -> Box<R, K, N>
template <typename R, typename K, typename F> static std::string with_box(int n, F &&f) {
    switch (n) {
        case 16: return f(Box<R, K, 16>{});
        case 32: return f(Box<R, K, 32>{});
        case 48: return f(Box<R, K, 48>{});
        case 64: return f(Box<R, K, 64>{});
        case 96: return f(Box<R, K, 96>{});
        case 128: return f(Box<R, K, 128>{});
        case 256: return f(Box<R, K, 256>{});
        case 512: return f(Box<R, K, 512>{});
        case 1024:
            // the mixed mode's FP64 exchange tiles do not fit shared memory at 1024
            if constexpr (std::is_same<R, K>::value) return f(Box<R, K, 1024>{});
            else return "grid size 1024 is not supported in mixed precision";
        default: return "unsupported grid size " + std::to_string(n);
    }
}
template <typename F> static std::string with_box2(int n, int prec, F &&f) {
    switch (prec) {
        case 0: return with_box<double, double>(n, f);
        case 1: return with_box<float, float>(n, f);
        case 2: return with_box<float, double>(n, f);
        default: return "unknown precision " + std::to_string(prec);
    }
}
// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
static std::string encode_map(CUtensorMap *m, void *base, bool f64, int rank, const cuuint64_t *dims,
                              const cuuint64_t *strides, const cuuint32_t *box) {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    {
        std::lock_guard<std::mutex> lk(setup_mutex());
        if (!fn) {
            cudaDriverEntryPointQueryResult q;
            CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void **)&fn, cudaEnableDefault, &q));
            if (q != cudaDriverEntryPointSuccess || !fn) {
                fn = nullptr;
                return "cuTensorMapEncodeTiled unavailable";
            }
        }
    }
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(m, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank,
                    base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? "" : "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
}

// y-pass map: [x][y][W complex] as (2W reals, N, N); x-pass map: (2*N*W reals, N).
// Boxes: Ly (Lx) lines by boxr rows.
static std::string make_axis_maps(CUtensorMap *my, CUtensorMap *mx, void *base, bool f64, int N, int W, int Ly,
                                  int Lx, int boxr) {
    const cuuint64_t es = f64 ? 8 : 4;
    const cuuint64_t dy[3] = {cuuint64_t(2) * W, cuuint64_t(N), cuuint64_t(N)};
    const cuuint64_t sy[2] = {cuuint64_t(2) * W * es, cuuint64_t(2) * W * N * es};
    const cuuint32_t by[3] = {cuuint32_t(2 * Ly), cuuint32_t(boxr), 1};
    std::string e = encode_map(my, base, f64, 3, dy, sy, by);
    if (!e.empty()) return e;
    const cuuint64_t dx[2] = {cuuint64_t(2) * N * W, cuuint64_t(N)};
    const cuuint64_t sx[1] = {cuuint64_t(2) * W * N * es};
    const cuuint32_t bx[2] = {cuuint32_t(2 * Lx), cuuint32_t(boxr)};
    return encode_map(mx, base, f64, 2, dx, sx, bx);
}

// arithmetic type of a precision mode: 0 double, 1 float
static int compute_kind(int prec) { return prec == 1 ? 1 : 0; }
static size_t storage_bytes(int prec) { return prec == 0 ? 8 : 4; }

// twiddles exp(-2 pi i m / n), m < n, from long double; FP32 tables pair each
// rounded twiddle with its rounding remainder (exact - rounded): entries 2m, 2m+1
template <typename C> static std::vector<C> twiddles(int n) {
    using T = decltype(C{}.x);
    const int per = sizeof(T) == 4 ? 2 : 1;
    std::vector<C> t(size_t(per) * n);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < n; ++m) {
        const long double ang = -twopi * (long double)m / (long double)n;
        const long double c = cosl(ang), s = sinl(ang);
        C &h = t[size_t(per) * m];
        h.x = (T)c;
        h.y = (T)s;
        if (per == 2) {
            t[2 * size_t(m) + 1].x = (T)(c - (long double)h.x);
            t[2 * size_t(m) + 1].y = (T)(s - (long double)h.y);
        }
    }
    return t;
}

// cached per-(n, precision) tables on the current device
static std::string get_twiddles(int n, int prec, void **out) {
    struct Entry { int dev, n, prec; void *p; };
    std::lock_guard<std::mutex> lk(setup_mutex());
    static std::vector<Entry> cache;
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    for (auto &e : cache)
        if (e.dev == dev && e.n == n && e.prec == prec) { *out = e.p; return ""; }
    void *p = nullptr;
    if (prec == 0) {
        auto t = twiddles<double2>(n);
        CUDA_TRY(cudaMalloc(&p, sizeof(double2) * n));
        CUDA_TRY(cudaMemcpy(p, t.data(), sizeof(double2) * n, cudaMemcpyHostToDevice));
    } else {
        auto t = twiddles<float2>(n);
        CUDA_TRY(cudaMalloc(&p, sizeof(float2) * t.size()));
        CUDA_TRY(cudaMemcpy(p, t.data(), sizeof(float2) * t.size(), cudaMemcpyHostToDevice));
    }
    cache.push_back({dev, n, prec, p});
    *out = p;
    return "";
}

// ------------------------------------------------------------ StepEngine --
StepEngine::~StepEngine() {
    cudaFree(psi_);
    cudaFree(phi_);
    cudaFree(rhok_);
    cudaFree(drift64_);
    cudaFree(drift32_);
    cudaFree(ts_);
    cudaFree(gmax_);
    cudaFree(part_);
    cudaFree(log_);
    cudaFree(ckpt_psi_);
    cudaFree(ckpt_phi_);
    cudaFree(seg_psi_);
    cudaFree(seg_phi_);
    cudaFree(g_);
    cudaFree(w_);
    cudaFree(pw_);
    cudaFree(ts_adj_);
    cudaFree(drift64_adj_);
    cudaFree(drift32_adj_);
    if (copy_stream_) cudaStreamSynchronize(copy_stream_);
    for (int s = 0; s < 2; ++s) {
        cudaFree(stage_[s]);
        if (ev_copied_[s]) cudaEventDestroy(ev_copied_[s]);
        if (ev_free_[s]) cudaEventDestroy(ev_free_[s]);
    }
    if (copy_stream_) cudaStreamDestroy(copy_stream_);
}

std::string StepEngine::ensure_staging() {
    if (stage_[0]) return "";
    CUDA_TRY(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
    for (int s = 0; s < 2; ++s) {
        CUDA_TRY(cudaMalloc(&stage_[s], kStageElems * sizeof(double2)));
        CUDA_TRY(cudaEventCreateWithFlags(&ev_copied_[s], cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&ev_free_[s], cudaEventDisableTiming));
    }
    return "";
}

std::string StepEngine::init(const EngineConfig &cfg, cudaStream_t stream) {
    cfg_ = cfg;
    stream_ = stream;
    const int N = cfg.N;
    if (!supported_n(N, cfg.precision)) return "unsupported grid size " + std::to_string(N);
    const size_t n3 = n3_();
    const size_t rs = storage_bytes(cfg.precision), cs = 2 * rs;
    const int nhp = cfg.precision == 0 ? half_pitch<double>(N) : half_pitch<float>(N);
    CUDA_TRY(cudaMalloc(&psi_, n3 * cs));
    CUDA_TRY(cudaMalloc(&phi_, n3 * rs));
    CUDA_TRY(cudaMalloc(&rhok_, size_t(N) * N * nhp * cs));
    CUDA_TRY(cudaMemsetAsync(rhok_, 0, size_t(N) * N * nhp * cs, stream_));
    CUDA_TRY(cudaMalloc(&drift64_, sizeof(double2) * N));
    CUDA_TRY(cudaMalloc(&drift32_, sizeof(float2) * N));
    CUDA_TRY(cudaMalloc(&ts_, sizeof(TState)));
    CUDA_TRY(cudaMemsetAsync(ts_, 0, sizeof(TState), stream_));
    std::string e = get_twiddles(N, compute_kind(cfg.precision), &tw_);
    if (!e.empty()) return e;
    e = get_twiddles(N / 2, compute_kind(cfg.precision), &twh_);
    if (!e.empty()) return e;
    e = with_box2(N, cfg.precision, [](auto box) { return decltype(box)::configure(); });
    if (!e.empty()) return e;
    // TMA descriptors for the pipelined y/x passes
    use_tma_ = N >= 128 && std::getenv("IFDM_NO_TMA") == nullptr;
    if (use_tma_) {
        const bool f64 = cfg.precision == 0;
        with_box2(N, cfg.precision, [&](auto box) -> std::string {
            decltype(box)::tma_lines(tma_ly_, tma_lx_);
            return "";
        });
        const int boxr = N < 256 ? N : 256;
        e = make_axis_maps(&map_psi_y_, &map_psi_x_, psi_, f64, N, N, tma_ly_, tma_lx_, boxr);
        if (e.empty()) e = make_axis_maps(&map_rho_y_, &map_rho_x_, rhok_, f64, N, nhp, tma_ly_, tma_lx_, boxr);
        if (!e.empty()) return e;
    }
    // max|phi| scan window of the reference: first N^3 doubles of the padded
    // [N][N][2(N/2+1)] array (the vector holds only N^3 elements,
    // src/struct3D.h:110,117; scanned at src/CosmoBEC_MPI.cpp:26)
    const long P = 2 * (N / 2 + 1);
    const long tot = long(N) * N * N;
    win_rows_ = tot / P;
    win_tail_ = int(tot - win_rows_ * P);
    return "";
}

size_t StepEngine::n3_() const { return size_t(cfg_.N) * cfg_.N * cfg_.N; }

std::string StepEngine::set_physics(double a, double rhoc) {
    using namespace phys;
    cfg_.rhoc = rhoc;
    const double m = cfg_.mfdm, ms = cfg_.mfdm_solar;
    const double S2 = rhoc / ms;
    S_ = std::sqrt(S2);
    Phi0_ = 4.0 * M_PI * bigG * rhoc * (cfg_.xmax / M_PI) * (cfg_.xmax / M_PI);
    Phys &ph = phys_;
    ph.A_KE = 4. / (3. * M_PI) * (m / pow(c, 2)) / hbar * pow(cfg_.dx, 2);
    ph.B_PE = 2. * M_PI * hbar / (m / pow(c, 2));
    ph.C_QI = cfg_.g != 0 ? 2. * M_PI * hbar / fabs(cfg_.g) : 0.0;
    ph.g = cfg_.g;
    ph.H0 = H_0;
    ph.Om = Omega_m0;
    ph.kP = m / pow(c, 2) / hbar * Phi0_;
    ph.kQ = cfg_.g / hbar * S2;
    ph.kin = 0.5 * hbar / (m / pow(c, 2)) * (M_PI / cfg_.xmax) * (M_PI / cfg_.xmax);
    ph.Phi0 = Phi0_;
    ph.S2 = S2;
    ph.dt_scale = 1.0;
    ph.N = cfg_.N;
    ph.dither = (cfg_.precision == 1 && std::getenv("IFDM_NO_DITHER") == nullptr) ? 1 : 0;
    ph.limit = 64;
    TState t;
    std::memset(&t, 0, sizeof t);
    t.a = a;
    CUDA_TRY(cudaMemcpyAsync(ts_, &t, sizeof t, cudaMemcpyHostToDevice, stream_));
    CUDA_TRY(cudaStreamSynchronize(stream_));
    return "";
}

std::string StepEngine::load_psi(const double *psi, bool on_device, double a, double rhoc) {
    std::string e = set_physics(a, rhoc);
    if (!e.empty()) return e;
    const size_t n3 = n3_();
    const double invS = 1.0 / S_;
    const int prec = cfg_.precision;
    if (on_device) {
        if (prec == 0) k_psi_in<double><<<1184, 256, 0, stream_>>>((const double2 *)psi, (double2 *)psi_, invS, n3);
        else k_psi_in<float><<<1184, 256, 0, stream_>>>((const double2 *)psi, (float2 *)psi_, invS, n3);

        CUDA_TRY(cudaGetLastError());
    } else {
        // chunk i: host -> slot i%2 on the copy stream, then the conversion on
        // the compute stream; the copy of chunk i+1 runs during conversion i,
        // and a slot is refilled only after its previous conversion finished
        std::string e2 = ensure_staging();
        if (!e2.empty()) return e2;
        int i = 0;
        for (size_t off = 0; off < n3; off += kStageElems, ++i) {
            const int s = i & 1;
            const size_t cnt = std::min(kStageElems, n3 - off);
            CUDA_TRY(cudaStreamWaitEvent(copy_stream_, ev_free_[s], 0));
            CUDA_TRY(cudaMemcpyAsync(stage_[s], psi + 2 * off, cnt * sizeof(double2), cudaMemcpyHostToDevice,
                                     copy_stream_));
            CUDA_TRY(cudaEventRecord(ev_copied_[s], copy_stream_));
            CUDA_TRY(cudaStreamWaitEvent(stream_, ev_copied_[s], 0));
            if (prec == 0)
                k_psi_in<double><<<1184, 256, 0, stream_>>>(stage_[s], (double2 *)psi_ + off, invS, cnt);
            else
                k_psi_in<float><<<1184, 256, 0, stream_>>>(stage_[s], (float2 *)psi_ + off, invS, cnt);
            CUDA_TRY(cudaGetLastError());
            CUDA_TRY(cudaEventRecord(ev_free_[s], stream_));
        }
        // the caller may reuse its buffer once every copy has landed
        CUDA_TRY(cudaStreamSynchronize(copy_stream_));
    }
    return launch_initial_density();
}

std::string StepEngine::psi_to_host(double *host_out, int which) {
    std::string e = ensure_staging();
    if (!e.empty()) return e;
    const size_t n3 = n3_();
    int i = 0;
    for (size_t off = 0; off < n3; off += kStageElems, ++i) {
        const int s = i & 1;
        const size_t cnt = std::min(kStageElems, n3 - off);
        // slot s is rewritten only after its previous copy to the host finished
        CUDA_TRY(cudaStreamWaitEvent(stream_, ev_free_[s], 0));
        if (cfg_.precision == 0)
            k_psi_out<double><<<1184, 256, 0, stream_>>>((const double2 *)psi_ + off, (const double *)phi_ + off, ts_,
                                                         which, S_, stage_[s], cnt);
        else
            k_psi_out<float><<<1184, 256, 0, stream_>>>((const float2 *)psi_ + off, (const float *)phi_ + off, ts_,
                                                        which, S_, stage_[s], cnt);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaEventRecord(ev_copied_[s], stream_));
        CUDA_TRY(cudaStreamWaitEvent(copy_stream_, ev_copied_[s], 0));
        CUDA_TRY(cudaMemcpyAsync(host_out + 2 * off, stage_[s], cnt * sizeof(double2), cudaMemcpyDeviceToHost,
                                 copy_stream_));
        CUDA_TRY(cudaEventRecord(ev_free_[s], copy_stream_));
    }
    CUDA_TRY(cudaStreamSynchronize(copy_stream_));
    return "";
}

std::string StepEngine::launch_initial_density() {
    return with_box2(cfg_.N, cfg_.precision, [&](auto box) -> std::string {
        using B = decltype(box);
        using C = typename B::C;
        using G = typename B::G;
        using R = typename B::R;
        G *psi = (G *)psi_, *rhok = (G *)rhok_;
        R *phi = (R *)phi_;
        const C *tw = (const C *)tw_, *twh = (const C *)twh_;
        if (!part_) CUDA_TRY(cudaMalloc(&part_, sizeof(double) * 3 * B::zrows()));
        B::initial_density(stream_, psi, rhok, ts_, part_, tw, twh);
        const CUtensorMap tm[4] = {map_psi_y_, map_psi_x_, map_rho_y_, map_rho_x_};
        for (int p = 6; p <= 9; ++p)
            B::pass(p, stream_, psi, phi, rhok, ts_, nullptr, tw, twh, win_rows_, win_tail_, use_tma_ ? tm : nullptr);
        CUDA_TRY(cudaGetLastError());
        return "";
    });
}

std::string StepEngine::launch_timestep(double dt_scale) {
    Phys ph = phys_;
    ph.dt_scale = dt_scale;
    const int nt = cfg_.N < 32 ? 32 : (cfg_.N > 512 ? 512 : cfg_.N);
    k_timestep<<<1, nt, 0, stream_>>>(ts_, ph, drift64_, drift32_);
    CUDA_TRY(cudaGetLastError());
    return "";
}

std::string StepEngine::launch_passes(cudaEvent_t *ev) {
    return with_box2(cfg_.N, cfg_.precision, [&](auto box) -> std::string {
        using B = decltype(box);
        using C = typename B::C;
        using G = typename B::G;
        using R = typename B::R;
        G *psi = (G *)psi_, *rhok = (G *)rhok_;
        R *phi = (R *)phi_;
        const C *tw = (const C *)tw_, *twh = (const C *)twh_;
        const C *drift = compute_kind(cfg_.precision) == 0 ? (const C *)(void *)drift64_ : (const C *)(void *)drift32_;
        const CUtensorMap tm[4] = {map_psi_y_, map_psi_x_, map_rho_y_, map_rho_x_};
        for (int p = 1; p <= 9; ++p) {
            B::pass(p, stream_, psi, phi, rhok, ts_, drift, tw, twh, win_rows_, win_tail_, use_tma_ ? tm : nullptr);
            if (ev) CUDA_TRY(cudaEventRecord(ev[p], stream_));
        }
        CUDA_TRY(cudaGetLastError());
        return "";
    });
}

std::string StepEngine::timestep_only(double dt_scale) { return launch_timestep(dt_scale); }
std::string StepEngine::passes_only() { return launch_passes(nullptr); }

std::string StepEngine::step(int nsteps, double dt_scale) {
    for (int i = 0; i < nsteps; ++i) {
        std::string e = launch_timestep(dt_scale);
        if (!e.empty()) return e;
        e = launch_passes(nullptr);
        if (!e.empty()) return e;
    }
    return "";
}

std::string StepEngine::profile(int nsteps, double dt_scale, std::vector<double> &ms) {
    cudaEvent_t ev[kNumPasses + 1];
    for (auto &e : ev) CUDA_TRY(cudaEventCreate(&e));
    ms.assign(kNumPasses, 0.0);
    for (int i = 0; i < nsteps; ++i) {
        CUDA_TRY(cudaEventRecord(ev[0], stream_));
        std::string e = launch_timestep(dt_scale);
        if (!e.empty()) return e;
        CUDA_TRY(cudaEventRecord(ev[1], stream_));
        // passes record ev[p] after pass p; shift so ev[p+1] follows pass p
        cudaEvent_t pe[kNumPasses];
        for (int p = 1; p <= 9; ++p) pe[p] = ev[p + 1];
        e = launch_passes(pe);
        if (!e.empty()) return e;
        CUDA_TRY(cudaEventSynchronize(ev[kNumPasses]));
        for (int p = 0; p < kNumPasses; ++p) {
            float t = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&t, ev[p], ev[p + 1]));
            ms[p] += t;
        }
    }
    for (auto &v : ms) v /= nsteps;
    for (auto &e : ev) cudaEventDestroy(e);
    return "";
}

std::vector<double> StepEngine::pass_bytes() const {
    const double n3 = (double)n3_();
    const double N = cfg_.N;
    const double nh = N * N * (N / 2 + 1);
    const double rs = (double)storage_bytes(cfg_.precision), cs = 2 * rs;
    return {0.0,
            n3 * (2 * cs + rs),         // P1 psi in/out + phi in
            2 * cs * n3,                // P2
            2 * cs * n3,                // P3
            2 * cs * n3,                // P4
            2 * cs * n3 + cs * nh,      // P5 psi in/out + half spectrum out
            2 * cs * nh,                // P6
            2 * cs * nh,                // P7
            2 * cs * nh,                // P8
            cs * nh + rs * n3};         // P9 half spectrum in + phi out
}

std::string StepEngine::psi_out(double *dev_out, int which) {
    const size_t n3 = n3_();
    if (cfg_.precision == 0)
        k_psi_out<double><<<1184, 256, 0, stream_>>>((const double2 *)psi_, (const double *)phi_, ts_, which, S_,
                                                     (double2 *)dev_out, n3);
    else
        k_psi_out<float><<<1184, 256, 0, stream_>>>((const float2 *)psi_, (const float *)phi_, ts_, which, S_,
                                                    (double2 *)dev_out, n3);
    CUDA_TRY(cudaGetLastError());
    return "";
}

std::string StepEngine::phi_out(double *dev_out) {
    const size_t n3 = n3_();
    if (cfg_.precision == 0)
        k_phi_out<double><<<1184, 256, 0, stream_>>>((const double *)phi_, Phi0_, dev_out, n3);
    else
        k_phi_out<float><<<1184, 256, 0, stream_>>>((const float *)phi_, Phi0_, dev_out, n3);
    CUDA_TRY(cudaGetLastError());
    return "";
}

std::string StepEngine::read_state(TState &out) {
    CUDA_TRY(cudaMemcpyAsync(&out, ts_, sizeof(TState), cudaMemcpyDeviceToHost, stream_));
    CUDA_TRY(cudaStreamSynchronize(stream_));
    return "";
}

// ------------------------------------------------------------------ adjoint --
std::string StepEngine::ensure_adjoint_buffers(int nsteps, int ckpt) {
    const size_t n3 = n3_();
    const size_t rs = storage_bytes(cfg_.precision), cs = 2 * rs;
    const int nck = (nsteps + ckpt - 1) / ckpt;
    if (nsteps > log_cap_) {
        cudaFree(log_);
        log_ = nullptr;
        CUDA_TRY(cudaMalloc(&log_, sizeof(StepLog) * nsteps));
        log_cap_ = nsteps;
    }
    if (nck > nckpt_cap_) {
        cudaFree(ckpt_psi_);
        cudaFree(ckpt_phi_);
        ckpt_psi_ = ckpt_phi_ = nullptr;
        CUDA_TRY(cudaMalloc(&ckpt_psi_, n3 * cs * nck));
        CUDA_TRY(cudaMalloc(&ckpt_phi_, n3 * rs * nck));
        nckpt_cap_ = nck;
    }
    if (ckpt > seg_cap_) {
        cudaFree(seg_psi_);
        cudaFree(seg_phi_);
        seg_psi_ = seg_phi_ = nullptr;
        CUDA_TRY(cudaMalloc(&seg_psi_, n3 * cs * ckpt));
        CUDA_TRY(cudaMalloc(&seg_phi_, n3 * rs * ckpt));
        seg_cap_ = ckpt;
    }
    if (!g_) {
        CUDA_TRY(cudaMalloc(&g_, n3 * cs));
        CUDA_TRY(cudaMalloc(&w_, n3 * rs));
        CUDA_TRY(cudaMalloc(&pw_, n3 * rs));
        CUDA_TRY(cudaMalloc(&ts_adj_, sizeof(TState)));
        CUDA_TRY(cudaMemsetAsync(ts_adj_, 0, sizeof(TState), stream_));
        CUDA_TRY(cudaMalloc(&gmax_, sizeof(unsigned long long)));
        CUDA_TRY(cudaMalloc(&drift64_adj_, sizeof(double2) * cfg_.N));
        CUDA_TRY(cudaMalloc(&drift32_adj_, sizeof(float2) * cfg_.N));
        if (use_tma_) {
            const int N = cfg_.N, boxr = N < 256 ? N : 256;
            std::string e = make_axis_maps(&map_g_y_, &map_g_x_, g_, cfg_.precision == 0, N, N, tma_ly_, tma_lx_, boxr);
            if (!e.empty()) return e;
        }
    }
    return "";
}

std::string StepEngine::record(int nsteps, double dt_scale, int ckpt) {
    if (nsteps <= 0 || ckpt <= 0) return "record: nsteps and checkpoint interval must be positive";
    std::string e = ensure_adjoint_buffers(nsteps, ckpt);
    if (!e.empty()) return e;
    const size_t n3 = n3_();
    const size_t rs = storage_bytes(cfg_.precision), cs = 2 * rs;
    ckpt_every_ = ckpt;
    recorded_ = 0;
    StepLog *lg = static_cast<StepLog *>(log_);
    for (int n = 0; n < nsteps; ++n) {
        if (n % ckpt == 0) {
            const size_t k = size_t(n / ckpt);
            CUDA_TRY(cudaMemcpyAsync((char *)ckpt_psi_ + k * n3 * cs, psi_, n3 * cs, cudaMemcpyDeviceToDevice, stream_));
            CUDA_TRY(cudaMemcpyAsync((char *)ckpt_phi_ + k * n3 * rs, phi_, n3 * rs, cudaMemcpyDeviceToDevice, stream_));
        }
        e = launch_timestep(dt_scale);
        if (!e.empty()) return e;
        k_log_step<<<1, 1, 0, stream_>>>(ts_, lg + n);
        e = launch_passes(nullptr);
        if (!e.empty()) return e;
    }
    recorded_ = nsteps;
    return "";
}

// one kick adjoint on g_: w, pw = phi_s[w], combine
std::string StepEngine::adjoint_kick(void *psi, void *phi, double a, double aP, double b, double alpha,
                                     long long tag) {
    const size_t n3 = n3_();
    return with_box2(cfg_.N, cfg_.precision, [&](auto box) -> std::string {
        using B = decltype(box);
        using C = typename B::C;
        using G = typename B::G;
        using R = typename B::R;
        using K = typename B::K;
        const C *tw = (const C *)tw_, *twh = (const C *)twh_;
        const CUtensorMap tm[4] = {map_g_y_, map_g_x_, map_rho_y_, map_rho_x_};
        k_adj_w<R, K><<<1184, 256, 0, stream_>>>((const G *)g_, (const G *)psi, (const R *)phi, a, b, alpha, (R *)w_,
                                                 n3);
        B::poisson_of(stream_, (const R *)w_, (R *)pw_, (G *)rhok_, ts_adj_, tw, twh, use_tma_ ? tm : nullptr);
        k_adj_combine<R, K><<<1184, 256, 0, stream_>>>((G *)g_, (const G *)psi, (const R *)phi, (const R *)pw_,
                                                       (const R *)w_, a, aP, b, alpha, n3,
                                                       (uint32_t)(tag * 0x9e3779b9ull) ^ 0x7f4a7c15u);
        CUDA_TRY(cudaGetLastError());
        return "";
    });
}

std::string StepEngine::adjoint(const double *g_final_dev, double *g0_dev) {
    if (recorded_ <= 0) return "adjoint: no recorded steps";
    const size_t n3 = n3_();
    const size_t rs = storage_bytes(cfg_.precision), cs = 2 * rs;
    const int M = recorded_, K = ckpt_every_;
    std::vector<StepLog> lg(M);
    CUDA_TRY(cudaMemcpyAsync(lg.data(), log_, sizeof(StepLog) * M, cudaMemcpyDeviceToHost, stream_));
    TState fin{};
    CUDA_TRY(cudaMemcpyAsync(&fin, ts_, sizeof(TState), cudaMemcpyDeviceToHost, stream_));
    CUDA_TRY(cudaStreamSynchronize(stream_));
    // natural units -> gradient with respect to the stored (scaled) field:
    // g_s = S g.  S ~ 1e50, so in FP32 storage S g overflows for any
    // cotangent of order one; the sweep is linear in g, so FP32 and mixed
    // carry lambda S g with a power of two lambda that brings max|lambda S g|
    // into [1, 2) (a power of two changes no rounding) and divide it out at
    // the end.  FP64 keeps lambda = 1.
    double lambda = 1.0;
    if (cfg_.precision != 0) {
        CUDA_TRY(cudaMemsetAsync(gmax_, 0, sizeof(unsigned long long), stream_));
        k_absmax<<<1184, 256, 0, stream_>>>(g_final_dev, 2 * n3, gmax_);
        CUDA_TRY(cudaGetLastError());
        unsigned long long bits = 0;
        CUDA_TRY(cudaMemcpyAsync(&bits, gmax_, sizeof(bits), cudaMemcpyDeviceToHost, stream_));
        CUDA_TRY(cudaStreamSynchronize(stream_));
        double gmax = 0.0;
        std::memcpy(&gmax, &bits, sizeof(gmax));
        const double top = gmax * S_;
        if (top > 0.0 && std::isfinite(top)) lambda = std::ldexp(1.0, -std::ilogb(top));
    }
    if (cfg_.precision == 0)
        k_scale_in<double><<<1184, 256, 0, stream_>>>((const double2 *)g_final_dev, (double2 *)g_, S_, n3);
    else
        k_scale_in<float><<<1184, 256, 0, stream_>>>((const double2 *)g_final_dev, (float2 *)g_, S_ * lambda, n3);
    CUDA_TRY(cudaGetLastError());
    // the output map: psi_out = S psi exp(-i (pendP phi + pendQ |psi|^2 - gphase))
    std::string e = adjoint_kick(psi_, phi_, fin.pendP, fin.pendP, fin.pendQ, -fin.gphase, 1ll << 40);
    if (!e.empty()) return e;
    for (int seg = (M - 1) / K; seg >= 0; --seg) {
        const int start = seg * K, end = std::min(M, start + K);
        // replay the segment from its checkpoint, keeping every (psi_n, phi_n)
        CUDA_TRY(cudaMemcpyAsync(psi_, (char *)ckpt_psi_ + size_t(seg) * n3 * cs, n3 * cs, cudaMemcpyDeviceToDevice,
                                 stream_));
        CUDA_TRY(cudaMemcpyAsync(phi_, (char *)ckpt_phi_ + size_t(seg) * n3 * rs, n3 * rs, cudaMemcpyDeviceToDevice,
                                 stream_));
        for (int n = start; n < end; ++n) {
            CUDA_TRY(cudaMemcpyAsync((char *)seg_psi_ + size_t(n - start) * n3 * cs, psi_, n3 * cs,
                                     cudaMemcpyDeviceToDevice, stream_));
            CUDA_TRY(cudaMemcpyAsync((char *)seg_phi_ + size_t(n - start) * n3 * rs, phi_, n3 * rs,
                                     cudaMemcpyDeviceToDevice, stream_));
            if (n + 1 < end) {  // the last state of the segment is not needed
                // same step counter as the forward pass, so stochastic rounding repeats exactly
                k_replay_step<<<1, 256, 0, stream_>>>(ts_, (const StepLog *)log_ + n, cfg_.N, 0, n + 1, drift64_,
                                                      drift32_);
                e = launch_passes(nullptr);
                if (!e.empty()) return e;
            }
        }
        for (int n = end - 1; n >= start; --n) {
            k_replay_step<<<1, 256, 0, stream_>>>(ts_adj_, (const StepLog *)log_ + n, cfg_.N, 1, (1ll << 32) + n,
                                                  drift64_adj_, drift32_adj_);
            e = with_box2(cfg_.N, cfg_.precision, [&](auto box) -> std::string {
                using B = decltype(box);
                using C = typename B::C;
                using G = typename B::G;
                const C *tw = (const C *)tw_;
                const C *dconj = compute_kind(cfg_.precision) == 0 ? (const C *)(void *)drift64_adj_
                                                                   : (const C *)(void *)drift32_adj_;
                const CUtensorMap tm[4] = {map_g_y_, map_g_x_, map_rho_y_, map_rho_x_};
                B::adj_drift(stream_, (G *)g_, ts_adj_, dconj, tw, use_tma_ ? tm : nullptr,
                             (uint32_t)(n * 0x85ebca6bull) ^ 0xc2b2ae35u);
                CUDA_TRY(cudaGetLastError());
                return "";
            });
            if (!e.empty()) return e;
            const StepLog &L = lg[n];
            e = adjoint_kick((char *)seg_psi_ + size_t(n - start) * n3 * cs,
                             (char *)seg_phi_ + size_t(n - start) * n3 * rs, L.coefP, L.coefP, L.coefQ, L.alpha, n);
            if (!e.empty()) return e;
        }
    }
    // gradient with respect to the natural-unit psi_0 = S psi_s: g0 = g_s / S
    if (cfg_.precision == 0)
        k_scale_out<double><<<1184, 256, 0, stream_>>>((const double2 *)g_, (double2 *)g0_dev, 1.0 / S_, n3);
    else
        k_scale_out<float><<<1184, 256, 0, stream_>>>((const float2 *)g_, (double2 *)g0_dev, 1.0 / (S_ * lambda),
                                                      n3);
    CUDA_TRY(cudaGetLastError());
    recorded_ = 0;  // the replay consumed the state; record again before another adjoint
    return "";
}

std::string fft_slab(void *data, int n, int planes, int axis, int precision, int sign, int op, int y0,
                     cudaStream_t stream) {
    if (!supported_n(n, precision)) return "unsupported grid size " + std::to_string(n);
    void *tw = nullptr;
    std::string e = get_twiddles(n, compute_kind(precision), &tw);
    if (!e.empty()) return e;
    return with_box2(n, precision, [&](auto box) -> std::string {
        using B = decltype(box);
        using C = typename B::C;
        using G = typename B::G;
        std::string e2 = B::configure();
        if (!e2.empty()) return e2;
        e2 = B::fft_slab((G *)data, planes, axis, sign, op, y0, (const C *)tw, stream);
        if (!e2.empty()) return e2;
        CUDA_TRY(cudaGetLastError());
        return "";
    });
}

std::string fft3d(void *data, int n, int precision, int sign, cudaStream_t stream) {
    if (!supported_n(n, precision)) return "unsupported grid size " + std::to_string(n);
    void *tw = nullptr;
    std::string e = get_twiddles(n, compute_kind(precision), &tw);
    if (!e.empty()) return e;
    return with_box2(n, precision, [&](auto box) -> std::string {
        using B = decltype(box);
        using C = typename B::C;
        using G = typename B::G;
        std::string e2 = B::configure();
        if (!e2.empty()) return e2;
        B::fft3d((G *)data, sign, (const C *)tw, stream);
        CUDA_TRY(cudaGetLastError());
        return "";
    });
}

}  // namespace ifdm
