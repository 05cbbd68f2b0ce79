// batch_launch.cuh -- host-side launchers of the batch kernels of one precision.
//
// Each precision's kernels are instantiated in their own translation unit
// (batch_fp64.cu, batch_fp32.cu, batch_mixed.cu) so they compile in parallel;
// the engine reaches them through the BatchKernels function table.
#pragma once

#include "batch_kernels.cuh"

#include <string>

namespace ifdm {

struct BatchKernels {
    // items per phase and dynamic shared memory of an N-box; false if N is not a batch size
    bool (*items)(int N, int *items, size_t *smem);
    // set the shared-memory attributes of the (N, V) kernels; *fit = persistent CTAs per SM that fit
    std::string (*setup)(int N, int V, size_t smem, int *fit);
    cudaError_t (*persistent)(int N, int V, int grid, size_t smem, cudaStream_t s, const BatchArgs &a);
    cudaError_t (*phase)(int N, int V, int ph, int tiles, int nboxes, size_t smem, cudaStream_t s,
                         const BatchBox *boxes);
};

const BatchKernels &batch_kernels(int precision);  // 0 FP64, 1 FP32, 2 mixed

template <typename R, typename K, int N, int V> struct BatchLaunch {
    static std::string setup(size_t smem, int *fit) {
        const int sm = (int)smem;
        cudaError_t e = cudaFuncSetAttribute(k_batch<R, K, N, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        const void *ph[kBatchPhases] = {
            (const void *)k_batch_phase<R, K, N, V, 0>, (const void *)k_batch_phase<R, K, N, V, 1>,
            (const void *)k_batch_phase<R, K, N, V, 2>, (const void *)k_batch_phase<R, K, N, V, 3>,
            (const void *)k_batch_phase<R, K, N, V, 4>, (const void *)k_batch_phase<R, K, N, V, 5>,
            (const void *)k_batch_phase<R, K, N, V, 6>, (const void *)k_batch_phase<R, K, N, V, 7>,
            (const void *)k_batch_phase<R, K, N, V, 8>, (const void *)k_batch_phase<R, K, N, V, 9>};
        for (int p = 0; p < kBatchPhases && e == cudaSuccess; ++p)
            e = cudaFuncSetAttribute(ph[p], cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(fit, k_batch<R, K, N, V>, kBatchThreads, smem);
        return e == cudaSuccess ? "" : std::string("batch kernel setup: ") + cudaGetErrorString(e);
    }
    static cudaError_t persistent(int grid, size_t smem, cudaStream_t s, const BatchArgs &a) {
        k_batch<R, K, N, V><<<grid, kBatchThreads, smem, s>>>(a);
        return cudaGetLastError();
    }
    static cudaError_t phase(int ph, int tiles, int nboxes, size_t smem, cudaStream_t s, const BatchBox *b) {
        const dim3 g((unsigned)tiles, (unsigned)nboxes);
        switch (ph) {
            case 0: k_batch_phase<R, K, N, V, 0><<<g, kBatchThreads, smem, s>>>(b); break;
            case 1: k_batch_phase<R, K, N, V, 1><<<g, kBatchThreads, smem, s>>>(b); break;
            case 2: k_batch_phase<R, K, N, V, 2><<<g, kBatchThreads, smem, s>>>(b); break;
            case 3: k_batch_phase<R, K, N, V, 3><<<g, kBatchThreads, smem, s>>>(b); break;
            case 4: k_batch_phase<R, K, N, V, 4><<<g, kBatchThreads, smem, s>>>(b); break;
            case 5: k_batch_phase<R, K, N, V, 5><<<g, kBatchThreads, smem, s>>>(b); break;
            case 6: k_batch_phase<R, K, N, V, 6><<<g, kBatchThreads, smem, s>>>(b); break;
            case 7: k_batch_phase<R, K, N, V, 7><<<g, kBatchThreads, smem, s>>>(b); break;
            case 8: k_batch_phase<R, K, N, V, 8><<<g, kBatchThreads, smem, s>>>(b); break;
            case 9: k_batch_phase<R, K, N, V, 9><<<g, kBatchThreads, smem, s>>>(b); break;
            default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
};

// (N, V) -> BatchLaunch; V = 1 exists where PlanV<N, 1> differs from Plan<N>
template <typename R, typename K, typename F> static bool with_batch_nv(int N, int V, F &&f) {
    switch (N) {
        case 16: f(BatchLaunch<R, K, 16, 0>{}); return true;
        case 32: V ? f(BatchLaunch<R, K, 32, 1>{}) : f(BatchLaunch<R, K, 32, 0>{}); return true;
        case 48: V ? f(BatchLaunch<R, K, 48, 1>{}) : f(BatchLaunch<R, K, 48, 0>{}); return true;
        case 64: V ? f(BatchLaunch<R, K, 64, 1>{}) : f(BatchLaunch<R, K, 64, 0>{}); return true;
        case 96: V ? f(BatchLaunch<R, K, 96, 1>{}) : f(BatchLaunch<R, K, 96, 0>{}); return true;
        case 128: f(BatchLaunch<R, K, 128, 0>{}); return true;
        default: return false;
    }
}

template <typename R, typename K> struct BatchTable {
    template <int N> static void fill(int *items, size_t *smem) {
        for (int p = 0; p < kBatchPhases; ++p) items[p] = batch_items<R, K, N>(p);
        *smem = batch_smem<R, K, N>();
    }
    static bool items(int N, int *it, size_t *smem) {
        switch (N) {
            case 16: fill<16>(it, smem); return true;
            case 32: fill<32>(it, smem); return true;
            case 48: fill<48>(it, smem); return true;
            case 64: fill<64>(it, smem); return true;
            case 96: fill<96>(it, smem); return true;
            case 128: fill<128>(it, smem); return true;
            default: return false;
        }
    }
    static std::string setup(int N, int V, size_t smem, int *fit) {
        std::string e = "batch: res " + std::to_string(N) + " is not a batch size";
        with_batch_nv<R, K>(N, V, [&](auto L) { e = decltype(L)::setup(smem, fit); });
        return e;
    }
    static cudaError_t persistent(int N, int V, int grid, size_t smem, cudaStream_t s, const BatchArgs &a) {
        cudaError_t e = cudaErrorInvalidValue;
        with_batch_nv<R, K>(N, V, [&](auto L) { e = decltype(L)::persistent(grid, smem, s, a); });
        return e;
    }
    static cudaError_t phase(int N, int V, int ph, int tiles, int nboxes, size_t smem, cudaStream_t s,
                             const BatchBox *b) {
        cudaError_t e = cudaErrorInvalidValue;
        with_batch_nv<R, K>(N, V, [&](auto L) { e = decltype(L)::phase(ph, tiles, nboxes, smem, s, b); });
        return e;
    }
    static const BatchKernels &table() {
        static const BatchKernels t{&items, &setup, &persistent, &phase};
        return t;
    }
};

}  // namespace ifdm
