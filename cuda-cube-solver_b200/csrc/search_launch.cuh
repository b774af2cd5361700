// Launch of the search kernel variants of one table kind (both formats); each launch_*.cu file
// instantiates it for one kind, so the kernels compile in parallel.
#pragma once

#include "ccs_internal.h"
#include "dispatch.cuh"
#include "search_kernel.cuh"
#include "search_phased.cuh"

namespace ccs {

template <int MODE, int NEC, int FMT, int THREADS, bool SMEM, int MINB>
int launch_variant(ccs_handle* h, const SearchParams& P, int grid, cudaStream_t stream) {
    auto* k = search_kernel<MODE, NEC, FMT, THREADS, SMEM, MINB>;
    constexpr size_t dyn = search_dyn_smem<SMEM, THREADS>();
    if (dyn) CCS_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    k<<<grid, THREADS, dyn, stream>>>(h->d_tables, P);
    CCS_CUDA_TRY(cudaGetLastError());
    return CCS_OK;
}

template <int MODE, int NEC, int FMT, int THREADS, int MINB, bool LOOKAHEAD = false>
int launch_phased(ccs_handle* h, const SearchParams& P, int grid, cudaStream_t stream) {
    auto* k = search_kernel_phased<MODE, NEC, FMT, THREADS, MINB, LOOKAHEAD>;
    constexpr size_t dyn = search_dyn_smem<true, THREADS>();
    if (dyn) CCS_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    k<<<grid, THREADS, dyn, stream>>>(h->d_tables, P);
    CCS_CUDA_TRY(cudaGetLastError());
    return CCS_OK;
}

// Kernel variants (ccs_solve_opts.variant, resolved 1..11): see resolve_variant in solve.cu.
template <int MODE, int NEC>
int launch_kind(ccs_handle* h, const SearchParams& P, int grid, cudaStream_t stream, int variant) {
    return dispatch_fmt(h->format, [&](auto F) {
        constexpr int FMT = decltype(F)::value;
        if (variant == 2) return launch_phased<MODE, NEC, FMT, 256, 2, true>(h, P, grid, stream);
        if (variant == 3) return launch_phased<MODE, NEC, FMT, 256, 3>(h, P, grid, stream);
        if (variant == 4) return launch_variant<MODE, NEC, FMT, 256, false, 2>(h, P, grid, stream);
        if (variant == 5) return launch_variant<MODE, NEC, FMT, 512, true, 2>(h, P, grid, stream);
        if (variant == 6) return launch_phased<MODE, NEC, FMT, 128, 4>(h, P, grid, stream);
        if (variant == 7) return launch_phased<MODE, NEC, FMT, 512, 1>(h, P, grid, stream);
        if (variant == 8) return launch_phased<MODE, NEC, FMT, 256, 3, true>(h, P, grid, stream);
        if (variant == 9) return launch_phased<MODE, NEC, FMT, 256, 4>(h, P, grid, stream);
        if (variant == 10) return launch_phased<MODE, NEC, FMT, 224, 3>(h, P, grid, stream);
        if (variant == 11) return launch_phased<MODE, NEC, FMT, 128, 5>(h, P, grid, stream);
        return launch_phased<MODE, NEC, FMT, 256, 2>(h, P, grid, stream);
    });
}

// Local memory (per-lane DFS stacks) and threads per block of a variant's kernel.
template <int MODE, int NEC>
int kernel_footprint_kind(ccs_handle* h, int variant, size_t* local_bytes, int* threads) {
    return dispatch_fmt(h->format, [&](auto F) {
        constexpr int FMT = decltype(F)::value;
        cudaFuncAttributes a{};
        int t = 256;
        cudaError_t e;
        if (variant == 2) e = cudaFuncGetAttributes(&a, search_kernel_phased<MODE, NEC, FMT, 256, 2, true>);
        else if (variant == 3) e = cudaFuncGetAttributes(&a, search_kernel_phased<MODE, NEC, FMT, 256, 3>);
        else if (variant == 4) e = cudaFuncGetAttributes(&a, search_kernel<MODE, NEC, FMT, 256, false, 2>);
        else if (variant == 5) e = (t = 512, cudaFuncGetAttributes(&a, search_kernel<MODE, NEC, FMT, 512, true, 2>));
        else if (variant == 6) e = (t = 128, cudaFuncGetAttributes(&a, search_kernel_phased<MODE, NEC, FMT, 128, 4>));
        else if (variant == 7) e = (t = 512, cudaFuncGetAttributes(&a, search_kernel_phased<MODE, NEC, FMT, 512, 1>));
        else if (variant == 8) e = cudaFuncGetAttributes(&a, search_kernel_phased<MODE, NEC, FMT, 256, 3, true>);
        else if (variant == 9) e = cudaFuncGetAttributes(&a, search_kernel_phased<MODE, NEC, FMT, 256, 4>);
        else if (variant == 10) e = (t = 224, cudaFuncGetAttributes(&a, search_kernel_phased<MODE, NEC, FMT, 224, 3>));
        else if (variant == 11) e = (t = 128, cudaFuncGetAttributes(&a, search_kernel_phased<MODE, NEC, FMT, 128, 5>));
        else e = cudaFuncGetAttributes(&a, search_kernel_phased<MODE, NEC, FMT, 256, 2>);
        CCS_CUDA_TRY(e);
        *local_bytes = a.localSizeBytes;
        *threads = t;
        return CCS_OK;
    });
}

}  // namespace ccs
