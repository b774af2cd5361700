// Random 32-byte sector gather ceiling of the GPU (the table probes' memory roofline), and the
// probe step alone (index + table read per random state) for comparison with the full search.
#include <cuda_runtime.h>

#include <chrono>

#include "ccs_internal.h"
#include "cube_dev.cuh"
#include "dispatch.cuh"

using namespace ccs;

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 31;
    x *= 0x7FB5D329728EA185ull;
    x ^= x >> 27;
    x *= 0x81DADEF4BC2DD44Dull;
    return x ^ (x >> 33);
}

// Each thread keeps LANES independent random sector loads in flight per round.
template <int LANES>
__global__ void __launch_bounds__(256) k_gather(const uint32_t* __restrict__ buf, uint64_t n_sectors, int rounds,
                                                unsigned long long* __restrict__ sink) {
    uint64_t x[LANES];
    uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
#pragma unroll
    for (int l = 0; l < LANES; ++l) x[l] = mix64(tid * LANES + l + 1);
    uint32_t acc = 0;
    for (int r = 0; r < rounds; ++r) {
        uint32_t w[LANES][8];
#pragma unroll
        for (int l = 0; l < LANES; ++l) {
            x[l] = mix64(x[l]);
            uint64_t s = (uint64_t)(((unsigned __int128)x[l] * n_sectors) >> 64);
            load_sector(buf + s * 8u, w[l]);
        }
#pragma unroll
        for (int l = 0; l < LANES; ++l) acc += w[l][0] ^ pick8(w[l], (uint32_t)(x[l] >> 13) & 7u);
    }
    if (acc == 0x12345678u) atomicAdd(sink, 1ull);  // keeps the loads alive
}

// The probe step alone: random table entries -> representative state (outside the timed loop is
// not possible per entry, so states are generated by unranking) -> index -> lower bound.
template <int MODE, int NEC, int FMT>
__global__ void __launch_bounds__(256) k_probe_only(const DevTables* __restrict__ gT, const uint32_t* __restrict__ classidx,
                                                    const uint32_t* __restrict__ states, uint64_t n_states,
                                                    const uint32_t* __restrict__ table, int rounds,
                                                    unsigned long long* __restrict__ sink) {
    __shared__ DevTables T;
    stage_tables(T, gT);
    uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t x = mix64(tid + 7);
    uint32_t acc = 0;
    for (int r = 0; r < rounds; ++r) {
        x = mix64(x);
        uint64_t i = (uint64_t)(((unsigned __int128)x * n_states) >> 64);
        State s{__ldg(states + 5 * i), __ldg(states + 5 * i + 1), __ldg(states + 5 * i + 2), __ldg(states + 5 * i + 3),
                __ldg(states + 5 * i + 4)};
        move_right(T, s, (int)(x >> 59) % 18);
        acc += lower_bound_dev<FMT>(table, table_index_dev<MODE, NEC>(T, classidx, s));
    }
    if (acc == 0x12345678u) atomicAdd(sink, 1ull);
}

}  // namespace

// The ceiling is the best of a few launch shapes (independent loads in flight per thread x
// resident blocks per SM), so that it does not understate what the memory system delivers.
template <int LANES>
static int time_gather(const uint32_t* buf, uint64_t n_sectors, int grid, int rounds, unsigned long long* sink,
                       cudaEvent_t a, cudaEvent_t b, double* rate, float* t_ms) {
    k_gather<LANES><<<grid, 256>>>(buf, n_sectors, 2, sink);  // warm-up
    CCS_CUDA_TRY(cudaEventRecord(a));
    k_gather<LANES><<<grid, 256>>>(buf, n_sectors, rounds, sink);
    CCS_CUDA_TRY(cudaEventRecord(b));
    CCS_CUDA_TRY(cudaEventSynchronize(b));
    float t = 0;
    CCS_CUDA_TRY(cudaEventElapsedTime(&t, a, b));
    *rate = (double)grid * 256.0 * LANES * rounds / (t * 1e-3);
    *t_ms = t;
    return CCS_OK;
}

extern "C" int ccs_gather_bench(int device, uint64_t bytes, int rounds, double* sectors_per_s, double* ms) {
    if (rounds <= 0 || bytes < 32) return fail(CCS_E_ARG, "bad arguments");
    CCS_CUDA_TRY(cudaSetDevice(device));
    int sms = 0;
    CCS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    DeviceBuffer<uint32_t> buf(bytes / 4);
    DeviceBuffer<unsigned long long> sink(1);
    if (!buf.ok() || !sink.ok()) return fail(CCS_E_NOMEM, "gather buffer of %llu bytes", (unsigned long long)bytes);
    CCS_CUDA_TRY(cudaMemset(buf.p, 0x5A, bytes));
    const uint64_t n_sectors = bytes / 32;
    cudaEvent_t a, b;
    CCS_CUDA_TRY(cudaEventCreate(&a));
    CCS_CUDA_TRY(cudaEventCreate(&b));
    double best = 0, rate = 0;
    float best_ms = 0, t = 0;
    int rc = CCS_OK;
    for (int bps : {4, 8}) {
        const int grid = sms * bps;
        if (rc == CCS_OK) rc = time_gather<4>(buf.p, n_sectors, grid, rounds * 2, sink.p, a, b, &rate, &t);
        if (rc == CCS_OK && rate > best) best = rate, best_ms = t;
        if (rc == CCS_OK) rc = time_gather<8>(buf.p, n_sectors, grid, rounds, sink.p, a, b, &rate, &t);
        if (rc == CCS_OK && rate > best) best = rate, best_ms = t;
        if (rc == CCS_OK) rc = time_gather<16>(buf.p, n_sectors, grid, (rounds + 1) / 2, sink.p, a, b, &rate, &t);
        if (rc == CCS_OK && rate > best) best = rate, best_ms = t;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc != CCS_OK) return rc;
    if (ms) *ms = best_ms;
    if (sectors_per_s) *sectors_per_s = best;
    return CCS_OK;
}

extern "C" int ccs_probe_bench(ccs_handle* h, int n_states, int rounds, double* probes_per_s, double* ms) {
    if (!h || n_states <= 0 || rounds <= 0) return fail(CCS_E_ARG, "bad arguments");
    if (!h->d_table) return fail(CCS_E_STATE, "no table loaded");
    CCS_CUDA_TRY(cudaSetDevice(h->device));
    // Random table entries, unranked into states on the host side of the library.
    std::vector<uint64_t> idx(n_states);
    uint64_t x = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < n_states; ++i) {
        x ^= x << 13, x ^= x >> 7, x ^= x << 17;
        idx[i] = x % h->kind.n_entries;
    }
    std::vector<uint32_t> states(5ull * n_states);
    CCS_TRY(ccs_unrank(h, idx.data(), n_states, states.data()));
    DeviceBuffer<uint32_t> ds(5ull * n_states);
    DeviceBuffer<unsigned long long> sink(1);
    if (!ds.ok() || !sink.ok()) return fail(CCS_E_NOMEM, "probe bench buffers");
    CCS_CUDA_TRY(cudaMemcpy(ds.p, states.data(), 20ull * n_states, cudaMemcpyHostToDevice));
    const int grid = h->sms * 8;
    cudaEvent_t a, b;
    CCS_CUDA_TRY(cudaEventCreate(&a));
    CCS_CUDA_TRY(cudaEventCreate(&b));
    float t = 0;
    CCS_TRY(dispatch_kind(h->kind, [&](auto M, auto N) {
        return dispatch_fmt(h->format, [&](auto F) {
            constexpr int MODE = decltype(M)::value, NEC = decltype(N)::value, FMT = decltype(F)::value;
            k_probe_only<MODE, NEC, FMT><<<grid, 256>>>(h->d_tables, h->d_classidx, ds.p, n_states, h->d_table, 4, sink.p);
            CCS_CUDA_TRY(cudaEventRecord(a));
            k_probe_only<MODE, NEC, FMT><<<grid, 256>>>(h->d_tables, h->d_classidx, ds.p, n_states, h->d_table, rounds, sink.p);
            CCS_CUDA_TRY(cudaEventRecord(b));
            CCS_CUDA_TRY(cudaEventSynchronize(b));
            CCS_CUDA_TRY(cudaEventElapsedTime(&t, a, b));
            return CCS_OK;
        });
    }));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ms) *ms = t;
    if (probes_per_s) *probes_per_s = (double)grid * 256.0 * rounds / (t * 1e-3);
    return CCS_OK;
}
