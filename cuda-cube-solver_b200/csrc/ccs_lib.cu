// libccs: the C ABI of include/ccs.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/ccs.h"
#include "ccs_internal.h"
#include "cube_dev.cuh"

using namespace ccs;

// ---- errors ----------------------------------------------------------------------------

namespace ccs {
thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}
}  // namespace ccs

#define CUDA_TRY CCS_CUDA_TRY
#define TRY CCS_TRY

// ---- kinds -------------------------------------------------------------------------------

namespace ccs {
static std::mutex g_kind_mutex;
static std::map<std::string, KindDesc> g_kinds;

int get_kind(const char* name, KindDesc* out) {
    if (!name) return fail(CCS_E_ARG, "kind name is NULL");
    std::lock_guard<std::mutex> lock(g_kind_mutex);
    auto it = g_kinds.find(name);
    if (it == g_kinds.end()) {
        KindDesc k;
        try {
            if (!preset_kind(name, &k)) return fail(CCS_E_ARG, "unknown table kind %s", name);
        } catch (const std::exception& e) {
            return fail(CCS_E_ARG, "%s", e.what());
        }
        it = g_kinds.emplace(name, k).first;
    }
    *out = it->second;
    return CCS_OK;
}

bool kind_supported(const KindDesc& k) {
    return k.mode == KIND_304 || (k.mode == KIND_GEN && (k.nec == 8 || k.nec == 12 || k.nec == 16 || k.nec == 24));
}

uint64_t table_bytes_for(const KindDesc& k, int fmt) {
    uint64_t per = fmt == CCS_FMT_B3 ? B3_ENTRIES : BLOCK_ENTRIES;
    return (k.n_entries + per - 1) / per * 32ull;
}
}  // namespace ccs

#include "dispatch.cuh"

// ---- utility kernels ---------------------------------------------------------------------

template <int MODE, int NEC>
__global__ void k_index(const DevTables* __restrict__ gT, const uint32_t* __restrict__ classidx,
                        const uint32_t* __restrict__ states, int n, int move, uint64_t* __restrict__ out_idx,
                        uint32_t* __restrict__ out_states) {
    __shared__ DevTables T;
    stage_tables(T, gT);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    State s{states[5 * i], states[5 * i + 1], states[5 * i + 2], states[5 * i + 3], states[5 * i + 4]};
    if (move >= 0) move_right(T, s, move);
    if (move <= -2) move_left(T, s, -2 - move);
    out_idx[i] = table_index_dev<MODE, NEC>(T, classidx, s);
    out_states[5 * i] = s.c0;
    out_states[5 * i + 1] = s.c1;
    out_states[5 * i + 2] = s.e0;
    out_states[5 * i + 3] = s.e1;
    out_states[5 * i + 4] = s.e2;
}

template <int MODE, int NEC>
__global__ void k_unrank(const DevTables* __restrict__ gT, const uint32_t* __restrict__ class_rep,
                         const uint64_t* __restrict__ idx, int n, uint32_t* __restrict__ out_states) {
    __shared__ DevTables T;
    stage_tables(T, gT);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    State s;
    unrank_dev<MODE, NEC>(T, class_rep, idx[i], s);
    out_states[5 * i] = s.c0;
    out_states[5 * i + 1] = s.c1;
    out_states[5 * i + 2] = s.e0;
    out_states[5 * i + 3] = s.e1;
    out_states[5 * i + 4] = s.e2;
}

template <int MODE, int NEC, int FMT>
__global__ void k_lower_bound(const DevTables* __restrict__ gT, const uint32_t* __restrict__ classidx,
                              const uint32_t* __restrict__ table, const uint32_t* __restrict__ states, int n,
                              uint32_t* __restrict__ out) {
    __shared__ DevTables T;
    stage_tables(T, gT);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    State s{states[5 * i], states[5 * i + 1], states[5 * i + 2], states[5 * i + 3], states[5 * i + 4]};
    out[i] = lower_bound_dev<FMT>(table, table_index_dev<MODE, NEC>(T, classidx, s));
}

// ---- handle ------------------------------------------------------------------------------

namespace ccs {

int set_kind(ccs_handle* h, const char* name) {
    KindDesc k;
    TRY(get_kind(name, &k));
    if (!kind_supported(k)) return fail(CCS_E_ARG, "kind %s: %d E-content classes are not compiled in", name, k.nec);
    if (h->kind_ready && h->kind_name == name) return CCS_OK;
    CUDA_TRY(cudaSetDevice(h->device));
    if (!h->d_tables) {
        CUDA_TRY(cudaMalloc(&h->d_tables, sizeof(DevTables)));
        const CornerClasses& cc = corner_classes();
        CUDA_TRY(cudaMalloc(&h->d_classidx, cc.classidx.size() * 4));
        CUDA_TRY(cudaMalloc(&h->d_class_rep, cc.rep.size() * 4));
        CUDA_TRY(cudaMalloc(&h->d_class_stab, cc.stab.size() * 2));
        CUDA_TRY(cudaMemcpy(h->d_classidx, cc.classidx.data(), cc.classidx.size() * 4, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(h->d_class_rep, cc.rep.data(), cc.rep.size() * 4, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(h->d_class_stab, cc.stab.data(), cc.stab.size() * 2, cudaMemcpyHostToDevice));
    }
    auto T = std::make_unique<DevTables>();
    build_dev_tables(k, T.get());
    CUDA_TRY(cudaMemcpy(h->d_tables, T.get(), sizeof(DevTables), cudaMemcpyHostToDevice));
    h->kind = k;
    h->kind_name = name;
    h->kind_ready = true;
    return CCS_OK;
}

void free_table(ccs_handle* h) {
    if (h->d_table) cudaFree(h->d_table);
    h->d_table = nullptr;
    h->table_bytes = 0;
    h->format = -1;
    if (h->d_table2) cudaFree(h->d_table2);
    h->d_table2 = nullptr;
    h->table2_bytes = 0;
    h->kind2_name.clear();
}

}  // namespace ccs

// ---- public API --------------------------------------------------------------------------

extern "C" {

int ccs_version(void) { return (0 << 16) | 1; }

const char* ccs_last_error(void) { return g_last_error.c_str(); }

int ccs_mem_info(int device, uint64_t* free_bytes, uint64_t* total_bytes) {
    CUDA_TRY(cudaSetDevice(device));
    size_t f = 0, t = 0;
    CUDA_TRY(cudaMemGetInfo(&f, &t));
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return CCS_OK;
}

int ccs_device_sms(int device, int* sms) {
    CUDA_TRY(cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, device));
    return CCS_OK;
}

int ccs_open(int device, ccs_handle** out) {
    if (!out) return fail(CCS_E_ARG, "out is NULL");
    auto h = std::make_unique<ccs_handle>();
    h->device = device;
    CUDA_TRY(cudaSetDevice(device));
    CUDA_TRY(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device));
    CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreate(&h->ev0));
    CUDA_TRY(cudaEventCreate(&h->ev1));
    *out = h.release();
    return CCS_OK;
}

int ccs_close(ccs_handle* h) {
    if (!h) return CCS_OK;
    cudaSetDevice(h->device);
    if (h->server) server_stop(h);
    free_table(h);
    cudaFree(h->d_tables);
    cudaFree(h->d_classidx);
    cudaFree(h->d_class_rep);
    cudaFree(h->d_class_stab);
    cudaFree(h->d_slots);
    cudaFree(h->d_q);
    cudaFree(h->d_ring);
    cudaFree(h->d_don);
    for (auto* p : h->d_prefix) cudaFree(p);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CCS_OK;
}

int ccs_kind_info(const char* kind, int* nec, uint64_t* n_entries) {
    KindDesc k;
    TRY(get_kind(kind, &k));
    if (nec) *nec = k.nec;
    if (n_entries) *n_entries = k.n_entries;
    return CCS_OK;
}

int ccs_register_group_kind(const char* name, int n_gens, const int32_t* perms, const int32_t* flips) {
    if (!name || n_gens < 0 || (n_gens && (!perms || !flips))) return fail(CCS_E_ARG, "bad generator arguments");
    std::vector<std::pair<std::vector<int>, std::vector<int>>> gens;
    for (int i = 0; i < n_gens; ++i)
        gens.push_back({std::vector<int>(perms + 4 * i, perms + 4 * i + 4), std::vector<int>(flips + 4 * i, flips + 4 * i + 4)});
    try {
        KindDesc k = make_group_kind(name, gens);
        std::lock_guard<std::mutex> lock(g_kind_mutex);
        g_kinds[name] = k;
    } catch (const std::exception& e) {
        return fail(CCS_E_ARG, "%s", e.what());
    }
    return CCS_OK;
}

int ccs_kind_tables(const char* kind, uint32_t* classidx, uint32_t* class_rep, uint16_t* class_stab,
                    uint16_t* gen_class, uint16_t* gen_rep) {
    KindDesc k;
    TRY(get_kind(kind, &k));
    const CornerClasses& cc = corner_classes();
    if (classidx) std::memcpy(classidx, cc.classidx.data(), cc.classidx.size() * 4);
    if (class_rep) std::memcpy(class_rep, cc.rep.data(), cc.rep.size() * 4);
    if (class_stab) std::memcpy(class_stab, cc.stab.data(), cc.stab.size() * 2);
    if (gen_class) std::memcpy(gen_class, k.gen_class, sizeof k.gen_class);
    if (gen_rep) std::memcpy(gen_rep, k.gen_rep, sizeof k.gen_rep);
    return CCS_OK;
}

int ccs_set_kind(ccs_handle* h, const char* kind) {
    if (!h) return fail(CCS_E_ARG, "NULL handle");
    return set_kind(h, kind);
}

int ccs_table_bytes(ccs_handle* h, uint64_t* n_bytes) {
    if (!h || !n_bytes) return fail(CCS_E_ARG, "NULL argument");
    *n_bytes = h->table_bytes;
    return CCS_OK;
}

int ccs_table_copy(ccs_handle* h, void* dst, uint64_t n_bytes) {
    if (!h || !dst) return fail(CCS_E_ARG, "NULL argument");
    if (!h->d_table) return fail(CCS_E_STATE, "no table loaded");
    if (n_bytes != h->table_bytes) return fail(CCS_E_ARG, "buffer is %llu bytes, table %llu", (unsigned long long)n_bytes,
                                               (unsigned long long)h->table_bytes);
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaMemcpy(dst, h->d_table, n_bytes, cudaMemcpyDeviceToHost));
    return CCS_OK;
}

int ccs_index(ccs_handle* h, const uint32_t* states, int n, int move, uint64_t* out_idx, uint32_t* out_states) {
    if (!h || (n > 0 && (!states || !out_idx))) return fail(CCS_E_ARG, "NULL argument");
    if (!h->kind_ready) return fail(CCS_E_STATE, "no table kind selected (load or build a table first)");
    if (n <= 0) return CCS_OK;
    if (move < -19 || move > 17) return fail(CCS_E_ARG, "move %d out of range", move);
    CUDA_TRY(cudaSetDevice(h->device));
    DeviceBuffer<uint32_t> ds(5ull * n), dso(5ull * n);
    DeviceBuffer<uint64_t> di(n);
    if (!ds.ok() || !dso.ok() || !di.ok()) return fail(CCS_E_NOMEM, "device allocation failed");
    CUDA_TRY(cudaMemcpyAsync(ds.p, states, 20ull * n, cudaMemcpyHostToDevice, h->stream));
    TRY(dispatch_kind(h->kind, [&](auto M, auto N) {
        k_index<decltype(M)::value, decltype(N)::value><<<(n + 127) / 128, 128, 0, h->stream>>>(
            h->d_tables, h->d_classidx, ds.p, n, move, di.p, dso.p);
        return CCS_OK;
    }));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out_idx, di.p, 8ull * n, cudaMemcpyDeviceToHost, h->stream));
    if (out_states) CUDA_TRY(cudaMemcpyAsync(out_states, dso.p, 20ull * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return CCS_OK;
}

int ccs_unrank(ccs_handle* h, const uint64_t* idx, int n, uint32_t* out_states) {
    if (!h || (n > 0 && (!idx || !out_states))) return fail(CCS_E_ARG, "NULL argument");
    if (!h->kind_ready) return fail(CCS_E_STATE, "no table kind selected (load or build a table first)");
    if (n <= 0) return CCS_OK;
    for (int i = 0; i < n; ++i)
        if (idx[i] >= h->kind.n_entries) return fail(CCS_E_ARG, "index %llu out of range", (unsigned long long)idx[i]);
    CUDA_TRY(cudaSetDevice(h->device));
    DeviceBuffer<uint64_t> di(n);
    DeviceBuffer<uint32_t> ds(5ull * n);
    if (!ds.ok() || !di.ok()) return fail(CCS_E_NOMEM, "device allocation failed");
    CUDA_TRY(cudaMemcpyAsync(di.p, idx, 8ull * n, cudaMemcpyHostToDevice, h->stream));
    TRY(dispatch_kind(h->kind, [&](auto M, auto N) {
        k_unrank<decltype(M)::value, decltype(N)::value><<<(n + 127) / 128, 128, 0, h->stream>>>(
            h->d_tables, h->d_class_rep, di.p, n, ds.p);
        return CCS_OK;
    }));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out_states, ds.p, 20ull * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return CCS_OK;
}

int ccs_lower_bound(ccs_handle* h, const uint32_t* states, int n, uint32_t* out) {
    if (!h || (n > 0 && (!states || !out))) return fail(CCS_E_ARG, "NULL argument");
    if (!h->d_table) return fail(CCS_E_STATE, "no table loaded");
    if (n <= 0) return CCS_OK;
    CUDA_TRY(cudaSetDevice(h->device));
    DeviceBuffer<uint32_t> ds(5ull * n), dout(n);
    if (!ds.ok() || !dout.ok()) return fail(CCS_E_NOMEM, "device allocation failed");
    CUDA_TRY(cudaMemcpyAsync(ds.p, states, 20ull * n, cudaMemcpyHostToDevice, h->stream));
    TRY(dispatch_kind(h->kind, [&](auto M, auto N) {
        return dispatch_fmt(h->format, [&](auto F) {
            k_lower_bound<decltype(M)::value, decltype(N)::value, decltype(F)::value>
                <<<(n + 127) / 128, 128, 0, h->stream>>>(h->d_tables, h->d_classidx, h->d_table, ds.p, n, dout.p);
            return CCS_OK;
        });
    }));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, dout.p, 4ull * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return CCS_OK;
}

int ccs_root_bounds(ccs_handle* h, const uint32_t* states, int n, uint32_t* out_h6) {
    if (!h || (n > 0 && (!states || !out_h6))) return fail(CCS_E_ARG, "NULL argument");
    if (n <= 0) return CCS_OK;
    std::vector<uint32_t> frames(30ull * n);
    for (int i = 0; i < n; ++i) cube_frames(states + 5ull * i, frames.data() + 30ull * i);
    return ccs_lower_bound(h, frames.data(), 6 * n, out_h6);
}

}  // extern "C"
