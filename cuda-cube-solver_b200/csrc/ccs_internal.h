// Internal declarations shared by the libccs translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ccs.h"
#include "cube_model.h"
#include "dev_tables.h"
#include "search.cuh"

namespace ccs {

extern thread_local std::string g_last_error;
int fail(int code, const char* fmt, ...);

#define CCS_CUDA_TRY(expr)                                                                              \
    do {                                                                                                \
        cudaError_t _e = (expr);                                                                        \
        if (_e != cudaSuccess)                                                                          \
            return ::ccs::fail(_e == cudaErrorMemoryAllocation ? CCS_E_NOMEM : CCS_E_CUDA, "%s: %s (%s:%d)", \
                               #expr, cudaGetErrorString(_e), __FILE__, __LINE__);                      \
    } while (0)

#define CCS_TRY(expr)                \
    do {                             \
        int _r = (expr);             \
        if (_r != CCS_OK) return _r; \
    } while (0)

template <typename T>
struct DeviceBuffer {
    T* p = nullptr;
    explicit DeviceBuffer(size_t n) {
        if (cudaMalloc(&p, n * sizeof(T) + 16) != cudaSuccess) p = nullptr;
    }
    ~DeviceBuffer() {
        if (p) cudaFree(p);
    }
    bool ok() const { return p != nullptr; }
    T* release() {  // the caller owns the allocation from here on (cudaFree)
        T* q = p;
        p = nullptr;
        return q;
    }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

int get_kind(const char* name, KindDesc* out);
bool kind_supported(const KindDesc& k);
uint64_t table_bytes_for(const KindDesc& k, int fmt);

// The six search frames of a packed state: g, R g R^-1, R^2 g R^-2, then their inverses
// (solver.frames, solver.py:58-64); out[30].
void cube_frames(const uint32_t state[5], uint32_t out[30]);

// Canonical move sequences of a length in the reference's order (solver.canonical_prefixes,
// solver.py:33-48), packed 5 bits per move, first move in the low bits.
std::vector<uint32_t> canonical_prefixes(int length);

struct Server;

}  // namespace ccs

struct ccs_handle {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    std::string kind_name;
    ccs::KindDesc kind;
    bool kind_ready = false;
    ccs::DevTables* d_tables = nullptr;
    uint32_t* d_classidx = nullptr;
    uint32_t* d_class_rep = nullptr;
    uint16_t* d_class_stab = nullptr;
    int format = -1;
    uint32_t* d_table = nullptr;
    uint64_t table_bytes = 0;
    // optional second resident table of a compatible kind (same class count and format)
    std::string kind2_name;
    uint32_t* d_table2 = nullptr;
    uint64_t table2_bytes = 0;
    ccs::Slot* d_slots = nullptr;
    uint32_t slot_cap = 0;
    ccs::QueueState* d_q = nullptr;
    unsigned long long* d_ring = nullptr;
    uint32_t ring_cap = 0;
    ccs::DonationCell* d_don = nullptr;  // work-stealing cells (ccs::DON_CELLS)
    uint32_t* d_prefix[ccs::MAX_PLEN + 1] = {};
    uint32_t n_prefix[ccs::MAX_PLEN + 1] = {};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_kernel_ms = 0;
    uint64_t last_probes = 0;
    uint64_t last_donated = 0;
    uint64_t last_h2d = 0, last_d2h = 0;
    int last_launches = 0;
    ccs::Server* server = nullptr;
    std::vector<ccs_bfs_pass> last_passes;  // the last table build's BFS passes
};

namespace ccs {
constexpr uint32_t DON_CELLS = 4096;  // donation cells of a handle's search buffers (128 KB)
int set_kind(ccs_handle* h, const char* name);
void free_table(ccs_handle* h);
int ensure_search_buffers(ccs_handle* h, uint32_t slots);
int launch_search(ccs_handle* h, const ccs_solve_opts* opts, cudaStream_t stream, SearchParams* params_out);
int server_stop(ccs_handle* h);
}  // namespace ccs
