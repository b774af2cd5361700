// libccs: continuous-batching server.
//
// A service thread owns the search buffers of the handle.  Submitted cubes wait in a host queue
// until a slot is free; the thread writes the slot and an admission-ring entry into device memory
// on a copy stream while the persistent search kernel keeps running on the compute stream, so a
// new cube starts as soon as a lane picks its admission up, next to the cubes already searching.
// Lanes record finished slots in a host-mapped completion log; the thread reads the slot back,
// frees it and hands the result to ccs_server_poll.  The kernel leaves when it runs out of work
// (or after a bounded idle wait) and the thread relaunches it when cubes are in flight.
#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <cstring>
#include <deque>
#include <utility>
#include <vector>

#include "ccs_internal.h"
#include "dispatch.cuh"
#include "search_kernel.cuh"

using namespace ccs;

namespace ccs {
void fill_params(ccs_handle* h, const ccs_solve_opts* o, SearchParams* P);
int resolve_variant(const ccs_solve_opts* o, int cubes);
int grid_for(ccs_handle* h, const ccs_solve_opts* o, int variant);
int launch_kernel(ccs_handle* h, const SearchParams& P, int grid, cudaStream_t stream, int variant);
void make_slot(const uint32_t state[5], uint32_t request, uint32_t table, Slot* s);
void fill_result(const Slot& s, ccs_result* r);

struct Server {
    ccs_handle* h = nullptr;
    ccs_solve_opts opts{};
    uint32_t n_slots = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t kernel_done = nullptr;
    bool kernel_running = false;
    SearchParams P{};
    int grid = 0;
    int variant = 3;  // resolved kernel variant
    unsigned long long* done_log = nullptr;  // host-mapped
    unsigned long long* d_done_log = nullptr;
    uint32_t log_cap = 0;
    unsigned long long consumed = 0;
    unsigned long long admit_pos = 0;
    std::vector<uint32_t> free_slots;
    std::vector<uint64_t> slot_request;
    std::vector<uint32_t> slot_gen;  // reuse count of each slot
    uint32_t in_flight = 0;
    // Device-memory budget (0: none): a cube is admitted only while the fixed footprint plus the
    // bytes of every cube in flight stays within it.
    uint64_t budget = 0, fixed_bytes = 0, per_cube = 0;
    uint32_t peak_in_flight = 0;

    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    int error = CCS_OK;
    std::string error_msg;
    uint64_t next_id = 1;
    std::deque<std::pair<uint64_t, std::array<uint32_t, 6>>> pending;  // state words, table id
    std::deque<std::pair<uint64_t, ccs_result>> finished;
    std::thread thread;

    int step();
    void run();
};

int Server::step() {
    // 1. completions
    for (;;) {
        unsigned long long e = ((volatile unsigned long long*)done_log)[consumed % log_cap];
        if ((e >> 32) != consumed / log_cap + 1) break;
        uint32_t s = (uint32_t)e;
        Slot sl;
        CCS_CUDA_TRY(cudaMemcpyAsync(&sl, h->d_slots + s, sizeof sl, cudaMemcpyDeviceToHost, copy));
        CCS_CUDA_TRY(cudaStreamSynchronize(copy));
        ccs_result r;
        fill_result(sl, &r);
        {
            std::lock_guard<std::mutex> lock(mu);
            finished.emplace_back(slot_request[s], r);
        }
        free_slots.push_back(s);
        --in_flight;
        ++consumed;
    }
    // 2. admissions
    std::vector<std::pair<uint64_t, std::array<uint32_t, 6>>> take;
    {
        std::lock_guard<std::mutex> lock(mu);
        while (!pending.empty() && take.size() < free_slots.size() &&
               (budget == 0 || fixed_bytes + (in_flight + take.size() + 1) * per_cube <= budget)) {
            take.push_back(pending.front());
            pending.pop_front();
        }
    }
    if (!take.empty()) {
        for (auto& t : take) {
            uint32_t s = free_slots.back();
            free_slots.pop_back();
            slot_request[s] = t.first;
            Slot sl;
            make_slot(t.second.data(), (uint32_t)t.first, t.second[5], &sl);
            sl.gen = ++slot_gen[s] & GEN_MASK;  // tells an entry left from the slot's last cube apart
            CCS_CUDA_TRY(cudaMemcpyAsync(h->d_slots + s, &sl, sizeof sl, cudaMemcpyHostToDevice, copy));
            unsigned long long pos = admit_pos++;
            unsigned long long entry = ((pos / P.admit_cap) << 32) | s;
            CCS_CUDA_TRY(cudaMemcpyAsync(P.admit + pos % P.admit_cap, &entry, 8, cudaMemcpyHostToDevice, copy));
            CCS_CUDA_TRY(cudaStreamSynchronize(copy));  // slot and entry land before the tail moves
            ++in_flight;
        }
        if (in_flight > peak_in_flight) peak_in_flight = in_flight;
        unsigned long long tail = admit_pos;
        CCS_CUDA_TRY(cudaMemcpyAsync(&h->d_q->admit_tail, &tail, 8, cudaMemcpyHostToDevice, copy));
        CCS_CUDA_TRY(cudaStreamSynchronize(copy));
    }
    // 3. keep a search launch running while cubes are in flight
    if (kernel_running && cudaEventQuery(kernel_done) == cudaSuccess) kernel_running = false;
    if (!kernel_running && in_flight > 0) {
        CCS_TRY(launch_kernel(h, P, grid, h->stream, variant));
        CCS_CUDA_TRY(cudaEventRecord(kernel_done, h->stream));
        kernel_running = true;
    }
    return CCS_OK;
}

void Server::run() {
    while (true) {
        {
            std::unique_lock<std::mutex> lock(mu);
            if (stop) break;
            if (pending.empty() && in_flight == 0) cv.wait_for(lock, std::chrono::milliseconds(2));
            if (stop) break;
        }
        int rc = step();
        if (rc != CCS_OK) {
            std::lock_guard<std::mutex> lock(mu);
            error = rc;
            error_msg = g_last_error;
            stop = true;
            break;
        }
        if (in_flight > 0) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

int server_stop(ccs_handle* h) {
    Server* s = h->server;
    if (!s) return CCS_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->thread.joinable()) s->thread.join();
    // Ask the lanes to drop their items and leave, then wait for the launch to end.
    uint32_t one = 1;
    cudaMemcpyAsync(&h->d_q->yield, &one, 4, cudaMemcpyHostToDevice, s->copy);
    cudaStreamSynchronize(s->copy);
    cudaStreamSynchronize(h->stream);
    if (s->done_log) cudaFreeHost(s->done_log);
    if (s->copy) cudaStreamDestroy(s->copy);
    if (s->kernel_done) cudaEventDestroy(s->kernel_done);
    h->server = nullptr;
    delete s;
    return CCS_OK;
}

// Bytes of device memory a cube in flight holds: its slot, four work-ring positions and its
// admission entry.  The search stacks are per lane (local memory of the persistent launch), fixed
// by the grid whatever the number of cubes, so they count in the fixed footprint.
constexpr uint64_t SERVER_BYTES_PER_CUBE = sizeof(Slot) + 5ull * sizeof(unsigned long long);
constexpr uint32_t SERVER_MAX_SLOTS = 65536;

template <int MODE, int NEC>
int kernel_footprint_kind(ccs_handle* h, int variant, size_t* local_bytes, int* threads);

// The automatic server shape is 256 x 2 with sibling lookahead (variant 2), the low-latency one:
// on B200 a stream at 10 requests/s has a p50 of 21 ms with it and 46 ms with 256 x 3; at 100
// requests/s (90% uniform, 9% of length >= 18, 1% superflips) 256 x 3 is ahead (91 cubes/s
// sustained, p50 94 ms, against 87-89 cubes/s, p50 123-165 ms).
static int server_variant(const ccs_solve_opts* opts) {
    return opts && opts->variant > 0 ? resolve_variant(opts, 0) : 2;
}

// Device memory the server holds whatever the number of cubes: resident tables, constants,
// prefix lists, queue state, donation cells and the persistent launch's per-lane stacks.
int server_fixed_bytes(ccs_handle* h, const ccs_solve_opts* opts, uint64_t* out) {
    const int variant = server_variant(opts);
    const int grid = grid_for(h, opts, variant);
    size_t local = 0;
    int threads = 0;
    CCS_TRY(dispatch_kind(h->kind, [&](auto M, auto N) {
        return kernel_footprint_kind<decltype(M)::value, decltype(N)::value>(h, variant, &local, &threads);
    }));
    uint64_t prefixes = 0;
    for (int L = 0; L <= MAX_PLEN; ++L) prefixes += 4ull * h->n_prefix[L];
    *out = h->table_bytes + h->table2_bytes + sizeof(DevTables) + 153090ull * 4 + 9930ull * 6 + prefixes +
           sizeof(QueueState) + sizeof(DonationCell) * DON_CELLS + (uint64_t)local * threads * grid;
    return CCS_OK;
}

}  // namespace ccs

extern "C" int ccs_server_start_budget(ccs_handle* h, uint64_t budget_bytes, const ccs_solve_opts* opts,
                                       int* slots_out) {
    if (!h) return fail(CCS_E_ARG, "NULL handle");
    if (!h->d_table) return fail(CCS_E_STATE, "no table loaded");
    CCS_TRY(ensure_search_buffers(h, 1));  // (the prefix lists count in the fixed footprint)
    uint64_t fixed = 0;
    CCS_TRY(server_fixed_bytes(h, opts, &fixed));
    if (budget_bytes < fixed + SERVER_BYTES_PER_CUBE)
        return fail(CCS_E_NOMEM, "budget of %llu bytes: the tables, constants and stacks alone take %llu",
                    (unsigned long long)budget_bytes, (unsigned long long)fixed);
    const uint64_t fit = (budget_bytes - fixed) / SERVER_BYTES_PER_CUBE;
    const int slots = (int)(fit < SERVER_MAX_SLOTS ? fit : SERVER_MAX_SLOTS);
    CCS_TRY(ccs_server_start(h, slots, opts));
    Server* s = h->server;
    s->budget = budget_bytes;
    s->fixed_bytes = fixed;
    s->per_cube = SERVER_BYTES_PER_CUBE;
    if (slots_out) *slots_out = slots;
    return CCS_OK;
}

extern "C" int ccs_server_memory(ccs_handle* h, uint64_t* budget, uint64_t* fixed, uint64_t* per_cube,
                                 uint64_t* peak_in_flight) {
    if (!h) return fail(CCS_E_ARG, "NULL handle");
    Server* s = h->server;
    if (!s) return fail(CCS_E_STATE, "server not running");
    std::lock_guard<std::mutex> lock(s->mu);
    if (budget) *budget = s->budget;
    if (fixed) *fixed = s->fixed_bytes;
    if (per_cube) *per_cube = SERVER_BYTES_PER_CUBE;
    if (peak_in_flight) *peak_in_flight = s->peak_in_flight;
    return CCS_OK;
}

extern "C" int ccs_server_start(ccs_handle* h, int slots, const ccs_solve_opts* opts) {
    if (!h || slots <= 0) return fail(CCS_E_ARG, "bad arguments");
    if ((uint32_t)slots >= MAX_SLOTS) return fail(CCS_E_ARG, "%d slots: at most %u", slots, MAX_SLOTS - 1);
    if (!h->d_table) return fail(CCS_E_STATE, "no table loaded");
    if (h->server) return fail(CCS_E_STATE, "server already running");
    CCS_TRY(ensure_search_buffers(h, (uint32_t)slots));
    auto s = std::make_unique<Server>();
    s->h = h;
    if (opts) s->opts = *opts;
    s->n_slots = (uint32_t)slots;
    CCS_CUDA_TRY(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking));
    CCS_CUDA_TRY(cudaEventCreateWithFlags(&s->kernel_done, cudaEventDisableTiming));
    s->log_cap = 2u * (uint32_t)slots + 64u;
    CCS_CUDA_TRY(cudaHostAlloc(&s->done_log, 8ull * s->log_cap, cudaHostAllocMapped));
    std::memset(s->done_log, 0, 8ull * s->log_cap);
    CCS_CUDA_TRY(cudaHostGetDevicePointer(&s->d_done_log, s->done_log, 0));
    fill_params(h, opts, &s->P);
    s->P.n_slots = (uint32_t)slots;
    s->P.persistent = 1;
    // Served cubes keep the plain deeper thresholds: with the few-cube rule on, the served
    // stream's p50 rose from 43 to 131 ms on B200 (it pays off for a lone batch or plain solve).
    s->P.few_max_active = 0;
    s->P.idle_limit = 1u << 16;  // ~0.25 s of idle polling, then the launch ends (relaunched on demand)
    // Served streams steal with whole idle warps asking (opts->steal 0 or 2; 1: any idle lane
    // asks; < 0: off).  Measured on B200 (256 x 2 with lookahead; 90% uniform, 9% of length >= 18,
    // 1% superflips): sustained 86.8-89.0 cubes/s at 100 requests/s with whole warps asking, 77.8
    // with any lane asking, 75.4 without stealing.
    if (!opts || opts->steal == 0) s->P.don_eager = 0u;
    // A live head entry moves to the tail once the queue spans half the scan window (opts->rotate
    // -1: half the ring): under overload one long-lived entry otherwise holds the head while
    // arrivals queue past the lanes' reach.  Measured on B200 at 200 requests/s (the mix above):
    // uniform cubes' p95 latency 1.9-2.5 s with it, 9-57 s without.
    if (!opts || opts->rotate >= 0) s->P.head_limit = std::max<unsigned long long>(s->P.spread / 2u, 32u);
    s->P.done_log = s->d_done_log;
    s->P.done_log_cap = s->log_cap;
    s->variant = server_variant(opts);
    s->grid = grid_for(h, opts, s->variant);
    QueueState q;
    std::memset(&q, 0, sizeof q);
    CCS_CUDA_TRY(cudaMemsetAsync(h->d_ring, 0xFF, sizeof(unsigned long long) * (h->ring_cap + h->slot_cap), s->copy));
    CCS_CUDA_TRY(cudaMemsetAsync(h->d_don, 0, sizeof(DonationCell) * DON_CELLS, s->copy));
    CCS_CUDA_TRY(cudaMemcpyAsync(h->d_q, &q, sizeof q, cudaMemcpyHostToDevice, s->copy));
    CCS_CUDA_TRY(cudaStreamSynchronize(s->copy));
    s->slot_request.assign(h->slot_cap, 0);
    s->slot_gen.assign(h->slot_cap, 0);
    for (uint32_t i = (uint32_t)slots; i-- > 0;) s->free_slots.push_back(i);
    Server* raw = s.release();
    h->server = raw;
    raw->thread = std::thread([raw] { raw->run(); });
    return CCS_OK;
}

extern "C" int ccs_server_submit(ccs_handle* h, const uint32_t* state, uint64_t* request_id) {
    return ccs_server_submit_table(h, state, 0, request_id);
}

extern "C" int ccs_server_submit_table(ccs_handle* h, const uint32_t* state, int table_id, uint64_t* request_id) {
    if (!h || !state) return fail(CCS_E_ARG, "NULL argument");
    Server* s = h->server;
    if (!s) return fail(CCS_E_STATE, "server not running");
    if (!is_legal(unpack(state))) return fail(CCS_E_ARG, "not a legal position");
    if (table_id < 0 || table_id > 1 || (table_id == 1 && !h->d_table2))
        return fail(CCS_E_ARG, "table id %d: 0, or 1 with a second table attached", table_id);
    std::array<uint32_t, 6> st;
    std::memcpy(st.data(), state, 20);
    st[5] = (uint32_t)table_id;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stop) return fail(s->error ? s->error : CCS_E_STATE, "server stopped: %s", s->error_msg.c_str());
        uint64_t id = s->next_id++;
        s->pending.emplace_back(id, st);
        if (request_id) *request_id = id;
    }
    s->cv.notify_all();
    return CCS_OK;
}

extern "C" int ccs_server_poll(ccs_handle* h, int max_out, uint64_t* request_ids, ccs_result* results, int* n_out) {
    if (!h || !n_out || (max_out > 0 && (!request_ids || !results))) return fail(CCS_E_ARG, "NULL argument");
    Server* s = h->server;
    if (!s) return fail(CCS_E_STATE, "server not running");
    std::lock_guard<std::mutex> lock(s->mu);
    int k = 0;
    while (k < max_out && !s->finished.empty()) {
        request_ids[k] = s->finished.front().first;
        results[k] = s->finished.front().second;
        s->finished.pop_front();
        ++k;
    }
    *n_out = k;
    if (k == 0 && s->error) return fail(s->error, "server stopped: %s", s->error_msg.c_str());
    return CCS_OK;
}

extern "C" int ccs_server_stop(ccs_handle* h) {
    if (!h) return fail(CCS_E_ARG, "NULL handle");
    return server_stop(h);
}
