// libccs: batched solving that allocates nothing.
//
// Some callers cannot allocate device memory at solve time: a process whose device memory is
// owned by a caching pool or a framework allocator (a cudaMalloc of its own would fragment that
// pool or fail because the pool holds the memory), or a solver embedded in a service that fixes
// its memory footprint at start-up.  ccs_solve_noalloc serves them: it runs the same search kernel
// as ccs_solve, but the search buffers (cube slots, queue state, work and admission rings, prefix
// lists) are one file-scope __device__ array of fixed size, part of the library's image on every
// GPU that loads it, and the host staging is file-scope host arrays.  The first call on a device
// (made with that device current) takes the array's device address with cudaGetSymbolAddress and
// uploads the prefix lists; make that first call before any stream capture.  Later calls copy the
// cubes in, clear the queue state and the rings, launch and read back.
//
// Limits: at most CCS_NOALLOC_MAX_CUBES cubes per call; prefixes of at most NOALLOC_MAX_PLEN
// moves, so an iteration of a very large tree keeps the base prefix length instead of a longer
// one (deeper_at0/1 are ignored); the first table only; at most NA_MAX_DEVICES devices.  One
// array per process and device, shared by every handle on that device: calls on one device are
// serialised by a per-device lock (they would race on the array otherwise), and the host staging
// is per device too, so calls on different devices run side by side.  A device reset reloads the
// array zeroed; a marker word in it tells the next call to set it up again.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <mutex>

#include "ccs_internal.h"

using namespace ccs;

namespace ccs {
void fill_params(ccs_handle* h, const ccs_solve_opts* o, SearchParams* P);
int resolve_variant(const ccs_solve_opts* o, int cubes);
int grid_for(ccs_handle* h, const ccs_solve_opts* o, int variant);
int launch_kernel(ccs_handle* h, const SearchParams& P, int grid, cudaStream_t stream, int variant);
void make_slot(const uint32_t state[5], uint32_t request, uint32_t table, Slot* s);
void fill_result(const Slot& s, ccs_result* r);
}  // namespace ccs

namespace {

constexpr int NOALLOC_MAX_PLEN = 4;
constexpr uint32_t NA_SLOTS = CCS_NOALLOC_MAX_CUBES;
constexpr uint32_t NA_RING = 4 * NA_SLOTS + 64;  // the allocating path's sizing
// canonical move sequences of length 0..4
constexpr uint32_t NA_PREFIX_COUNT[NOALLOC_MAX_PLEN + 1] = {1, 18, 243, 3240, 43254};
constexpr uint32_t NA_PREFIX_TOTAL = 1 + 18 + 243 + 3240 + 43254;

constexpr uint32_t NA_MARKER = 0x43435331u;  // "CCS1": the array has been set up on this device

struct NoAllocScratch {
    Slot slots[NA_SLOTS];
    QueueState q;
    uint32_t marker;  // NA_MARKER once the prefix lists are in place
    uint32_t pad[3];
    unsigned long long ring[NA_RING + NA_SLOTS];  // work ring, then the admission ring
    uint32_t prefix[NA_PREFIX_TOTAL];
};

static_assert(sizeof(NoAllocScratch) <= 320u * 1024u, "the fixed search buffers stay small");

// 304 KB of device memory, held by every GPU that loads the library until the process exits.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int NA_MAX_DEVICES = 16;

// Per device: the array's device address (found at set-up), the lock that serialises calls, and
// the host staging of a call (file scope: nothing is allocated per call).
struct DeviceState {
    NoAllocScratch* scratch = nullptr;
    std::mutex mu;
    Slot slots[NA_SLOTS];
    unsigned long long admit[NA_SLOTS];
};
DeviceState g_dev[NA_MAX_DEVICES];
uint32_t g_host_prefix[NA_PREFIX_TOTAL];  // written once, under g_prefix_mutex
std::mutex g_prefix_mutex;

// Canonical sequences of length `len` in lexicographic move order (the order of
// canonical_prefixes), 5 bits per move, first move lowest; returns the next free position.
uint32_t enumerate_prefixes(int len, int depth, int last, uint32_t seq, uint32_t* out, uint32_t pos) {
    if (depth == len) {
        out[pos] = seq;
        return pos + 1;
    }
    for (int m = 0; m < 18; ++m) {
        int lf = last / 3, mf = m / 3;
        if (last >= 0 && (mf == lf || (lf >= 3 && mf == lf - 3))) continue;
        pos = enumerate_prefixes(len, depth + 1, m, seq | ((uint32_t)m << (5 * depth)), out, pos);
    }
    return pos;
}

// With `device` current and its lock held: the array's device address, found and filled with the
// prefix lists on the first call for this device, and again after a device reset (the reloaded
// array has no marker).  The copies run on `st` and are complete when this returns.
int setup_device(int device, cudaStream_t st, NoAllocScratch** out) {
    DeviceState& D = g_dev[device];
    if (D.scratch) {
        uint32_t marker = 0;
        CCS_CUDA_TRY(cudaMemcpyAsync(&marker, &D.scratch->marker, sizeof marker, cudaMemcpyDeviceToHost, st));
        CCS_CUDA_TRY(cudaStreamSynchronize(st));
        if (marker != NA_MARKER) D.scratch = nullptr;
    }
    if (!D.scratch) {
        NoAllocScratch* p = nullptr;
        CCS_CUDA_TRY(cudaGetSymbolAddress((void**)&p, g_noalloc_scratch));
        {
            std::lock_guard<std::mutex> lock(g_prefix_mutex);
            uint32_t pos = 0;
            for (int L = 0; L <= NOALLOC_MAX_PLEN; ++L) {
                uint32_t end = enumerate_prefixes(L, 0, -1, 0u, g_host_prefix, pos);
                if (end - pos != NA_PREFIX_COUNT[L]) return fail(CCS_E_CHECK, "prefix count of length %d", L);
                pos = end;
            }
            CCS_CUDA_TRY(cudaMemcpyAsync(p->prefix, g_host_prefix, sizeof g_host_prefix, cudaMemcpyHostToDevice, st));
            CCS_CUDA_TRY(cudaStreamSynchronize(st));
        }
        static const uint32_t marker = NA_MARKER;
        CCS_CUDA_TRY(cudaMemcpyAsync(&p->marker, &marker, sizeof marker, cudaMemcpyHostToDevice, st));
        CCS_CUDA_TRY(cudaStreamSynchronize(st));
        D.scratch = p;
    }
    *out = D.scratch;
    return CCS_OK;
}

}  // namespace

extern "C" int ccs_solve_noalloc(ccs_handle* h, const uint32_t* states, int n, const ccs_solve_opts* opts,
                                 ccs_result* results) {
    if (!h || (n > 0 && (!states || !results))) return fail(CCS_E_ARG, "NULL argument");
    if (!h->d_table) return fail(CCS_E_STATE, "no table loaded");
    if (h->server) return fail(CCS_E_STATE, "the server is running on this handle");
    if (n < 0 || n > CCS_NOALLOC_MAX_CUBES)
        return fail(CCS_E_ARG, "%d cubes: ccs_solve_noalloc takes at most %d per call", n, CCS_NOALLOC_MAX_CUBES);
    if (opts && opts->base_plen > NOALLOC_MAX_PLEN)
        return fail(CCS_E_ARG, "base_plen %d: ccs_solve_noalloc takes prefixes of at most %d moves",
                    opts->base_plen, NOALLOC_MAX_PLEN);
    if (h->device < 0 || h->device >= NA_MAX_DEVICES)
        return fail(CCS_E_ARG, "device %d: ccs_solve_noalloc serves devices 0..%d", h->device, NA_MAX_DEVICES - 1);
    for (int i = 0; i < n; ++i)
        if (!is_legal(unpack(states + 5ull * i))) return fail(CCS_E_ARG, "cube %d is not a legal position", i);
    CCS_CUDA_TRY(cudaSetDevice(h->device));
    DeviceState& D = g_dev[h->device];
    std::lock_guard<std::mutex> lock(D.mu);  // one call at a time per device: they share the array
    cudaStream_t st = h->stream;
    NoAllocScratch* S = nullptr;
    CCS_TRY(setup_device(h->device, st, &S));
    if (n == 0) return CCS_OK;

    for (int i = 0; i < n; ++i) {
        make_slot(states + 5ull * i, (uint32_t)i, 0u, &D.slots[i]);
        D.admit[i] = (unsigned long long)i;  // lap 0
    }
    QueueState q;
    std::memset(&q, 0, sizeof q);
    q.admit_tail = (unsigned long long)n;

    SearchParams P;
    fill_params(h, opts, &P);
    P.slots = S->slots;
    P.q = &S->q;
    P.ring = S->ring;
    P.ring_cap = NA_RING;
    P.admit = S->ring + NA_RING;
    P.admit_cap = NA_SLOTS;
    P.n_slots = (uint32_t)n;
    uint32_t off = 0;
    for (int L = 0; L <= MAX_PLEN; ++L) {
        const bool have = L <= NOALLOC_MAX_PLEN;
        P.prefixes[L] = have ? S->prefix + off : nullptr;
        P.n_prefix[L] = have ? NA_PREFIX_COUNT[L] : 0u;
        if (have) off += NA_PREFIX_COUNT[L];
    }
    // every iteration stays at or below the base prefix length: no longer lists exist here
    P.deeper_at[0] = P.deeper_at[1] = ~0ull;
    P.max_plen = NOALLOC_MAX_PLEN;
    P.don = nullptr;  // no work stealing: its cells would be one more buffer
    P.don_cap = 0;

    // The array keeps the previous call's contents: the slots of this call, the queue state and
    // both rings are rewritten before the launch.
    CCS_CUDA_TRY(cudaMemcpyAsync(S->slots, D.slots, sizeof(Slot) * n, cudaMemcpyHostToDevice, st));
    CCS_CUDA_TRY(cudaMemsetAsync(S->ring, 0xFF, sizeof S->ring, st));
    CCS_CUDA_TRY(cudaMemcpyAsync(P.admit, D.admit, 8ull * n, cudaMemcpyHostToDevice, st));
    CCS_CUDA_TRY(cudaMemcpyAsync(&S->q, &q, sizeof q, cudaMemcpyHostToDevice, st));

    const int variant = resolve_variant(opts, n);
    const int grid = grid_for(h, opts, variant);
    const double timeout = opts && opts->timeout_s > 0 ? opts->timeout_s : 0;
    auto t0 = std::chrono::steady_clock::now();
    double kernel_ms = 0;
    int launches = 0;
    unsigned long long prev_probes = ~0ull;
    for (;;) {
        CCS_CUDA_TRY(cudaEventRecord(h->ev0, st));
        CCS_TRY(launch_kernel(h, P, grid, st, variant));
        CCS_CUDA_TRY(cudaEventRecord(h->ev1, st));
        CCS_CUDA_TRY(cudaMemcpyAsync(&q, &S->q, sizeof q, cudaMemcpyDeviceToHost, st));
        CCS_CUDA_TRY(cudaStreamSynchronize(st));
        float ms = 0;
        CCS_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        kernel_ms += ms;
        ++launches;
        if (q.active == 0 && q.admit_head >= q.admit_tail) break;
        if (q.probes == prev_probes)
            return fail(CCS_E_CHECK, "search made no progress (%u cubes unfinished, error bits %u)", q.active, q.error);
        prev_probes = q.probes;
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (timeout > 0 && el > timeout)
            return fail(CCS_E_TIMEOUT, "solve did not finish in %.1f s (%u cubes still searching)", timeout, q.active);
        if (launches > 100000) return fail(CCS_E_TIMEOUT, "too many relaunches");
    }
    h->last_kernel_ms = kernel_ms;
    h->last_probes = q.probes;
    h->last_launches = launches;
    CCS_CUDA_TRY(cudaMemcpyAsync(D.slots, S->slots, sizeof(Slot) * n, cudaMemcpyDeviceToHost, st));
    CCS_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) fill_result(D.slots[i], &results[i]);
    if (q.error & ERR_BOUND) return fail(CCS_E_CHECK, "a search passed the largest possible bound");
    return CCS_OK;
}
