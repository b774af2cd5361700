// libccs: batched solving and the continuous-batching server.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <vector>

#include "ccs_internal.h"
#include "dispatch.cuh"
#include "search_kernel.cuh"

using namespace ccs;

namespace ccs {

int ensure_search_buffers(ccs_handle* h, uint32_t slots) {
    CCS_CUDA_TRY(cudaSetDevice(h->device));
    if (!h->d_prefix[0]) {
        for (int L = 0; L <= MAX_PLEN; ++L) {
            std::vector<uint32_t> p = canonical_prefixes(L);
            h->n_prefix[L] = (uint32_t)p.size();
            CCS_CUDA_TRY(cudaMalloc(&h->d_prefix[L], p.size() * 4));
            CCS_CUDA_TRY(cudaMemcpy(h->d_prefix[L], p.data(), p.size() * 4, cudaMemcpyHostToDevice));
        }
    }
    if (!h->d_q) CCS_CUDA_TRY(cudaMalloc(&h->d_q, sizeof(QueueState)));
    if (!h->d_don) CCS_CUDA_TRY(cudaMalloc(&h->d_don, sizeof(DonationCell) * DON_CELLS));
    if (slots > h->slot_cap) {
        cudaFree(h->d_slots);
        cudaFree(h->d_ring);
        h->d_slots = nullptr;
        h->d_ring = nullptr;
        h->slot_cap = 0;
        uint32_t cap = std::max<uint32_t>(slots, 64u);
        CCS_CUDA_TRY(cudaMalloc(&h->d_slots, sizeof(Slot) * cap));
        // work ring: 4 positions per slot (its head is kept moving, see advance_head), then the
        // admission ring: one entry per slot
        CCS_CUDA_TRY(cudaMalloc(&h->d_ring, sizeof(unsigned long long) * (5ull * cap + 64)));
        h->slot_cap = cap;
        h->ring_cap = 4 * cap + 64;
    }
    return CCS_OK;
}

void fill_params(ccs_handle* h, const ccs_solve_opts* o, SearchParams* P) {
    std::memset(P, 0, sizeof *P);
    P->slots = h->d_slots;
    P->q = h->d_q;
    P->ring = h->d_ring;
    P->ring_cap = h->ring_cap;
    P->admit = h->d_ring + h->ring_cap;
    P->admit_cap = h->slot_cap;
    P->n_slots = h->slot_cap;
    P->classidx = h->d_classidx;
    P->table = h->d_table;
    P->table2 = h->d_table2 ? h->d_table2 : h->d_table;
    for (int L = 0; L <= MAX_PLEN; ++L) {
        P->prefixes[L] = h->d_prefix[L];
        P->n_prefix[L] = h->n_prefix[L];
    }
    int base = o && o->base_plen > 0 ? o->base_plen : 4;
    P->base_plen = (uint32_t)std::min(base, MAX_PLEN);
    P->max_plen = (uint32_t)MAX_PLEN;
    P->deeper_at[0] = (unsigned long long)(o && o->deeper_at0 > 0 ? o->deeper_at0 : 5e7);
    P->deeper_at[1] = (unsigned long long)(o && o->deeper_at1 > 0 ? o->deeper_at1 : 3e9);
    // Small iterations get shorter prefixes (fewer, larger items: fewer fetches); negative = off.
    P->shallow_at[0] = (unsigned long long)(o && o->shallow_at0 != 0 ? (o->shallow_at0 > 0 ? o->shallow_at0 : 0) : 1e5);
    P->shallow_at[1] = (unsigned long long)(o && o->shallow_at1 != 0 ? (o->shallow_at1 > 0 ? o->shallow_at1 : 0) : 1.5e6);
    P->shallow_min_active = 32;
    // A lone 20-move cube on B200: deeper prefixes from 1e6 / 6e7 nodes instead of 5e7 / 3e9 took
    // the superflip from 1.66 to 0.74 s on d4 and from 12.7 to 7.5 s on d4t.
    P->few_divisor = o && o->few_divisor > 0 ? (uint32_t)o->few_divisor : 50u;
    P->few_max_active = 4;  // (the server sets 0: see ccs_server_start)
    P->idle_limit = 1u << 21;  // ~8 s of idle polling (4 us back-off) before a warp leaves
    P->spread = o && o->spread > 0 ? (uint32_t)o->spread : 4096u;
    P->move_min = o && o->move_min > 0 ? (uint32_t)o->move_min : 8u;
    P->move_age = o && o->move_age > 0 ? (uint32_t)o->move_age : 4u;
    P->probe_min = o && o->probe_min > 0 ? (uint32_t)o->probe_min : 16u;
    // Work stealing: cells of the handle, on unless opts->steal < 0.
    const bool steal = h->d_don && !(o && o->steal < 0);
    P->don = steal ? h->d_don : nullptr;
    P->don_cap = steal ? DON_CELLS : 0u;
    P->don_target = o && o->steal_target > 0 ? (uint32_t)std::min<int>(o->steal_target, (int)DON_CELLS) : DON_CELLS / 8;
    P->don_min_depth = o && o->steal_depth > 0 ? (uint32_t)o->steal_depth : 2u;
    uint32_t period = o && o->steal_period > 0 ? (uint32_t)o->steal_period : 64u;
    while (period & (period - 1)) period &= period - 1;  // a power of two (rounded down)
    P->don_period = period;
    // Any lane without work asks for donations (steal 0), or only whole idle warps (steal 2).
    // Measured on B200 with 256 x 3: the 4,096-cube batch with 5% hard positions 220 against 194
    // cubes/s, a lone superflip on d4t 3.1 against 5.8 s, uniform batches within 4%.
    P->don_eager = o && o->steal == 2 ? 0u : 1u;
    P->don_min_prev = o && o->steal_min_nodes != 0 ? (o->steal_min_nodes > 0 ? (unsigned long long)o->steal_min_nodes : 0ull)
                                                   : 10000000ull;
    // Head rotation at half the scan window (rotate 1) or at half the ring (-1, the batch default).
    P->head_limit = o && o->rotate > 0 ? std::max<unsigned long long>(P->spread / 2u, 32u) : 0ull;
    P->done_log = nullptr;
    P->done_log_cap = 0;
}

// Kernel variants (ccs_solve_opts.variant): 1 = phase-ordered control, frames in shared memory,
// 256 threads x 2 blocks per SM (registers for every value, no spills; the throughput kernel);
// 2 = the same with sibling lookahead (two probe chains per lane: lower latency when few cubes
// are searched, more probes); 3 = phase-ordered, 256 x 3 (80 registers); 4 = loop control,
// frames in registers, 256 x 2; 5 = loop control, frames in shared memory, 512 x 2;
// 6 = phase-ordered, 128 x 4 (4 warps per block); 7 = phase-ordered, 512 x 1 (16 warps per block);
// 8 = sibling lookahead, 256 x 3; 9 = phase-ordered, 256 x 4 (32 warps per SM, 64 registers);
// 10 = phase-ordered, 224 x 3 (21 warps, 96 registers); 11 = phase-ordered, 128 x 5 (20 warps, 96).
// 0 = automatic: 2 for fewer than 64 cubes, else 3 (and 3 for the server).  Measured on B200
// (d4t, 1,024 uniform cubes): 3 reaches 338 cubes/s (31.0 G probes/s) against 283 for 1 and 292
// for 2 -- its 80-register cap spills a little, to an L1 that the table sectors no longer
// occupy; a lone cube is faster on 2 (plain 1-cube p50 16.6 ms against 25.0 ms).
int resolve_variant(const ccs_solve_opts* o, int cubes) {
    int v = o ? o->variant : 0;
    if (v <= 0 || v > 11) v = cubes > 0 && cubes < 64 ? 2 : 3;
    return v;
}

int grid_for(ccs_handle* h, const ccs_solve_opts* o, int variant) {
    int bps = o && o->blocks_per_sm > 0 ? o->blocks_per_sm
                                         : (variant == 3 || variant == 8 || variant == 10 ? 3
                                          : variant == 6 || variant == 9 ? 4
                                          : variant == 11 ? 5
                                          : variant == 7 ? 1 : 2);
    return bps * h->sms;
}

// The search kernels of each kind are compiled in their own translation unit (search_launch.cuh,
// launch_*.cu), so the instantiations build in parallel.
template <int MODE, int NEC>
int launch_kind(ccs_handle* h, const SearchParams& P, int grid, cudaStream_t stream, int variant);

// variant: a resolved one (1..7).
int launch_kernel(ccs_handle* h, const SearchParams& P, int grid, cudaStream_t stream, int variant) {
    return dispatch_kind(h->kind, [&](auto M, auto N) {
        return launch_kind<decltype(M)::value, decltype(N)::value>(h, P, grid, stream, variant);
    });
}

// Host slot record for a new cube: frames, no iteration yet (the admitting lane computes the
// root bounds and publishes the first one).
void make_slot(const uint32_t state[5], uint32_t request, uint32_t table, Slot* s) {
    std::memset(s, 0, sizeof *s);
    cube_frames(state, s->frame);
    s->status = SLOT_ACTIVE;
    s->ticket = TICKET_IDLE;
    s->request = request;
    s->table = table;
}

void fill_result(const Slot& s, ccs_result* r) {
    std::memset(r, 0, sizeof *r);
    if (s.status == SLOT_SOLVED) {
        r->status = CCS_OK;
        r->length = (int32_t)s.sol_len;
        std::memcpy(r->moves, s.sol, std::min<uint32_t>(s.sol_len, 24));
    } else {
        r->status = CCS_E_CHECK;
        r->length = -1;
    }
    r->nodes = s.nodes;
    r->probes = s.probes;
    r->seconds = s.t_done > s.t_admit ? (double)(s.t_done - s.t_admit) * 1e-9 : 0.0;
    for (int i = 0; i < 24; ++i) r->iter_nodes[i] = s.iter_nodes[i];
}

}  // namespace ccs

extern "C" int ccs_solve(ccs_handle* h, const uint32_t* states, int n, const ccs_solve_opts* opts, ccs_result* results) {
    return ccs_solve_tables(h, states, nullptr, n, opts, results);
}

extern "C" int ccs_solve_tables(ccs_handle* h, const uint32_t* states, const uint8_t* table_ids, int n,
                                const ccs_solve_opts* opts, ccs_result* results) {
    if (!h || (n > 0 && (!states || !results))) return fail(CCS_E_ARG, "NULL argument");
    if (!h->d_table) return fail(CCS_E_STATE, "no table loaded");
    for (int i = 0; table_ids && i < n; ++i) {
        if (table_ids[i] > 1) return fail(CCS_E_ARG, "table id %d of cube %d is not 0 or 1", table_ids[i], i);
        if (table_ids[i] == 1 && !h->d_table2) return fail(CCS_E_STATE, "cube %d asks for a second table; none attached", i);
    }
    if (h->server) return fail(CCS_E_STATE, "the server owns this handle's search buffers");
    if (n <= 0) return CCS_OK;
    if ((uint32_t)n >= MAX_SLOTS) return fail(CCS_E_ARG, "%d cubes in one call: at most %u", n, MAX_SLOTS - 1);
    for (int i = 0; i < n; ++i)
        if (!is_legal(unpack(states + 5ull * i))) return fail(CCS_E_ARG, "cube %d is not a legal position", i);
    CCS_TRY(ensure_search_buffers(h, (uint32_t)n));
    std::vector<Slot> host(n);
    for (int i = 0; i < n; ++i) make_slot(states + 5ull * i, (uint32_t)i, table_ids ? table_ids[i] : 0u, &host[i]);
    std::vector<unsigned long long> admit(n);
    for (int i = 0; i < n; ++i) admit[i] = (unsigned long long)i;  // lap 0
    QueueState q;
    std::memset(&q, 0, sizeof q);
    q.admit_tail = (unsigned long long)n;
    SearchParams P;
    fill_params(h, opts, &P);
    P.n_slots = (uint32_t)n;
    if (n < 64) {
        // Few cubes per call (the plain drop-in's shape) have their own defaults: a push or pop
        // runs as soon as one lane waits for it, a probe pass repeats while 8 lanes probe, and
        // deeper prefixes start 200x sooner while at most 4 cubes are in flight.  Measured on
        // B200 (d4t, 256 x 2 with lookahead, 60 uniform cubes one per call): 55.0 cubes/s with the
        // batch defaults (8 / 16 / 50); 58.0 with the first, 60.2 with the first two, 61.4 with
        // the first and the third; a lone superflip 2.6 s either way.
        if (!(opts && opts->move_min > 0)) P.move_min = 1u;
        if (!(opts && opts->probe_min > 0)) P.probe_min = 8u;
        if (!(opts && opts->few_divisor > 0)) P.few_divisor = 200u;
    }
    cudaStream_t st = h->stream;
    CCS_CUDA_TRY(cudaMemcpyAsync(h->d_slots, host.data(), sizeof(Slot) * n, cudaMemcpyHostToDevice, st));
    CCS_CUDA_TRY(cudaMemsetAsync(h->d_ring, 0xFF, sizeof(unsigned long long) * (h->ring_cap + h->slot_cap), st));
    CCS_CUDA_TRY(cudaMemsetAsync(h->d_don, 0, sizeof(DonationCell) * DON_CELLS, st));
    CCS_CUDA_TRY(cudaMemcpyAsync(P.admit, admit.data(), 8ull * n, cudaMemcpyHostToDevice, st));
    CCS_CUDA_TRY(cudaMemcpyAsync(h->d_q, &q, sizeof q, cudaMemcpyHostToDevice, st));

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
        CCS_CUDA_TRY(cudaMemcpyAsync(&q, h->d_q, sizeof q, cudaMemcpyDeviceToHost, st));
        CCS_CUDA_TRY(cudaStreamSynchronize(st));
        float ms = 0;
        CCS_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        kernel_ms += ms;
        ++launches;
        if (q.active == 0 && q.admit_head >= q.admit_tail) break;
        // A launch ends only when every warp is out of work; if a relaunch found none either,
        // an iteration was lost.
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
    h->last_donated = q.donated;
    h->last_launches = launches;
    // host <-> device bytes of this call: cube slots, admission entries and the queue state in;
    // the queue state after every launch and the cube slots out
    h->last_h2d = (sizeof(Slot) + 8ull) * (uint64_t)n + sizeof(QueueState);
    h->last_d2h = sizeof(QueueState) * (uint64_t)launches + sizeof(Slot) * (uint64_t)n;
    CCS_CUDA_TRY(cudaMemcpyAsync(host.data(), h->d_slots, sizeof(Slot) * n, cudaMemcpyDeviceToHost, st));
    CCS_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) fill_result(host[i], &results[i]);
    if (q.error & ERR_BOUND) return fail(CCS_E_CHECK, "a search passed the largest possible bound");
    return CCS_OK;
}

extern "C" int ccs_last_solve_io_bytes(ccs_handle* h, uint64_t* h2d, uint64_t* d2h) {
    if (!h) return fail(CCS_E_ARG, "NULL handle");
    if (h2d) *h2d = h->last_h2d;
    if (d2h) *d2h = h->last_d2h;
    return CCS_OK;
}

extern "C" int ccs_last_solve_donations(ccs_handle* h, uint64_t* donated) {
    if (!h || !donated) return fail(CCS_E_ARG, "NULL argument");
    *donated = h->last_donated;
    return CCS_OK;
}

extern "C" int ccs_last_solve_stats(ccs_handle* h, double* kernel_ms, uint64_t* probes, int* launches) {
    if (!h) return fail(CCS_E_ARG, "NULL handle");
    if (kernel_ms) *kernel_ms = h->last_kernel_ms;
    if (probes) *probes = h->last_probes;
    if (launches) *launches = h->last_launches;
    return CCS_OK;
}
