// The IDA* search kernel (persistent, continuous batching).
//
// Method (the reference's, kernels.cu:644-1801 and solver.py:254-320): IDA* over six frames of
// the cube -- g conjugated so each of its three axes becomes the U-D axis, and the inverses of
// those three -- with one lower bound per frame from the coset table; a child is pruned when
// g + 1 + bound > threshold; the coset axis rule excludes first moves on an axis whose inverse
// frame is tight, and prunes a child whose three forward (or three inverse) frames are all
// tight; an inverse frame on the move's own axis keeps its parent's value (same coset); frames
// are probed at the budget edge first, one below next, the rest last.
//
// Execution (this library's own): every lane runs its own depth-first search over one work item
// (a cube and a canonical move prefix).  Per warp iteration each lane performs exactly one table
// probe; control work (next child, push, pop, item fetch) runs between probes.  Work comes from
// a device ring of cube slots: the ticket of a slot hands out the prefix items of its current
// iteration, and the lane that finishes the last item of an iteration either records the
// solution or publishes the next iteration (bound + 1) and re-queues the slot, so a batch of
// cubes advances with no host round trip per bound.  Waits are bounded: a warp with nothing to
// do polls a limited number of times and then leaves; the host relaunches while cubes remain.
#pragma once

#include "cube_dev.cuh"
#include "search.cuh"

namespace ccs {

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t hget(uint32_t h, int k) { return (h >> (5 * k)) & 31u; }
__device__ __forceinline__ uint32_t hset(uint32_t h, int k, uint32_t v) {
    return (h & ~(31u << (5 * k))) | (v << (5 * k));
}
__device__ __forceinline__ uint32_t hrep(uint32_t v) { return v * 0x2108421u; }  // v in all six fields

// Axes (bit a: moves of faces a and a + 3) on which the next move may not lie: inverse frame
// 3 + a is tight, so no solution of exactly this length starts with a turn on axis a.
__device__ __forceinline__ uint32_t excluded_axes(uint32_t h, uint32_t budget) {
    uint32_t x = h ^ hrep(budget);
    return (uint32_t)(((x >> 15) & 31u) == 0u) | ((uint32_t)(((x >> 20) & 31u) == 0u) << 1) |
           ((uint32_t)(((x >> 25) & 31u) == 0u) << 2);
}

__device__ __forceinline__ uint32_t axis_move_mask(uint32_t axes) {
    return ((axes & 1u) ? 0x00E07u : 0u) | ((axes & 2u) ? 0x07038u : 0u) | ((axes & 4u) ? 0x381C0u : 0u);
}

// All three forward frames (or all three inverse frames) tight: no last (first) move possible.
__device__ __forceinline__ bool all_axes_tight(uint32_t c, uint32_t budget) {
    if (budget == 0u) return false;
    uint32_t x = c ^ hrep(budget);
    return (x & 0x7FFFu) == 0u || ((x >> 15) & 0x7FFFu) == 0u;
}

// Probe order masks: frames at the budget edge | one below << 6 | the rest << 12.
__device__ __forceinline__ uint32_t frame_order(uint32_t h, uint32_t edge) {
    uint32_t at = 0, below = 0;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        uint32_t v = hget(h, j);
        at |= (uint32_t)(v >= edge) << j;
        below |= (uint32_t)(v + 1u == edge) << j;
    }
    return at | (below << 6) | ((~(at | below) & 0x3Fu) << 12);
}

__device__ __forceinline__ int next_frame(uint32_t& rem) {
    if (!rem) return 6;
    int b = __ffs(rem) - 1;
    rem &= rem - 1;
    return b % 6;
}

__device__ __forceinline__ void frame_do(const DevTables& T, State& f, int k, int m) {
    if (k < 3) move_right(T, f, T.frame_move[k][m]);
    else move_left(T, f, T.inv_move[T.frame_move[k - 3][m]]);
}

__device__ __forceinline__ void frame_undo(const DevTables& T, State& f, int k, int m) {
    if (k < 3) move_right(T, f, T.inv_move[T.frame_move[k][m]]);
    else move_left(T, f, T.frame_move[k - 3][m]);
}

__device__ __forceinline__ uint64_t ticket_make(uint32_t plen, uint32_t bound, uint32_t epoch) {
    return ((uint64_t)plen << 56) | ((uint64_t)bound << 48) | ((uint64_t)(epoch & 0xFFFFu) << 32);
}

// Appends an entry (low word: generation << SLOT_BITS | slot) to the work ring.
__device__ __forceinline__ void enqueue_entry(const SearchParams& P, uint32_t low) {
    unsigned long long pos = atomicAdd(&P.q->tail, 1ull);
    unsigned long long lap = pos / P.ring_cap;
    atomicExch(&P.ring[pos % P.ring_cap], (lap << 32) | low);
}

// A cube has at most one live ring entry: it is queued only when it has none.  The flag holds
// the generation of the entry; the lane that retires that entry clears it and then re-checks the
// ticket, so an iteration published meanwhile is queued by one of the two.  An entry left from a
// reused slot's previous cube carries the old generation and clears nothing.
__device__ __forceinline__ void queue_slot(const SearchParams& P, uint32_t s) {
    const uint32_t gen = *(volatile uint32_t*)&P.slots[s].gen & GEN_MASK;
    if (atomicCAS(&P.slots[s].queued, 0u, QUEUED | gen) == 0u) enqueue_entry(P, (gen << SLOT_BITS) | s);
}

__device__ __forceinline__ bool ticket_open(const SearchParams& P, unsigned long long tk) {
    uint32_t i = (uint32_t)tk, pl = (uint32_t)(tk >> 56);
    return pl <= (uint32_t)MAX_PLEN && i < P.n_prefix[pl];
}

__device__ __forceinline__ void publish_epoch(const SearchParams& P, uint32_t s, uint32_t plen, uint32_t bound,
                                              uint32_t epoch) {
    Slot& sl = P.slots[s];
    sl.open = P.n_prefix[plen];
    __threadfence();
    atomicExch(&sl.ticket, ticket_make(plen, bound, epoch));
    __threadfence();
    queue_slot(P, s);
}

__device__ __forceinline__ void finish_slot(const SearchParams& P, uint32_t s, uint32_t status) {
    Slot& sl = P.slots[s];
    sl.t_done = globaltimer_ns();
    __threadfence();
    atomicExch(&sl.status, status);
    __threadfence();
    if (P.done_log) {
        unsigned long long k = atomicAdd(&P.q->finished, 1ull);
        volatile unsigned long long* log = P.done_log;
        log[k % P.done_log_cap] = ((unsigned long long)(k / P.done_log_cap + 1) << 32) | s;
        __threadfence_system();
    } else {
        atomicAdd(&P.q->finished, 1ull);
    }
    atomicSub(&P.q->active, 1u);
}

// Prefix length of the next iteration: base, plus one per "deeper" threshold the last iteration
// reached (a few huge subtrees would otherwise leave the GPU idle), minus one per "shallow"
// threshold it stayed under when many cubes are active (tiny items cost more to fetch than to
// search, and other cubes fill the lanes), at most the bound.  While at most P.few_max_active
// cubes are in flight the deeper thresholds are divided by P.few_divisor: a lone hard cube then
// gets the GPU's lanes in smaller items and its iterations end on shorter stragglers (with more
// cubes sharing the GPU, the extra items cost more than they balance).
__device__ __forceinline__ uint32_t next_plen(const SearchParams& P, unsigned long long last_nodes, uint32_t bound) {
    // cubes admitted and not finished (q->active also counts admissions being attempted, which
    // briefly overshoots when many lanes race for the admission ring)
    volatile QueueState* q = P.q;
    const unsigned long long fin = q->finished;  // read first: then fin <= admitted
    const unsigned long long in_flight = q->admit_head - fin;
    const bool many = in_flight >= P.shallow_min_active;  // enough cubes to keep lanes busy
    const bool few = in_flight <= P.few_max_active;       // one or two cubes own the GPU
    const unsigned long long d0 = few ? P.deeper_at[0] / P.few_divisor : P.deeper_at[0];
    const unsigned long long d1 = few ? P.deeper_at[1] / P.few_divisor : P.deeper_at[1];
    // signed: a base of 1 minus two shallow steps is -1, clamped to 1 (never a wrapped length)
    int pl = (int)P.base_plen + (int)(last_nodes >= d0) + (int)(last_nodes >= d1);
    if (many) pl -= (int)(last_nodes < P.shallow_at[0]) + (int)(last_nodes < P.shallow_at[1]);
    const int top = (int)P.max_plen;  // the longest prefix length with a list in this launch
    pl = pl < 1 ? 1 : (pl > top ? top : pl);
    return (uint32_t)pl < bound ? (uint32_t)pl : bound;
}

// A lane finished a work unit (an item or a donated subtree) of slot s's current epoch: true for
// the lane that finished its last one.
__device__ __forceinline__ bool finish_unit(const SearchParams& P, uint32_t s) {
    __threadfence();
    const bool last = atomicSub(&P.slots[s].open, 1u) == 1u;
    if (last) __threadfence();
    return last;
}

// Work stealing.  A lane whose item still has unexplored children at a shallow node of its path
// donates them when lanes starve: the node's depth, bounds, path and remaining children go into
// a free donation cell, the epoch's open count grows by one first (the donor still holds its own
// unit, so the count cannot reach zero meanwhile), and the donor skips those children.  An idle
// lane takes a cell, replays the path on the root frames and searches the children as a unit of
// its own, which it may split again.  Cells are claimed with compare-and-swap on their state and
// scanned a bounded number of times; nothing waits.
__device__ __forceinline__ bool post_donation(const SearchParams& P, uint32_t seed, uint32_t slot,
                                              unsigned long long w1, unsigned long long w2, unsigned long long w3) {
    for (uint32_t i = 0; i < 32u; ++i) {
        DonationCell& cell = P.don[(seed + i) % P.don_cap];
        if (*(volatile uint32_t*)&cell.state != DON_EMPTY) continue;
        if (atomicCAS(&cell.state, DON_EMPTY, DON_WRITING) != DON_EMPTY) continue;
        cell.slot = slot;
        cell.w1 = w1;
        cell.w2 = w2;
        cell.w3 = w3;
        __threadfence();
        atomicExch(&cell.state, DON_FULL);
        atomicAdd(&P.q->don_count, 1u);
        atomicAdd(&P.q->donated, 1ull);
        return true;
    }
    return false;
}

__device__ __forceinline__ bool take_donation(const SearchParams& P, uint32_t seed, uint32_t& slot,
                                              unsigned long long& w1, unsigned long long& w2,
                                              unsigned long long& w3) {
    if ((int)*(volatile uint32_t*)&P.q->don_count <= 0) return false;
    for (uint32_t i = 0; i < 64u; ++i) {
        DonationCell& cell = P.don[(seed + i) % P.don_cap];
        if (*(volatile uint32_t*)&cell.state != DON_FULL) continue;
        if (atomicCAS(&cell.state, DON_FULL, DON_READING) != DON_FULL) continue;
        __threadfence();
        slot = *(volatile uint32_t*)&cell.slot;
        w1 = *(volatile unsigned long long*)&cell.w1;
        w2 = *(volatile unsigned long long*)&cell.w2;
        w3 = *(volatile unsigned long long*)&cell.w3;
        __threadfence();
        atomicExch(&cell.state, DON_EMPTY);
        atomicSub(&P.q->don_count, 1u);
        return true;
    }
    return false;
}

enum FetchResult { FETCH_OK = 0, FETCH_EMPTY = 1, FETCH_FINISHED = 2, FETCH_ADMIT = 3 };

// A server launch has nothing left: no cube admitted and unfinished, none waiting for admission.
__device__ __forceinline__ bool server_idle(const SearchParams& P) {
    volatile QueueState* q = P.q;
    return q->active == 0u && q->admit_head >= q->admit_tail;
}

// Keeps the ring's head moving: retired entries are passed, and once the queued positions (tail -
// head) reach a limit a live entry at the head (a cube whose long iteration is still being handed
// out) is moved to the tail instead of holding every later position behind it.  Entries are plain
// slot references, so a moved one serves the same iteration from its new place.  Lanes start
// their scans within the first `spread` positions after the head, so with a limit of half of
// that (P.head_limit; the server's default) no queued cube falls out of every lane's reach behind
// one long-lived entry; with P.head_limit 0 the limit is half the ring.
static __device__ __noinline__ void advance_head(const SearchParams& P) {
    volatile QueueState* q = P.q;
    const unsigned long long limit = P.head_limit ? P.head_limit : P.ring_cap / 2u;
    for (int a = 0; a < 4; ++a) {
        unsigned long long h = q->head, t = q->tail;
        if (h >= t) return;
        unsigned long long* cell = P.ring + h % P.ring_cap;
        unsigned long long e = *(volatile unsigned long long*)cell;
        unsigned long long lap = e >> 32, want = h / P.ring_cap;
        if (lap < want || lap == 0xFFFFFFFFull) return;  // reserved by an enqueue, not yet written
        if (lap == want && (uint32_t)e != RING_RETIRED) {
            if (t - h < limit) return;  // within the limit: the live entry stays
            if (atomicCAS(cell, e, (e & 0xFFFFFFFF00000000ull) | RING_RETIRED) != e) return;
            enqueue_entry(P, (uint32_t)e);
        }
        atomicCAS((unsigned long long*)&P.q->head, h, h + 1);  // retired, moved or overwritten
    }
}

// Safety net run by an idle warp: queues any active cube whose current iteration still has items
// to hand out but which has no ring entry (none should exist).  Each call checks the next 256
// slots of a shared rotating window, so the check stays cheap however many slots there are.
static __device__ __noinline__ void requeue_stranded(const SearchParams& P) {
    const uint32_t n = P.n_slots < 256u ? P.n_slots : 256u;
    const uint32_t first = (uint32_t)(atomicAdd(&P.q->scan_pos, (unsigned long long)n) % P.n_slots);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t s = (first + i) % P.n_slots;
        const Slot& sl = P.slots[s];
        if (*(const volatile uint32_t*)&sl.status != SLOT_ACTIVE || *(const volatile uint32_t*)&sl.found ||
            *(const volatile uint32_t*)&sl.queued)
            continue;
        if (ticket_open(P, *(const volatile unsigned long long*)&sl.ticket)) queue_slot(P, s);
    }
}

// Next unit of work for a lane: a cube to admit (admission ring, first), or a prefix item of a
// queued iteration (work ring).  FETCH_FINISHED when nothing is queued, admitted or in flight.
__device__ __forceinline__ int fetch_item(const SearchParams& P, uint32_t seed, uint32_t& slot, uint32_t& idx,
                                          uint32_t& plen, uint32_t& bound, uint32_t& epoch) {
    volatile QueueState* q = P.q;
    for (int tries = 0; tries < 8; ++tries) {
        if (q->yield) return FETCH_FINISHED;  // the host is stopping this launch
        unsigned long long ah = q->admit_head;
        if (ah < q->admit_tail) {
            unsigned long long e = ((volatile unsigned long long*)P.admit)[ah % P.admit_cap];
            if ((e >> 32) != ah / P.admit_cap) return FETCH_EMPTY;  // reserved, not yet written
            atomicAdd(&P.q->active, 1u);  // counted before the entry leaves the ring
            if (atomicCAS((unsigned long long*)&P.q->admit_head, ah, ah + 1) == ah) {
                slot = (uint32_t)e;
                return FETCH_ADMIT;
            }
            atomicSub(&P.q->active, 1u);
            continue;
        }
        advance_head(P);
        unsigned long long h = q->head, t = q->tail;
        // Batches end when nothing is queued, admitted or in flight; a server's lanes keep
        // polling instead (a lane that took FETCH_FINISHED would stay idle for the rest of the
        // launch while new cubes arrive), and its warps leave after the idle limit.
        if (h >= t)
            return (!P.persistent && q->active == 0u && q->admit_head >= q->admit_tail) ? FETCH_FINISHED : FETCH_EMPTY;
        // Lanes start at a seeded position among the first `spread` queued iterations and scan
        // forward past handed-out entries, so the lanes spread over many cubes: each cube's items
        // are worked roughly in prefix order and a solution found early stops the rest of its
        // last iteration.
        unsigned long long win = t - h < P.spread ? t - h : P.spread;
        unsigned long long pos = h + (seed + (uint32_t)tries * 0x9E3779B1u) % win;
        for (int step = 0; step < 32; ++step) {
            unsigned long long* cell = P.ring + pos % P.ring_cap;
            unsigned long long e = *(volatile unsigned long long*)cell;
            if ((e >> 32) == pos / P.ring_cap) {  // written (unwritten or overwritten entries are skipped)
                const uint32_t low = (uint32_t)e;
                if (low != RING_RETIRED) {
                    const uint32_t s = low & SLOT_MASK;
                    unsigned long long tk = atomicAdd(&P.slots[s].ticket, 1ull);
                    uint32_t i = (uint32_t)tk, pl = (uint32_t)(tk >> 56);
                    if (pl <= (uint32_t)MAX_PLEN && i < P.n_prefix[pl]) {
                        slot = s;
                        idx = i;
                        plen = pl;
                        bound = (uint32_t)(tk >> 48) & 0xFFu;
                        epoch = (uint32_t)(tk >> 32) & 0xFFFFu;
                        return FETCH_OK;
                    }
                    // iteration handed out: retire the entry; if a new iteration was published
                    // meanwhile (its queue_slot saw this entry still live), queue it now
                    if (atomicCAS(cell, e, (e & 0xFFFFFFFF00000000ull) | RING_RETIRED) == e) {
                        const uint32_t flag = QUEUED | (low >> SLOT_BITS);
                        if (atomicCAS(&P.slots[s].queued, flag, 0u) == flag) {
                            __threadfence();
                            if (ticket_open(P, *(volatile unsigned long long*)&P.slots[s].ticket)) queue_slot(P, s);
                        }
                    }
                }
                if (pos == h) atomicCAS((unsigned long long*)&P.q->head, h, h + 1);
            }
            if (++pos >= t) pos = h;
        }
    }
    return FETCH_EMPTY;
}

template <int MODE, int NEC, int FMT>
__device__ __forceinline__ uint32_t probe_bound(const DevTables& T, const SearchParams& P, const State& s,
                                                bool second = false) {
    return probe_dev<MODE, NEC, FMT>(T, P.classidx, second ? P.table2 : P.table, s, second);
}

// Admission of a new cube: root bounds of its six frames, first threshold, first iteration.
template <int MODE, int NEC, int FMT>
__device__ void admit_slot(const DevTables& T, const SearchParams& P, uint32_t s) {
    Slot& sl = P.slots[s];
    State f0{sl.frame[0], sl.frame[1], sl.frame[2], sl.frame[3], sl.frame[4]};
    const bool second = sl.table != 0u;
    uint32_t h = 0, bound = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        State f{sl.frame[5 * k], sl.frame[5 * k + 1], sl.frame[5 * k + 2], sl.frame[5 * k + 3], sl.frame[5 * k + 4]};
        uint32_t v = probe_bound<MODE, NEC, FMT>(T, P, f, second);
        v = v > 31u ? 31u : v;
        h = hset(h, k, v);
        bound = v > bound ? v : bound;
    }
    atomicAdd(&sl.probes, 6ull);
    atomicAdd(&P.q->probes, 6ull);
    sl.h0 = h;
    sl.t_admit = globaltimer_ns();
    if (is_solved(f0)) {
        sl.sol_len = 0;
        sl.found = 1;
        finish_slot(P, s, SLOT_SOLVED);
        return;
    }
    if (bound == 0u) bound = 1u;  // not solved, so at least one move
    publish_epoch(P, s, next_plen(P, 0ull, bound), bound, 1u);
}

// The six frames of a lane's current node: in registers (FramesReg) or in shared memory, word-major
// with the lane index innermost so that every access of a warp is bank-conflict free (FramesSmem).
struct FramesReg {
    State f[6];
    __device__ __forceinline__ void init(uint32_t*, int) {}
    __device__ __forceinline__ State get(int k) const {
        State t = f[0];
#pragma unroll
        for (int j = 1; j < 6; ++j)
            if (k == j) t = f[j];
        return t;
    }
    __device__ __forceinline__ State first() const { return f[0]; }
    __device__ __forceinline__ void load(const uint32_t* src) {
#pragma unroll
        for (int j = 0; j < 6; ++j) f[j] = State{src[5 * j], src[5 * j + 1], src[5 * j + 2], src[5 * j + 3], src[5 * j + 4]};
    }
    __device__ __forceinline__ void step(const DevTables& T, int m) {
#pragma unroll
        for (int j = 0; j < 6; ++j) frame_do(T, f[j], j, m);
    }
    __device__ __forceinline__ void unstep(const DevTables& T, int m) {
#pragma unroll
        for (int j = 0; j < 6; ++j) frame_undo(T, f[j], j, m);
    }
};

template <int THREADS>
struct FramesSmem {
    uint32_t* w;  // word i of frame k at w[(5 k + i) * THREADS]
    __device__ __forceinline__ void init(uint32_t* base, int tid) { w = base + tid; }
    __device__ __forceinline__ State get(int k) const {
        const uint32_t* p = w + 5 * k * THREADS;
        return State{p[0], p[THREADS], p[2 * THREADS], p[3 * THREADS], p[4 * THREADS]};
    }
    __device__ __forceinline__ void put(int k, const State& s) {
        uint32_t* p = w + 5 * k * THREADS;
        p[0] = s.c0;
        p[THREADS] = s.c1;
        p[2 * THREADS] = s.e0;
        p[3 * THREADS] = s.e1;
        p[4 * THREADS] = s.e2;
    }
    __device__ __forceinline__ State first() const { return get(0); }
    __device__ __forceinline__ void load(const uint32_t* src) {
#pragma unroll
        for (int i = 0; i < 30; ++i) w[i * THREADS] = src[i];
    }
    __device__ __forceinline__ void step(const DevTables& T, int m) {
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            State t = get(j);
            frame_do(T, t, j, m);
            put(j, t);
        }
    }
    __device__ __forceinline__ void unstep(const DevTables& T, int m) {
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            State t = get(j);
            frame_undo(T, t, j, m);
            put(j, t);
        }
    }
};

template <bool SMEM, int THREADS>
struct FramesOf {
    using type = FramesReg;
};
template <int THREADS>
struct FramesOf<true, THREADS> {
    using type = FramesSmem<THREADS>;
};

// Dynamic shared memory of a launch: the frames, when they live there.
template <bool SMEM, int THREADS>
constexpr size_t search_dyn_smem() {
    return SMEM ? 30u * 4u * THREADS : 0u;
}

template <int MODE, int NEC, int FMT, int THREADS, bool SMEM, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) search_kernel(const DevTables* __restrict__ gT, SearchParams P) {
    __shared__ DevTables T;
    extern __shared__ uint32_t frame_smem[];
    stage_tables(T, gT);

    unsigned char path[MAX_DEPTH];
    uint32_t hstack[MAX_DEPTH];
    typename FramesOf<SMEM, THREADS>::type f;
    f.init(frame_smem, threadIdx.x);
    uint32_t h = 0, c = 0;        // packed bounds of the node and of the child under evaluation
    uint32_t slot = 0, idx = 0, plen = 0, bound = 0, epoch = 0, pseq = 0;
    int g = 0, last = -1, m = -1, k = 0;
    uint32_t todo = 0, ord = 0, rem = 0;
    unsigned long long nodes = 0, probes = 0;
    bool have_item = false, done = false, idle = false, second = false;
    uint32_t iter = 0, idle_polls = 0, backoff = 32;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lane_seed = (blockIdx.x * blockDim.x + threadIdx.x) * 0x9E3779B1u >> 7;

    for (;;) {
        bool eval = false;
        idle = false;
        // ---- control: until this lane has a child frame to probe (or nothing to do) ----
        while (!done) {
            if (m >= 0) {
                if (k < 6) {  // child m still has frames to probe
                    eval = true;
                    break;
                }
                if (k == 6 && !all_axes_tight(c, bound - (uint32_t)g - 1u)) {  // push the surviving child
                    f.step(T, m);
                    hstack[g] = h;
                    path[g] = (unsigned char)m;
                    h = c;
                    last = m;
                    ++g;
                    if ((uint32_t)g == bound) {
                        Slot& sl = P.slots[slot];
                        if (is_solved(f.first()) && atomicCAS(&sl.found, 0u, 1u) == 0u) {
                            sl.sol_len = (uint32_t)g;
                            for (int j = 0; j < g; ++j) sl.sol[j] = path[j];
                        }
                        todo = 0;
                    } else {
                        uint32_t allow = (uint32_t)g < plen ? 1u << ((pseq >> (5 * g)) & 31u) : T.amask[m + 1];
                        todo = allow & ~axis_move_mask(excluded_axes(h, bound - (uint32_t)g));
                        ord = frame_order(h, bound - (uint32_t)g);
                    }
                }
                m = -1;
                continue;
            }
            if (!have_item) {
                int r = fetch_item(P, lane_seed, slot, idx, plen, bound, epoch);
                if (r == FETCH_FINISHED) {
                    done = true;
                    break;
                }
                if (r == FETCH_EMPTY) {
                    idle = true;
                    break;
                }
                if (r == FETCH_ADMIT) {
                    admit_slot<MODE, NEC, FMT>(T, P, slot);
                    continue;
                }
                Slot& sl = P.slots[slot];
                if (*(volatile uint32_t*)&sl.found) {  // solved by another item: skip
                    if (finish_unit(P, slot)) finish_slot(P, slot, SLOT_SOLVED);
                    continue;
                }
f.load(sl.frame);
                h = sl.h0;
                pseq = plen ? __ldg(P.prefixes[plen] + idx) : 0u;
                g = 0;
                last = -1;
                nodes = 0;
                probes = 0;
                uint32_t allow = plen ? 1u << (pseq & 31u) : T.amask[0];
                todo = allow & ~axis_move_mask(excluded_axes(h, bound));
                ord = frame_order(h, bound);
                have_item = true;
                continue;
            }
            if ((++iter & 1023u) == 0u &&
                (*(volatile uint32_t*)&P.slots[slot].found || ((volatile QueueState*)P.q)->yield))
                todo = 0, g = 0;  // solved elsewhere, or the host is stopping: drop the rest of the item
            if (todo) {
                m = __ffs(todo) - 1;
                todo &= todo - 1;
                ++nodes;
                int inherit = 3 + (m / 3) % 3;  // inverse frame on the move's axis: same coset
                c = h;
                rem = ord & ~(0x41041u << inherit);
                k = next_frame(rem);
                eval = true;
                break;
            }
            // node exhausted (or the cube was solved elsewhere): pop, or finish the item
            if (g == 0) {
                Slot& sl = P.slots[slot];
                atomicAdd(&sl.nodes, nodes);
                atomicAdd(&sl.probes, probes);
                atomicAdd(&sl.iter_nodes[bound < 24u ? bound : 23u], nodes);
                atomicAdd(&P.q->probes, probes);
                if (finish_unit(P, slot)) {
                    if (*(volatile uint32_t*)&sl.found) {
                        finish_slot(P, slot, SLOT_SOLVED);
                    } else if (bound + 1u > MAX_BOUND) {
                        atomicOr(&P.q->error, ERR_BOUND);
                        finish_slot(P, slot, SLOT_ERROR);
                    } else {
                        unsigned long long last_nodes = *(volatile unsigned long long*)&sl.iter_nodes[bound];
                        publish_epoch(P, slot, next_plen(P, last_nodes, bound + 1u), bound + 1u, epoch + 1u);
                    }
                }
                have_item = false;
                continue;
            }
            --g;
            int pm = path[g];
            f.unstep(T, pm);
            h = hstack[g];
            last = g > 0 ? path[g - 1] : -1;
            todo = (uint32_t)g < plen ? 0u
                                      : T.amask[last + 1] & ~axis_move_mask(excluded_axes(h, bound - (uint32_t)g)) &
                                            ~((2u << pm) - 1u);
            ord = frame_order(h, bound - (uint32_t)g);
        }
        if (__all_sync(0xFFFFFFFFu, done)) break;
        // After the control phase every lane is probing, idle (no work queued) or done.
        if (__ballot_sync(0xFFFFFFFFu, eval) == 0u) {
            // No lane has a probe: the warp backs off; after too many empty polls in a row it
            // leaves (warp-uniform counter), and the host relaunches while cubes remain.
            if (++idle_polls > P.idle_limit) {
                // A batch launch leaves (the host relaunches while cubes remain); a server launch
                // leaves only when no cube is in flight, so every warp stays to serve new work.
                if (!P.persistent) {
                    if (lane == 0) atomicOr(&P.q->error, ERR_IDLE_LIMIT);
                    break;
                }
                if (__shfl_sync(0xFFFFFFFFu, (int)server_idle(P), 0)) break;
                idle_polls = 0;
            }
            if ((idle_polls & 1023u) == 64u && lane == 0) requeue_stranded(P);
            __nanosleep(backoff);
            backoff = backoff < 4096u ? backoff * 2u : 4096u;
            continue;
        }
        idle_polls = 0;
        backoff = 32;
        if (!eval) continue;

        // ---- one probe: frame k of child m ----
        State t = f.get(k);
        if (k < 3) move_right(T, t, T.frame_move[k][m]);
        else move_left(T, t, T.inv_move[T.frame_move[k - 3][m]]);
        uint32_t v = probe_bound<MODE, NEC, FMT>(T, P, t, second);
        ++probes;
        uint32_t parent = hget(h, k);
        if (k < 3 && parent) v = max(v, parent - 1u);  // a right move changes the coset distance by <= 1
        v = v > 31u ? 31u : v;
        c = hset(c, k, v);
        k = ((uint32_t)g + 1u + v > bound) ? 7 : next_frame(rem);
    }
}

}  // namespace ccs
