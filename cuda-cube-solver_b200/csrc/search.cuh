// Device-side data of the IDA* search: cube slots, the work ring, launch parameters.
#pragma once

#include <cstdint>

namespace ccs {

constexpr uint32_t SLOT_FREE = 0, SLOT_ACTIVE = 1, SLOT_SOLVED = 2, SLOT_ERROR = 3;
constexpr unsigned long long TICKET_IDLE = 0x7FFFFFFFull;  // ticket of a slot with no iteration: exhausted
constexpr int MAX_PLEN = 6;
constexpr uint32_t RING_RETIRED = 0xFFFFFFFFu;  // ring entry whose iteration is fully handed out
// A ring entry's low word: slot generation << SLOT_BITS | slot.  A server slot gets a new
// generation each time it is reused, so an entry left from the slot's previous cube is told apart.
constexpr uint32_t SLOT_BITS = 20, SLOT_MASK = (1u << SLOT_BITS) - 1u, GEN_MASK = 0xFFFu;
constexpr uint32_t MAX_SLOTS = SLOT_MASK;       // slot ids below 2^20 - 1 (the all-ones id is RING_RETIRED's)
constexpr uint32_t QUEUED = 0x80000000u;        // Slot.queued = QUEUED | generation of the live entry
constexpr uint32_t MAX_BOUND = 22;   // every position is solvable in 20 half-turn moves

// One cube under search.  The ticket is the work counter of the current IDA* iteration
// ("epoch"): plen << 56 | bound << 48 | epoch << 32 | next item index; one atomicAdd hands out
// an item together with the bound and prefix length it belongs to.
struct alignas(16) Slot {
    uint32_t frame[30];              // root frames: g, R g R^-1, R^2 g R^-2, then their inverses
    uint32_t h0;                     // root lower bounds, 5 bits per frame
    uint32_t status;
    unsigned long long ticket;
    uint32_t open;                   // work units of the current epoch not yet finished: its items,
                                     // plus subtrees donated by lanes still holding a unit (so it
                                     // reaches 0 exactly when the epoch's last unit finishes)
    uint32_t found;                  // set by the first lane that finds a solution
    uint32_t sol_len;
    uint32_t request;                // caller's tag (server request id)
    uint8_t sol[24];
    unsigned long long nodes, probes;
    unsigned long long iter_nodes[24];  // nodes per bound
    unsigned long long t_admit, t_done; // device globaltimer, ns
    uint32_t table;                  // 0: the handle's table, 1: its second resident table
    uint32_t queued;                 // QUEUED | gen while the work ring holds a live entry for this cube
    uint32_t gen;                    // generation of the slot (server: incremented on every reuse)
    uint32_t pad2[1];
};

struct QueueState {
    unsigned long long head, tail;   // ring positions, monotonic
    uint32_t active;                 // cubes admitted and not finished
    uint32_t error;                  // error bits (ERR_*)
    unsigned long long probes;       // table probes done by all lanes
    unsigned long long steps;        // lane steps (diagnostic)
    unsigned long long finished;     // cubes finished (monotonic)
    unsigned long long admit_head;   // admission ring: cubes waiting for a first iteration
    unsigned long long admit_tail;
    uint32_t yield;                  // host asks lanes to stop fetching new items
    uint32_t pad;
    unsigned long long scan_pos;     // rotating start of the stranded-cube check
    // Work-stealing words, on a cache line of their own: idle lanes poll them, and on the line of
    // the counters above their reads would queue behind every lane's atomics.
    alignas(128) uint32_t starving;  // set by a lane that found no item and no donated subtree
    uint32_t don_count;              // donated subtrees waiting in the donation cells
    unsigned long long donated;      // subtrees donated (diagnostic)
    uint32_t pad2[28];
};

// A donated subtree: the unexplored children of one node of a running item (the node at depth g0
// on the donor's path), handed to an idle lane.  Cell state: 0 empty, 1 being written, 2 full,
// 3 being read.  Payload: w1 = h of the node (30 bits) | g0 << 32 | bound << 37 | todo << 42;
// w2 / w3 = the path to the node, 5 bits per move (moves 0..11, 12..23).
struct alignas(32) DonationCell {
    uint32_t state;
    uint32_t slot;
    unsigned long long w1, w2, w3;
};
constexpr uint32_t DON_EMPTY = 0, DON_WRITING = 1, DON_FULL = 2, DON_READING = 3;

constexpr uint32_t ERR_IDLE_LIMIT = 1u, ERR_BOUND = 2u, ERR_STACK = 4u;

struct SearchParams {
    Slot* slots;
    QueueState* q;
    unsigned long long* ring;        // entries: lap << 32 | slot
    uint32_t ring_cap;
    unsigned long long* admit;       // admission entries: lap << 32 | slot
    uint32_t admit_cap;
    uint32_t n_slots;
    const uint32_t* classidx;
    const uint32_t* table;           // solving table (block or base 3)
    const uint32_t* table2;          // second resident table of a compatible kind (or = table)
    const uint32_t* prefixes[MAX_PLEN + 1];  // canonical move sequences, 5 bits per move
    uint32_t n_prefix[MAX_PLEN + 1];
    uint32_t base_plen;              // prefix length of a cube's first iterations
    uint32_t max_plen;               // longest prefix length whose list is present (<= MAX_PLEN)
    unsigned long long deeper_at[2]; // an iteration of at least this many nodes -> one move longer
    unsigned long long shallow_at[2]; // an iteration of fewer nodes -> one move shorter (0: off)
    uint32_t shallow_min_active;     // ... applied only while at least this many cubes are active
    uint32_t few_max_active;         // with at most this many cubes in flight ...
    uint32_t few_divisor;            // ... the deeper thresholds are divided by this
    uint32_t idle_limit;             // idle polls before a warp leaves (kernel relaunched by the host)
    uint32_t spread;                 // lanes take items from up to this many queued iterations
    uint32_t move_min;               // phased kernel: lanes waiting before a MOVE pass runs
    uint32_t move_age;               // phased kernel: iterations a waiting lane may be deferred
    uint32_t probe_min;              // phased kernel: probe pass repeats while this many lanes probe
    DonationCell* don;               // donation cells (null: no work stealing)
    uint32_t don_cap;                // number of cells
    uint32_t don_target;             // donors stop once this many subtrees wait
    uint32_t don_min_depth;          // a donated node has at least this many moves to the bound beyond
                                     // its largest frame bound (its slack)
    uint32_t don_period;             // a lane with work checks for starving lanes every this many iterations
    uint32_t don_eager;              // 1: a lane without work asks for donations (0: a whole idle warp)
    unsigned long long don_min_prev; // donate for cubes whose previous iteration had >= this many nodes
    uint32_t persistent;             // server: an empty queue is not the end (lanes wait for new cubes)
    unsigned long long head_limit;   // queued positions (tail - head) past which a live head entry moves
                                     // to the tail (0: half the ring)
    unsigned long long* done_log;    // host-mapped completion log (server), may be null
    uint32_t done_log_cap;
};

}  // namespace ccs
