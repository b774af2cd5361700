// The IDA* search kernel, phase-ordered form.
//
// Same method, queue and per-lane depth-first search as search_kernel (search_kernel.cuh), but
// the control between probes is a fixed sequence of predicated phases run once per warp
// iteration -- RESOLVE the evaluated child, MOVE (push or pop), FINISH the item, FETCH the next
// one, PICK the next child, PROBE one frame -- instead of a loop that each lane leaves at its own
// pace.  Push and pop are the same work (a move applied to all six frames; pop uses the inverse
// moves), so one MOVE pass serves every lane waiting for either, and it is deferred until enough
// lanes wait (P.move_min), a few iterations passed (P.move_age) or no lane could probe: the
// heaviest phase is then shared by many lanes instead of running for one.  Leaf survivors (child
// at depth == threshold) are checked for a solution without a push.  Frames live in shared memory
// (word-major, bank-conflict free), so the kernel fits 64 registers and 32 warps per SM.
#pragma once

#include "search_kernel.cuh"

namespace ccs {

template <int MODE, int NEC, int FMT, int THREADS, int MINB, bool LOOKAHEAD = false>
__global__ void __launch_bounds__(THREADS, MINB) search_kernel_phased(const DevTables* __restrict__ gT, SearchParams P) {
    __shared__ DevTables T;
    extern __shared__ uint32_t frame_smem[];
    stage_tables(T, gT);
    FramesSmem<THREADS> f;
    f.init(frame_smem, threadIdx.x);

    // Per level of the lane's path: the move taken, the node's bounds, and the children not yet
    // picked when it was left (a pop resumes exactly those: with LOOKAHEAD a sibling evaluated
    // ahead of a pushed child, pruned or stashed, is not picked again, and a donation empties the
    // entry of the level it gives away).
    unsigned char path[MAX_DEPTH];
    uint32_t hstack[MAX_DEPTH], tstack[MAX_DEPTH];
    uint32_t h = 0, c = 0, todo = 0, ord = 0, rem = 0;
    uint32_t slot = 0, idx = 0, plen = 0, bound = 0, epoch = 0, pseq = 0;
    int g = 0, m = -1, k = 0;
    uint32_t nodes = 0, probes = 0;
    bool have = false, done = false, second = false;
    uint32_t iter = 0, idle_polls = 0, backoff = 32, fetches = 0, fetch_wait = 0;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lane_seed = (blockIdx.x * blockDim.x + threadIdx.x) * 0x9E3779B1u >> 7;

    // Work stealing: gbase = depth of the lane's unit root (0 for an item, the donated node's depth
    // for a donated subtree).  With LOOKAHEAD a sibling stashed at a donated depth stays with the
    // donor (it was picked already, so it is not among the donated children).
    int gbase = 0;
    uint32_t don_tick = 0;
    int mv = 0;  // frame update this lane waits for: 0 none, 1 push child m, 2 pop one level
    // LOOKAHEAD: the next sibling of the child under evaluation, evaluated alongside it; when the
    // child is pushed, the sibling's partial evaluation waits in a per-level stash (bit g of
    // `stash`) and becomes the current child when the subtree pops back to level g.
    int m2 = -1, k2 = 7;
    uint32_t c2 = 0, rem2 = 0, stash = 0;
    uint32_t la_c[LOOKAHEAD ? MAX_DEPTH : 1], la_x[LOOKAHEAD ? MAX_DEPTH : 1];
    uint32_t move_age = 0;
    for (;;) {
        // RESOLVE the child under evaluation: drop a pruned one, test a leaf survivor for a
        // solution, and queue the push of an inner survivor.
        if (m >= 0 && k >= 6 && mv == 0) {
            if (k == 6 && !all_axes_tight(c, bound - (uint32_t)g - 1u)) {
                if ((uint32_t)g + 1u == bound) {
                    State t = f.get(0);
                    frame_do(T, t, 0, m);
                    Slot& sl = P.slots[slot];
                    if (is_solved(t) && atomicCAS(&sl.found, 0u, 1u) == 0u) {
                        sl.sol_len = (uint32_t)g + 1u;
                        for (int j = 0; j < g; ++j) sl.sol[j] = path[j];
                        sl.sol[g] = (uint8_t)m;
                    }
                } else {
                    mv = 1;
                }
            }
            if (mv == 0) m = -1;
            if (LOOKAHEAD && mv == 0 && m2 >= 0) {  // the child is done: its sibling takes over
                m = m2;
                c = c2;
                rem = rem2;
                k = k2;
                m2 = -1;
            }
        }
        // A node with no children left pops one level (a unit ends at its root depth).
        if (have && m < 0 && todo == 0u && g > gbase && mv == 0) mv = 2;
        // MOVE: push and pop both apply a move to all six frames (pop with the inverse moves), so
        // one pass serves every waiting lane; it runs once enough lanes wait, after a few
        // iterations, or when no lane could probe meanwhile.
        {
            const unsigned want = __ballot_sync(0xFFFFFFFFu, mv != 0);
            const unsigned ready = __ballot_sync(0xFFFFFFFFu, mv == 0 && ((m >= 0 && k < 6) || (have && todo != 0u)));
            if (want && ((uint32_t)__popc(want) >= P.move_min || ++move_age >= P.move_age || ready == 0u)) {
                move_age = 0;
                if (mv) {
                    const int mm = mv == 1 ? m : path[g - 1];
#pragma unroll
                    for (int j = 0; j < 6; ++j) {
                        State t = f.get(j);
                        if (j < 3) {
                            int r = T.frame_move[j][mm];
                            move_right(T, t, mv == 1 ? r : T.inv_move[r]);
                        } else {
                            int l = T.frame_move[j - 3][mm];
                            move_left(T, t, mv == 1 ? T.inv_move[l] : l);
                        }
                        f.put(j, t);
                    }
                    if (mv == 1) {
                        if (LOOKAHEAD && m2 >= 0 && k2 != 7) {  // (a pruned sibling is done)
                            la_c[g] = c2;
                            la_x[g] = rem2 | ((uint32_t)m2 << 18) | ((uint32_t)k2 << 23);
                            stash |= 1u << g;
                        }
                        m2 = -1;
                        hstack[g] = h;
                        tstack[g] = todo;
                        path[g] = (unsigned char)m;
                        h = c;
                        ++g;
                        uint32_t allow = (uint32_t)g < plen ? 1u << ((pseq >> (5 * g)) & 31u) : T.amask[m + 1];
                        todo = allow & ~axis_move_mask(excluded_axes(h, bound - (uint32_t)g));
                        ord = frame_order(h, bound - (uint32_t)g);
                        m = -1;
                    } else {
                        --g;
                        h = hstack[g];
                        todo = tstack[g];
                        if (todo) ord = frame_order(h, bound - (uint32_t)g);
                        if (LOOKAHEAD && ((stash >> g) & 1u)) {  // the stashed sibling resumes
                            stash &= ~(1u << g);
                            const uint32_t x = la_x[g];
                            c = la_c[g];
                            rem = x & 0x3FFFFu;
                            m = (int)((x >> 18) & 31u);
                            k = (int)((x >> 23) & 7u);
                        }
                    }
                    mv = 0;
                }
            }
        }
        // Solved elsewhere, or the host is stopping: drop the rest of the item.
        if (have && mv == 0 && (++iter & 255u) == 0u &&
            (*(volatile uint32_t*)&P.slots[slot].found || ((volatile QueueState*)P.q)->yield)) {
            todo = 0u;
            g = gbase;  // (the frames are reloaded with the next unit)
            m = -1;
            m2 = -1;
            stash = 0u;
        }
        // FINISH the unit; the lane finishing an iteration's last unit closes the iteration.
        if (have && mv == 0 && m < 0 && todo == 0u && g == gbase) {
            Slot& sl = P.slots[slot];
            atomicAdd(&sl.nodes, (unsigned long long)nodes);
            atomicAdd(&sl.probes, (unsigned long long)probes);
            atomicAdd(&sl.iter_nodes[bound < 24u ? bound : 23u], (unsigned long long)nodes);
            atomicAdd(&P.q->probes, (unsigned long long)probes);
            gbase = 0;
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
            have = false;
        }
        // FETCH the next item (or a cube to admit).
        if (!have && !done && fetch_wait) {
            --fetch_wait;  // the queue was empty: retry in a few iterations, not on every one
        } else if (!have && !done) {
            const uint32_t seed = lane_seed + (fetches++) * 0x2545F491u;
            int r = fetch_item(P, seed, slot, idx, plen, bound, epoch);
            unsigned long long w1 = 0, w2 = 0, w3 = 0;
            bool donated_unit = false;
            if (r == FETCH_EMPTY && P.don_cap) {
                donated_unit = take_donation(P, seed, slot, w1, w2, w3);
                if (donated_unit) r = FETCH_OK;
                else if (P.don_eager && !*(volatile uint32_t*)&P.q->starving)
                    *(volatile uint32_t*)&P.q->starving = 1u;  // eager: any lane without work asks
            }
            if (r == FETCH_EMPTY) fetch_wait = 16;
            if (r == FETCH_FINISHED) {
                done = true;
            } else if (r == FETCH_ADMIT) {
                admit_slot<MODE, NEC, FMT>(T, P, slot);
            } else if (r == FETCH_OK) {
                Slot& sl = P.slots[slot];
                if (*(volatile uint32_t*)&sl.found) {  // solved by another unit: count it done
                    if (finish_unit(P, slot)) finish_slot(P, slot, SLOT_SOLVED);
                } else if (donated_unit && (((w1 >> 32) & 31u) >= (uint32_t)MAX_DEPTH ||
                                                      ((w1 >> 37) & 31u) > MAX_BOUND)) {
                    atomicOr(&P.q->error, ERR_STACK);  // a malformed cell (never written by a donor)
                    if (finish_unit(P, slot)) finish_slot(P, slot, SLOT_ERROR);
                } else if (donated_unit) {
                    // a donated subtree: the node at depth g0 on the donor's path, its bounds and
                    // remaining children; the frames are the root's with the path replayed
                    const int g0 = (int)((w1 >> 32) & 31u);
                    bound = (uint32_t)((w1 >> 37) & 31u);
                    epoch = (uint32_t)(*(volatile unsigned long long*)&sl.ticket >> 32) & 0xFFFFu;
                    f.load(sl.frame);
                    for (int j = 0; j < g0; ++j) {
                        const int mj = (int)(((j < 12 ? w2 : w3) >> (5 * (j % 12))) & 31u);
                        path[j] = (unsigned char)mj;
                        f.step(T, mj);
                    }
                    second = sl.table != 0u;
                    h = (uint32_t)w1 & 0x3FFFFFFFu;
                    g = gbase = g0;
                    plen = 0;
                    pseq = 0;
                    nodes = 0;
                    probes = 0;
                    stash = 0u;
                    m2 = -1;
                    todo = (uint32_t)(w1 >> 42) & 0x3FFFFu;
                    ord = frame_order(h, bound - (uint32_t)g0);
                    have = true;
                } else {
                    f.load(sl.frame);
                    second = sl.table != 0u;
                    h = sl.h0;
                    pseq = plen ? __ldg(P.prefixes[plen] + idx) : 0u;
                    g = 0;
                    nodes = 0;
                    probes = 0;
                    stash = 0u;
                    m2 = -1;
                    uint32_t allow = plen ? 1u << (pseq & 31u) : T.amask[0];
                    todo = allow & ~axis_move_mask(excluded_axes(h, bound));
                    ord = frame_order(h, bound);
                    have = true;
                }
            }
        }
        // DONATE: while lanes starve, hand the remaining children of the shallowest node on this
        // lane's path that still has some (and enough slack to be worth a replay) to them -- for
        // a cube whose previous iteration reached P.don_min_prev nodes (its current one is big).
        if (P.don_cap && have && mv == 0 && (++don_tick & (P.don_period - 1u)) == 0u &&
            *(volatile uint32_t*)&P.q->starving &&
            (P.don_min_prev == 0ull || (bound > 0u && *(volatile unsigned long long*)&P.slots[slot].iter_nodes[
                                                         (bound - 1u) < 24u ? bound - 1u : 23u] >= P.don_min_prev))) {
            volatile QueueState* q = P.q;
            if ((int)q->don_count >= (int)P.don_target) {
                q->starving = 0u;
            } else {
                const int lo = gbase > (int)plen ? gbase : (int)plen;
                for (int l = lo; l <= g; ++l) {
                    if (bound < (uint32_t)l + P.don_min_depth) break;
                    const uint32_t rest = l == g ? todo : tstack[l];
                    if (!rest) continue;
                    const uint32_t hl = l == g ? h : hstack[l];
                    // slack: moves to the bound beyond the node's largest frame bound; a subtree
                    // grows about 13x per move of slack, so a tight node is not worth a replay
                    uint32_t hmax = 0;
#pragma unroll
                    for (int j = 0; j < 6; ++j) hmax = max(hmax, hget(hl, j));
                    if (bound < (uint32_t)l + hmax + P.don_min_depth) continue;
                    unsigned long long w2 = 0, w3 = 0;
                    for (int j = 0; j < l; ++j) {
                        if (j < 12) w2 |= (unsigned long long)path[j] << (5 * j);
                        else w3 |= (unsigned long long)path[j] << (5 * (j - 12));
                    }
                    const unsigned long long w1 = (unsigned long long)hl | ((unsigned long long)l << 32) |
                                                  ((unsigned long long)bound << 37) | ((unsigned long long)rest << 42);
                    atomicAdd(&P.slots[slot].open, 1u);  // before the post: the count never runs short
                    if (post_donation(P, lane_seed + don_tick, slot, w1, w2, w3)) {
                        if (l == g) todo = 0u;  // the donated children are no longer this lane's
                        else tstack[l] = 0u;
                    } else {
                        atomicSub(&P.slots[slot].open, 1u);  // (this lane's own unit keeps it above 0)
                    }
                    break;
                }
            }
        }
        // PICK the next child.
        if (have && mv == 0 && m < 0 && todo != 0u) {
            m = __ffs(todo) - 1;
            todo &= todo - 1;
            ++nodes;
            int inherit = 3 + (m / 3) % 3;  // inverse frame on the move's axis: same coset
            c = h;
            rem = ord & ~(0x41041u << inherit);
            k = next_frame(rem);
        }
        if (__all_sync(0xFFFFFFFFu, done)) break;
        const bool eval = mv == 0 && m >= 0 && k < 6;
        if (__ballot_sync(0xFFFFFFFFu, eval || have) == 0u) {
            // Nothing queued for this warp: ask lanes with work to donate subtrees (a whole idle
            // warp, not a lane between two items, is the signal), back off, and leave after too
            // many empty polls in a row.
            if (lane == 0 && P.don_cap && !*(volatile uint32_t*)&P.q->starving)
                *(volatile uint32_t*)&P.q->starving = 1u;
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
        // PROBE frame k of child m.  A lane whose child is pruned takes its next sibling at once
        // and the pass repeats while at least P.probe_min lanes have a probe; lanes that need the
        // control phases (a child that passed every frame, a node without children left) wait
        // for the pass to end.  Children are evaluated in the same order either way.
        bool ev = eval;
        for (;;) {
            if (ev && LOOKAHEAD) {
                // The child's next frame and the next sibling's next frame are probed together
                // (two independent load chains in flight).  Results are taken in DFS order: the
                // sibling becomes the current child when this one is pruned or resolved, and waits
                // in the stash while this one's subtree is searched.
                if (m2 >= 0 && k2 == 7) m2 = -1;  // the sibling was pruned: it is done
                if (m2 < 0 && todo != 0u) {
                    m2 = __ffs(todo) - 1;
                    todo &= todo - 1;
                    ++nodes;
                    c2 = h;
                    rem2 = ord & ~(0x41041u << (3 + (m2 / 3) % 3));
                    k2 = next_frame(rem2);
                }
                const bool two = m2 >= 0 && k2 < 6;
                const int kb = two ? k2 : k, mb = two ? m2 : m;
                State t = f.get(k), u = f.get(kb);
                frame_do(T, t, k, m);
                frame_do(T, u, kb, mb);
                const uint32_t* tab = second ? P.table2 : P.table;
                uint32_t v = probe_dev<MODE, NEC, FMT>(T, P.classidx, tab, t, second);
                uint32_t w = probe_dev<MODE, NEC, FMT>(T, P.classidx, tab, u, second);
                probes += two ? 2u : 1u;
                uint32_t parent = hget(h, k);
                if (k < 3 && parent) v = max(v, parent - 1u);
                v = v > 31u ? 31u : v;
                c = hset(c, k, v);
                k = ((uint32_t)g + 1u + v > bound) ? 7 : next_frame(rem);
                if (two) {
                    parent = hget(h, kb);
                    if (kb < 3 && parent) w = max(w, parent - 1u);
                    w = w > 31u ? 31u : w;
                    c2 = hset(c2, kb, w);
                    k2 = ((uint32_t)g + 1u + w > bound) ? 7 : next_frame(rem2);
                }
                if (k == 7 && m2 >= 0) {  // pruned: the sibling takes over
                    m = m2;
                    c = c2;
                    rem = rem2;
                    k = k2;
                    m2 = -1;
                }
            } else if (ev) {
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
            if (ev) {
                if (k == 7 && todo != 0u) {  // pruned: the next sibling (PICK)
                    m = __ffs(todo) - 1;
                    todo &= todo - 1;
                    ++nodes;
                    c = h;
                    rem = ord & ~(0x41041u << (3 + (m / 3) % 3));
                    k = next_frame(rem);
                }
            }
            ev = ev && k < 6;
            if ((uint32_t)__popc(__ballot_sync(0xFFFFFFFFu, ev)) < P.probe_min) break;
        }
    }
}

}  // namespace ccs
