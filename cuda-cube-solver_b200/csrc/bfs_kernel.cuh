// GPU breadth-first search of a coset table, and the encoders of its solving files.
//
// What is computed is the reference's (table.py:82-129, kernels.cu:485-624,1839-1869): the exact
// distance of every entry from the solved coset, with forward passes (expand every entry of the
// current depth: unrank, 18 moves, claim each neighbour and its stabiliser images) while the
// frontier is small and backward passes (an unvisited entry whose neighbour sits at the current
// depth is one deeper) afterwards.  The files are pure functions of those distances: per 32-byte
// sector a minimum and 2-bit offsets, or the base-3 code with a per-block cut.
//
// The representation is this library's own: one byte of exact depth per entry (0xFF =
// unvisited), 30 GB for the 30.2-billion-entry tables, which B200's HBM holds next to the output.
// A claim is a single atomicAnd on the byte's word (0xFF & (d | ~0xFF) = d; visited bytes are
// never touched because they are tested first), backward passes write only their own bytes and
// need no atomics, and the block / base-3 encoders are streaming passes over the depth bytes.
#pragma once

#include "cube_dev.cuh"

namespace ccs {

struct BfsParams {
    uint8_t* depth;                  // n_entries bytes, padded to a multiple of 16
    uint64_t n_entries;
    uint64_t n_chunks;               // 16-entry chunks
    const uint32_t* classidx;
    const uint32_t* class_rep;
    const uint16_t* class_stab;
    unsigned long long* counter;     // [0] entries found in this pass, [1] random depth-byte reads,
                                     // [2] claim attempts (atomics), for the pass's roofline
};

__device__ __forceinline__ uint32_t claim_entry(uint8_t* depth, uint64_t idx, uint32_t d1) {
    if (((volatile uint8_t*)depth)[idx] != 0xFFu) return 0;
    uint32_t* w = reinterpret_cast<uint32_t*>(depth + (idx & ~3ull));
    uint32_t sh = (uint32_t)(idx & 3u) * 8u;
    uint32_t old = atomicAnd(w, ~(0xFFu << sh) | (d1 << sh));
    return ((old >> sh) & 0xFFu) == 0xFFu;
}

// Claim the coset of state n and all its images under the symmetries fixing its corner class
// representative (kernels.cu:507-528).
template <int MODE, int NEC>
__device__ __forceinline__ uint32_t claim_with_stabilizer(const DevTables& T, const BfsParams& P, const State& n,
                                                          uint32_t d1) {
    uint32_t packed = __ldg(P.classidx + corner_raw_dev(T, n));
    uint32_t cls = packed >> 4, sym = packed & 15u;
    uint32_t stab = __ldg(P.class_stab + cls);
    uint64_t base = (uint64_t)cls * KindTraits<MODE, NEC>::N_EDGE;
    uint32_t claimed = 0;
    while (stab) {
        uint32_t t = __ffs(stab) - 1;
        stab &= stab - 1;
        claimed += claim_entry(P.depth, base + edge_coord_sym<MODE, NEC>(T, n, T.sym_mul[t][sym]), d1);
    }
    return claimed;
}

__device__ __forceinline__ void add_count(unsigned long long* counter, unsigned long long local) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31u) == 0 && local) atomicAdd(counter, local);
}

// Claims that found the byte unvisited (the atomic's return tells) and attempts, counted apart.
__device__ __forceinline__ uint32_t claim_counted(uint8_t* depth, uint64_t idx, uint32_t d1, uint32_t& attempts) {
    if (((volatile uint8_t*)depth)[idx] != 0xFFu) return 0;
    ++attempts;
    uint32_t* w = reinterpret_cast<uint32_t*>(depth + (idx & ~3ull));
    uint32_t sh = (uint32_t)(idx & 3u) * 8u;
    uint32_t old = atomicAnd(w, ~(0xFFu << sh) | (d1 << sh));
    return ((old >> sh) & 0xFFu) == 0xFFu;
}

template <int MODE, int NEC>
__global__ void bfs_seed(const DevTables* __restrict__ gT, BfsParams P) {
    __shared__ DevTables T;
    stage_tables(T, gT);
    if (threadIdx.x) return;
    State s{0x03020100u, 0x07060504u, 0x03020100u, 0x07060504u, 0x0B0A0908u};
    atomicAdd(P.counter, (unsigned long long)claim_with_stabilizer<MODE, NEC>(T, P, s, 0u));
}

// Lists, in shared memory, the entries of a warp's 32 consecutive 16-entry chunks whose depth
// byte equals `match` (as offsets 0..511 from the group's first entry); returns how many.
__device__ __forceinline__ uint32_t list_group(const BfsParams& P, uint64_t gi, uint32_t lane, uint32_t match,
                                               uint16_t* list) {
    const uint64_t ch = gi * 32u + lane;
    uint32_t sel = 0;  // bit j: entry j of this lane's chunk matches
    if (ch < P.n_chunks) {
        const uint4 v = reinterpret_cast<const uint4*>(P.depth)[ch];
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t x = w[q] ^ (match * 0x01010101u);
            const uint32_t hit = ~(((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x | 0x7F7F7F7Fu);  // 0x80 where byte == match
            sel |= ((((hit >> 7) & 0x01010101u) * 0x01020408u) >> 24) << (4 * q);
        }
    }
    const uint32_t cnt = __popc(sel);
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    uint32_t pos = incl - cnt;
    for (uint32_t mm = sel; mm; mm &= mm - 1) list[pos++] = (uint16_t)(lane * 16u + (__ffs(mm) - 1));
    __syncwarp();
    return __shfl_sync(0xFFFFFFFFu, incl, 31);
}

// Forward pass: expand every entry at depth d.  A warp lists the depth-d entries of 512
// consecutive entries and its lanes take them in turn; an entry's 18 neighbours are claimed one
// face at a time (three class lookups, then three depth tests in flight), each with its
// stabiliser images.
template <int MODE, int NEC>
__global__ void __launch_bounds__(256) bfs_forward(const DevTables* __restrict__ gT, BfsParams P, uint32_t d) {
    __shared__ DevTables T;
    __shared__ uint16_t list[8][512];
    stage_tables(T, gT);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    unsigned long long local = 0;
    uint32_t reads = 0, attempts = 0;
    const uint8_t* depth = P.depth;
    const uint32_t d1 = d + 1u;
    const uint64_t n_groups = (P.n_chunks + 31u) / 32u;
    const uint64_t n_warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t gi = blockIdx.x * (uint64_t)(blockDim.x >> 5) + warp; gi < n_groups; gi += n_warps) {
        const uint32_t total = list_group(P, gi, lane, d, list[warp]);
        for (uint32_t it = lane; it < total; it += 32u) {
            const uint64_t idx = gi * 512u + list[warp][it];
            if (idx >= P.n_entries) continue;
            State s;
            unrank_dev<MODE, NEC>(T, P.class_rep, idx, s);
            for (int f = 0; f < 6; ++f) {
                State n[3];
                uint32_t packed[3], stab[3];
                uint64_t j[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    n[i] = s;
                    move_right(T, n[i], 3 * f + i);
                    packed[i] = __ldg(P.classidx + corner_raw_dev(T, n[i]));
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) stab[i] = __ldg(P.class_stab + (packed[i] >> 4));
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const uint32_t t = stab[i] ? __ffs(stab[i]) - 1 : 0u;
                    j[i] = (uint64_t)(packed[i] >> 4) * KindTraits<MODE, NEC>::N_EDGE +
                           edge_coord_sym<MODE, NEC>(T, n[i], T.sym_mul[t][packed[i] & 15u]);
                }
                uint32_t b[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) b[i] = depth[j[i]];  // a stale 0xFF is settled by the atomic
                reads += 3u;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    if (stab[i] && b[i] == 0xFFu) local += claim_counted(P.depth, j[i], d1, attempts);
                    uint32_t rest = stab[i] & (stab[i] - 1);  // the other stabiliser images
                    while (rest) {
                        const uint32_t t = __ffs(rest) - 1;
                        rest &= rest - 1;
                        ++reads;
                        local += claim_counted(P.depth,
                                               (uint64_t)(packed[i] >> 4) * KindTraits<MODE, NEC>::N_EDGE +
                                                   edge_coord_sym<MODE, NEC>(T, n[i], T.sym_mul[t][packed[i] & 15u]),
                                               d1, attempts);
                    }
                }
            }
        }
        __syncwarp();
    }
    add_count(P.counter, local);
    add_count(P.counter + 1, reads);
    add_count(P.counter + 2, attempts);
}

// Backward pass: an unvisited entry with a neighbour at depth d is at depth d + 1.  A warp takes
// 32 consecutive 16-entry chunks (512 entries), lists their unvisited entries in shared memory,
// and its lanes take the listed entries in turn, so the work is shared evenly however the
// unvisited entries fall.  An entry tries its 18 neighbours one face at a time (three turns:
// three independent table reads in flight) and stops at the first face with a neighbour at depth
// d.  Lanes write single bytes: an entry's byte is only ever written by the lane that took it,
// and readers only test for depth d, which no write of this pass produces or removes.
template <int MODE, int NEC>
__global__ void __launch_bounds__(256) bfs_backward(const DevTables* __restrict__ gT, BfsParams P, uint32_t d) {
    __shared__ DevTables T;
    __shared__ uint16_t list[8][512];
    stage_tables(T, gT);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    unsigned long long local = 0;
    uint32_t reads = 0;
    const uint8_t* depth = P.depth;
    const uint64_t n_groups = (P.n_chunks + 31u) / 32u;
    const uint64_t n_warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t gi = blockIdx.x * (uint64_t)(blockDim.x >> 5) + warp; gi < n_groups; gi += n_warps) {
        const uint32_t total = list_group(P, gi, lane, 0xFFu, list[warp]);
        for (uint32_t it = lane; it < total; it += 32u) {
            const uint64_t idx = gi * 512u + list[warp][it];
            if (idx >= P.n_entries) continue;
            State s;
            unrank_dev<MODE, NEC>(T, P.class_rep, idx, s);
            bool found = false;
            for (int f = 0; f < 6 && !found; ++f) {
                State n0 = s, n1 = s, n2 = s;
                move_right(T, n0, 3 * f);
                move_right(T, n1, 3 * f + 1);
                move_right(T, n2, 3 * f + 2);
                const uint64_t j0 = table_index_dev<MODE, NEC>(T, P.classidx, n0);
                const uint64_t j1 = table_index_dev<MODE, NEC>(T, P.classidx, n1);
                const uint64_t j2 = table_index_dev<MODE, NEC>(T, P.classidx, n2);
                const uint32_t b0 = depth[j0], b1 = depth[j1], b2 = depth[j2];
                reads += 3u;
                found = b0 == d || b1 == d || b2 == d;
            }
            if (found) {
                P.depth[idx] = (uint8_t)(d + 1u);
                ++local;
            }
        }
        __syncwarp();
    }
    add_count(P.counter, local);
    add_count(P.counter + 1, reads);
}

// Histogram of depth values (0..31, plus unvisited in bin 32).
__global__ void __launch_bounds__(256) bfs_histogram(const uint8_t* __restrict__ depth, uint64_t n_entries,
                                                     unsigned long long* __restrict__ hist) {
    __shared__ unsigned long long sh[33];
    if (threadIdx.x < 33) sh[threadIdx.x] = 0;
    __syncthreads();
    uint64_t n_chunks = (n_entries + 15) / 16;
    const uint4* chunks = reinterpret_cast<const uint4*>(depth);
    uint32_t local[33];
#pragma unroll
    for (int i = 0; i < 33; ++i) local[i] = 0;
    for (uint64_t ch = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; ch < n_chunks;
         ch += (uint64_t)gridDim.x * blockDim.x) {
        uint4 v = chunks[ch];
        uint32_t w[4] = {v.x, v.y, v.z, v.w};
        for (int q = 0; q < 16; ++q) {
            uint64_t idx = ch * 16u + q;
            if (idx >= n_entries) break;
            uint32_t b = (w[q >> 2] >> (8 * (q & 3))) & 0xFFu;
            local[b > 31u ? 32u : b] += 1u;
        }
    }
    for (int i = 0; i < 33; ++i)
        if (local[i]) atomicAdd(&sh[i], (unsigned long long)local[i]);
    __syncthreads();
    if (threadIdx.x < 33 && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

// 2-bit block file: per 124-entry block, u8 minimum then offsets min(depth - minimum, 3) at bit
// 8 + 2j; entries past the end keep offset 0 (kernels.cu:396-434, 485-503).  A CTA stages 256
// blocks (31,744 bytes = 1,984 aligned 16-byte chunks) in shared memory.
__global__ void __launch_bounds__(256) encode_block(const uint8_t* __restrict__ depth, uint64_t n_entries,
                                                    uint64_t n_blocks, uint32_t* __restrict__ out) {
    __shared__ uint4 tile[1984];
    const uint8_t* tb = reinterpret_cast<const uint8_t*>(tile);
    for (uint64_t b0 = (uint64_t)blockIdx.x * 256u; b0 < n_blocks; b0 += (uint64_t)gridDim.x * 256u) {
        const uint4* src = reinterpret_cast<const uint4*>(depth + b0 * 124u);
        uint64_t avail = (n_entries + 15) / 16 - b0 * 124u / 16;  // depth array is padded to 16
        for (int i = threadIdx.x; i < 1984; i += 256) tile[i] = (uint64_t)i < avail ? src[i] : make_uint4(~0u, ~0u, ~0u, ~0u);
        __syncthreads();
        uint64_t b = b0 + threadIdx.x;
        if (b < n_blocks) {
            uint64_t first = b * 124u;
            uint32_t n = (uint32_t)min((uint64_t)124u, n_entries - first);
            const uint8_t* v = tb + threadIdx.x * 124u;
            uint32_t mn = 255;
            for (uint32_t j = 0; j < n; ++j) mn = min(mn, (uint32_t)v[j]);
            uint32_t words[8] = {mn, 0, 0, 0, 0, 0, 0, 0};
            for (uint32_t j = 0; j < n; ++j) {
                uint32_t off = min((uint32_t)v[j] - mn, 3u);
                uint32_t pos = 8u + 2u * j;
                words[pos >> 5] |= off << (pos & 31u);
            }
            uint4* o = reinterpret_cast<uint4*>(out + b * 8u);
            o[0] = make_uint4(words[0], words[1], words[2], words[3]);
            o[1] = make_uint4(words[4], words[5], words[6], words[7]);
        }
        __syncthreads();
    }
}

// Base-3 file (kernels.cu:1839-1869).  The value of an entry is what the reference recovers from
// its 2-bit block and mod-3 tables: exact up to the 124-block minimum + 5, otherwise the
// smallest value >= minimum + 3 with the right residue.  Per 155-entry block: minimum m, cut
// c in 0..3 maximising the sum of the encoded bounds (lowest c on ties), header m | c << 6, then
// five base-3 digits per byte (least significant = first entry).  `value(x)` gives entry x's
// value; the two sources below are the exact-depth array and the mod-3 + block tables.
template <class Value>
__device__ __forceinline__ void encode_b3_block(uint64_t b, uint64_t n_entries, Value value, uint32_t* __restrict__ out) {
    uint64_t first = b * 155u;
    uint32_t n = (uint32_t)min((uint64_t)155u, n_entries - first);
    unsigned char v[155];
    uint32_t m = 255;
    for (uint32_t j = 0; j < n; ++j) {
        v[j] = (unsigned char)value(first + j);
        m = min(m, (uint32_t)v[j]);
    }
    uint32_t best = 0, best_score = 0;
    for (uint32_t c = 0; c < 4; ++c) {
        uint32_t score = 0;
        for (uint32_t j = 0; j < n; ++j) score += v[j] <= m + c ? m : (v[j] == m + c + 1 ? m + c + 1 : m + c + 2);
        if (score > best_score) best_score = score, best = c;
    }
    unsigned char bytes[32];
    bytes[0] = (unsigned char)(m | (best << 6));
    for (uint32_t q = 0; q < 31; ++q) {
        uint32_t x = 0;
        for (int k = 4; k >= 0; --k) {
            uint32_t j = q * 5u + (uint32_t)k, dg = 0;
            if (j < n) dg = v[j] <= m + best ? 0u : (v[j] == m + best + 1 ? 1u : 2u);
            x = x * 3u + dg;
        }
        bytes[1 + q] = (unsigned char)x;
    }
    uint32_t* o = out + b * 8u;
    for (int w = 0; w < 8; ++w)
        o[w] = bytes[4 * w] | (bytes[4 * w + 1] << 8) | (bytes[4 * w + 2] << 16) | ((uint32_t)bytes[4 * w + 3] << 24);
}

__global__ void __launch_bounds__(128) encode_b3(const uint8_t* __restrict__ depth, const uint32_t* __restrict__ blk,
                                                 uint64_t n_entries, uint64_t n_blocks, uint32_t* __restrict__ out) {
    uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (b >= n_blocks) return;
    encode_b3_block(b, n_entries, [&](uint64_t x) -> uint32_t {
        uint32_t dx = depth[x];
        uint32_t m124 = __ldg(blk + (x / 124u) * 8u) & 0xFFu;
        return dx <= m124 + 5u ? dx : m124 + 3u + (dx - m124 - 3u) % 3u;
    }, out);
}

// The same file from the reference's two tables (build_b3_table, table.py:52-79): a block offset
// below 3 gives the value; offset 3 (at least minimum + 3) takes the smallest value >= minimum + 3
// whose residue is the mod-3 table's -- the exact depth when it is at most minimum + 5.
__global__ void __launch_bounds__(128) encode_b3_mod3(const uint32_t* __restrict__ mod3, const uint32_t* __restrict__ blk,
                                                      uint64_t n_entries, uint64_t n_blocks, uint32_t* __restrict__ out) {
    uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (b >= n_blocks) return;
    encode_b3_block(b, n_entries, [&](uint64_t x) -> uint32_t {
        const uint64_t sec = x / 124u;
        const uint32_t j = (uint32_t)(x - sec * 124u), pos = 8u + 2u * j;
        const uint32_t m124 = __ldg(blk + sec * 8u) & 0xFFu;
        const uint32_t off = (__ldg(blk + sec * 8u + (pos >> 5)) >> (pos & 31u)) & 3u;
        if (off < 3u) return m124 + off;
        const uint32_t r = (__ldg(mod3 + (x >> 4)) >> (2u * (uint32_t)(x & 15u))) & 3u;
        const uint32_t lo = m124 + 3u;
        return lo + (r + 3u - lo % 3u) % 3u;
    }, out);
}

// Mod-3 file: per little-endian uint32 sixteen entries, two bits each, depth mod 3 (3 for an
// unvisited entry and past the end, as the reference's table starts all ones; table.py:94-95).
__global__ void __launch_bounds__(256) encode_mod3(const uint8_t* __restrict__ depth, uint64_t n_words,
                                                   uint32_t* __restrict__ out) {
    const uint4* chunks = reinterpret_cast<const uint4*>(depth);  // 16 depth bytes per output word
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < n_words; w += (uint64_t)gridDim.x * blockDim.x) {
        uint4 v = chunks[w];
        uint32_t in[4] = {v.x, v.y, v.z, v.w}, word = 0;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            uint32_t d = (in[q >> 2] >> (8 * (q & 3))) & 0xFFu;
            word |= (d == 0xFFu ? 3u : d % 3u) << (2 * q);
        }
        out[w] = word;
    }
}

// Base-3 digit of entry j of a sector: byte 1 + j / 5, place j % 5 (least significant first).
__device__ __forceinline__ uint32_t decode_digit_b3(const uint32_t w[8], uint32_t j) {
    const uint32_t q = 1u + j / 5u, k = j % 5u;
    const uint32_t byte = (w[q >> 2] >> (8u * (q & 3u))) & 0xFFu;
    const uint32_t pw = k == 0 ? 1u : k == 1 ? 3u : k == 2 ? 9u : k == 3 ? 27u : 81u;
    return (byte / pw) % 3u;
}

// Entries of a solving table per decoded value (bins[0 .. n_bins-1], the last also holding larger
// values).  Block sectors are counted with popcounts: offset k of the valid entries goes to bin
// minimum + k; base-3 sectors per digit (0 -> m, 1 -> m + cut + 1, 2 -> m + cut + 2).
template <int FMT>
__global__ void __launch_bounds__(256) table_histogram(const uint32_t* __restrict__ tab, uint64_t n_entries,
                                                       uint32_t n_bins, unsigned long long* __restrict__ bins) {
    __shared__ unsigned long long sh[64];
    for (uint32_t i = threadIdx.x; i < 64; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    constexpr uint32_t PER = SectorTraits<FMT>::PER;
    const uint64_t n_sec = (n_entries + PER - 1) / PER;
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sec; s += (uint64_t)gridDim.x * blockDim.x) {
        const uint4* p = reinterpret_cast<const uint4*>(tab + s * 8u);
        const uint4 a = p[0], c = p[1];
        const uint32_t w[8] = {a.x, a.y, a.z, a.w, c.x, c.y, c.z, c.w};
        const uint32_t n = (uint32_t)min((uint64_t)PER, n_entries - s * PER);
        uint32_t cnt[4] = {0, 0, 0, 0}, base[4];
        if (FMT == FMT_BLOCK) {
            // entry j's offset sits at bits 8 + 2j; word i holds entries [16i - 4, 16i + 12)
            for (int i = 0; i < 8; ++i) {
                const int j0 = 16 * i - 4;  // entry of the word's bit 0
                uint32_t valid = 0;
                for (int t = 0; t < 16; ++t) {
                    const int j = j0 + t;
                    if (j >= 0 && j < (int)n) valid |= 1u << (2 * t);
                }
                const uint32_t lo = w[i] & valid, hi = (w[i] >> 1) & valid;
                cnt[1] += __popc(lo & ~hi);
                cnt[2] += __popc(hi & ~lo);
                cnt[3] += __popc(lo & hi);
            }
            cnt[0] = n - cnt[1] - cnt[2] - cnt[3];
            const uint32_t m = w[0] & 0xFFu;
            for (int k = 0; k < 4; ++k) base[k] = m + k;
        } else {
            for (uint32_t j = 0; j < n; ++j) cnt[decode_digit_b3(w, j)] += 1;
            const uint32_t m = w[0] & 63u, cut = (w[0] >> 6) & 3u;
            base[0] = m, base[1] = m + cut + 1u, base[2] = m + cut + 2u, base[3] = 0;
        }
        for (int k = 0; k < 4; ++k)
            if (cnt[k]) atomicAdd(&sh[min(base[k], n_bins - 1u)], (unsigned long long)cnt[k]);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n_bins; i += blockDim.x)
        if (sh[i]) atomicAdd(&bins[i], sh[i]);
}

}  // namespace ccs
