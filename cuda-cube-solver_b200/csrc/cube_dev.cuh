// Device cube math for libccs: moves on packed states, the symmetry-reduced table index, table
// decoding.  All integer; written for sm_100a.
//
// Index semantics follow the reference's kernels.cu:134-215 and :275-279 (corner raw coordinate,
// class and symmetry from classidx, edge coordinate of the conjugated edges) and the block /
// base-3 decoders of kernels.cu:396-434.  The formulation is this library's own: a U-D symmetry
// keeps the E layer and maps the U and D layers onto themselves, so the position permutation of
// an edge word is a single byte permute and the cubie relabel reduces to a flip mask, a U/D swap
// flag and a label-string table; masks are gathered with multiplies; E flips and non-E flips come
// from one 256-entry table per word; the E-content class is read straight from the 8-bit label
// string.
#pragma once

#include <cstdint>

#include "dev_tables.h"

namespace ccs {

struct State {
    uint32_t c0, c1, e0, e1, e2;
};

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t s) { return __byte_perm(a, b, s); }

// Corner bytes cp | o << 3 with o in 0..4 after an addition: bring o back to 0..2.  A byte is
// >= 24 exactly when o >= 3; (byte + 8) then has bit 5 set and subtracting 0x20 - 0x08 = 0x18
// per such byte wraps it.
__device__ __forceinline__ uint32_t wrap_twist(uint32_t a) {
    uint32_t t = (a + 0x08080808u) & 0x20202020u;
    return a - t + (t >> 2);
}

// Bit b of every byte, gathered into 4 bits (byte 0 -> bit 0).
__device__ __forceinline__ uint32_t gather4(uint32_t v, int b) {
    return (((v >> b) & 0x01010101u) * 0x01020408u) >> 24;
}

// Low 2 bits of every byte, gathered into 8 bits (byte 0 -> bits 0-1).
__device__ __forceinline__ uint32_t labels8(uint32_t v) { return ((v & 0x03030303u) * 0x01041040u) >> 24; }

// Byte-wise values < 8 as a prmt selector (nibble j = byte j).
__device__ __forceinline__ uint32_t nib_sel(uint32_t v) { return prmt(v | (v >> 4), 0u, 0x4420u); }

// Corner words of s * m (the corner half of move_right).
__device__ __forceinline__ void corners_right(const DevTables& T, uint32_t& c0, uint32_t& c1, int m) {
    uint32_t a = prmt(c0, c1, T.mv_csel[m][0]) + T.mv_cadd[m][0];
    uint32_t b = prmt(c0, c1, T.mv_csel[m][1]) + T.mv_cadd[m][1];
    c0 = wrap_twist(a);
    c1 = wrap_twist(b);
}

// Corner words of m * s (the corner half of move_left).
__device__ __forceinline__ void corners_left(const DevTables& T, uint32_t& c0, uint32_t& c1, int m) {
    const uint32_t l0 = T.lf_c[m][0], l1 = T.lf_c[m][1];
    c0 = wrap_twist(prmt(l0, l1, nib_sel(c0 & 0x07070707u)) + (c0 & 0x18181818u));
    c1 = wrap_twist(prmt(l0, l1, nib_sel(c1 & 0x07070707u)) + (c1 & 0x18181818u));
}

__device__ __forceinline__ void move_right(const DevTables& T, State& s, int m) {
    corners_right(T, s.c0, s.c1, m);
    uint32_t o[3];
#pragma unroll
    for (int w = 0; w < 3; ++w) {
        uint32_t x = prmt(s.e0, s.e1, T.mv_esel[m][w]);
        uint32_t y = prmt(s.e2, s.e2, T.mv_esel2[m][w]);
        uint32_t k = T.mv_emsk[m][w];
        o[w] = ((x & ~k) | (y & k)) ^ T.mv_eflp[m][w];
    }
    s.e0 = o[0];
    s.e1 = o[1];
    s.e2 = o[2];
}

// s <- m * s: every cubie c (and its orientation) is renamed through the move.
__device__ __forceinline__ void move_left(const DevTables& T, State& s, int m) {
    corners_left(T, s.c0, s.c1, m);
    const uint32_t r0 = T.lf_e[m][0], r1 = T.lf_e[m][1], r2 = T.lf_e[m][2];
    uint32_t e[3] = {s.e0, s.e1, s.e2};
#pragma unroll
    for (int w = 0; w < 3; ++w) {
        uint32_t v = e[w];
        uint32_t sel = nib_sel(v & 0x07070707u);
        uint32_t hi = ((v >> 3) & 0x01010101u) * 0xFFu;  // cubies 8..11 rename through r2
        e[w] = ((prmt(r0, r1, sel) & ~hi) | (prmt(r2, r2, sel) & hi)) ^ (v & 0x10101010u);
    }
    s.e0 = e[0];
    s.e1 = e[1];
    s.e2 = e[2];
}

__device__ __forceinline__ uint32_t corner_raw_words(const DevTables& T, uint32_t c0, uint32_t c1) {
    uint32_t olo = (c0 >> 3) & 0x03030303u;
    uint32_t ohi = (c1 >> 3) & 0x00030303u;
    uint32_t twist = __dp4a(olo, 0x1B090301u, 0u) + 81u * __dp4a(ohi, 0x00090301u, 0u);
    uint32_t dmask = gather4(c0, 2) | (gather4(c1, 2) << 4);
    return twist * 70u + T.ccomb_rank[dmask];
}

__device__ __forceinline__ uint32_t corner_raw_dev(const DevTables& T, const State& s) {
    return corner_raw_words(T, s.c0, s.c1);
}

// Edge coordinate of M_sym g M_sym^-1, computed without conjugating the cubie labels: a U-D
// symmetry maps E cubies to E cubies and U cubies all to U or all to D, so after moving the bytes
// to their conjugated positions (one prmt per word) the E mask is read directly, the flips need
// one XOR (flip of E positions and of E cubies, T.sy_fx), the U mask at most a complement
// (T.sy_swap), and the E labels one 256-entry relabel of the compacted label string (T.sy_lab).
// MODE KIND_GEN: (slice * 256 + non-E flips) * NEC + class of the E content;
// KIND_304: (slice * 70 + U layout of the non-E positions) * 16 + E flips.
template <int MODE, int NEC>
__device__ __forceinline__ uint32_t edge_coord_sym(const DevTables& T, const State& s, int sym, bool second = false) {
    uint32_t p0 = prmt(s.e0, s.e1, T.sy_psel[sym][0]);
    uint32_t p1 = prmt(s.e0, s.e1, T.sy_psel[sym][1]);
    uint32_t p2 = prmt(s.e2, s.e2, T.sy_psel[sym][2]);
    uint32_t em0 = gather4(p0, 3), em1 = gather4(p1, 3), em2 = gather4(p2, 3);
    uint32_t emask = em0 | (em1 << 4) | (em2 << 8);
    uint32_t omask = gather4(p0, 4) | (gather4(p1, 4) << 4) | (gather4(p2, 4) << 8);
    omask ^= (0xF00u ^ emask) & (0u - (uint32_t)T.sy_fx[sym]);
    uint32_t n0 = __popc(em0), n1 = __popc(em1);
    uint32_t f0 = T.flp[(em0 << 4) | (omask & 15u)], f1 = T.flp[(em1 << 4) | ((omask >> 4) & 15u)],
             f2 = T.flp[(em2 << 4) | (omask >> 8)];
    uint32_t eflips = (f0 & 15u) | ((f1 & 15u) << n0) | ((f2 & 15u) << (n0 + n1));
    uint32_t slice = T.slice_rank[emask];
    if (MODE == KIND_304) {
        uint32_t umask = gather4(~(p0 | (p0 >> 1)), 2) | (gather4(~(p1 | (p1 >> 1)), 2) << 4) |
                         (gather4(~(p2 | (p2 >> 1)), 2) << 8);
        umask ^= 0xFFFu & (0u - (uint32_t)T.sy_swap[sym]);
        uint32_t u = T.ump[(em0 << 4) | (umask & 15u)] | (T.ump[(em1 << 4) | ((umask >> 4) & 15u)] << (4 - n0)) |
                     (T.ump[(em2 << 4) | (umask >> 8)] << (8 - n0 - n1));
        return (slice * 70u + T.ccomb_rank[u]) * 16u + eflips;
    } else {
        uint32_t nflips = (f0 >> 4) | ((f1 >> 4) << (4 - n0)) | ((f2 >> 4) << (8 - n0 - n1));
        uint32_t eord = T.cmp4[em0][labels8(p0)] | ((uint32_t)T.cmp4[em1][labels8(p1)] << (2 * n0)) |
                        ((uint32_t)T.cmp4[em2][labels8(p2)] << (2 * (n0 + n1)));
        const uint16_t* genc = second ? T.genc2 : T.genc;
        return (slice * 256u + nflips) * (uint32_t)NEC + genc[((uint32_t)T.sy_lab[sym][eord] << 4) | eflips];  // rank * 16 + flips
    }
}

template <int MODE, int NEC>
struct KindTraits {
    static constexpr uint64_t N_EDGE = MODE == KIND_304 ? 495ull * 70ull * 16ull : 495ull * 256ull * (uint64_t)NEC;
};

// Table formats.
enum Format : int { FMT_BLOCK = 0, FMT_B3 = 1 };

// second: index into the second resident table's kind (genc2).
template <int MODE, int NEC>
__device__ __forceinline__ uint64_t table_index_dev(const DevTables& T, const uint32_t* __restrict__ classidx,
                                                    const State& s, bool second = false) {
    uint32_t packed = __ldg(classidx + corner_raw_dev(T, s));
    return (uint64_t)(packed >> 4) * KindTraits<MODE, NEC>::N_EDGE + edge_coord_sym<MODE, NEC>(T, s, packed & 15u, second);
}



// The whole 32-byte sector of a probe in one 256-bit load: one sector request instead of two
// (the minimum and the offset word travel separately otherwise).  The table is read-only while
// searching, so the load may be scheduled freely.  Measured on B200 with random sectors of an
// 8 GB buffer (ncu): a plain ld.global.nc moves 129 DRAM bytes per 32-byte sector and 4.5 L2
// sectors per load; the .L2::64B size hint halves both (68 B, 2.5) and raises the random-sector
// rate by 8%; .L1::no_allocate keeps these never-reused sectors out of L1 (the corner classes and
// the lanes' stacks use it).  CCS_SECTOR_LOAD_FORM: 0 plain, 1 .L2::64B, 2 both (default).
#ifndef CCS_SECTOR_LOAD_FORM
#define CCS_SECTOR_LOAD_FORM 2
#endif
__device__ __forceinline__ void load_sector(const uint32_t* p, uint32_t w[8]) {
#ifdef CCS_HOST_EMULATION  // host build of this header for the CPU tests
    for (int i = 0; i < 8; ++i) w[i] = p[i];
#else
#if CCS_SECTOR_LOAD_FORM == 0
#define CCS_LD_SECTOR "ld.global.nc.v8.u32"
#elif CCS_SECTOR_LOAD_FORM == 1
#define CCS_LD_SECTOR "ld.global.nc.L2::64B.v8.u32"
#else
#define CCS_LD_SECTOR "ld.global.nc.L1::no_allocate.L2::64B.v8.u32"
#endif
    asm(CCS_LD_SECTOR " {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
        : "l"(p));
#undef CCS_LD_SECTOR
#endif
}

__device__ __forceinline__ uint32_t pick8(const uint32_t w[8], uint32_t i) {
    uint32_t r = w[0];
#pragma unroll
    for (uint32_t j = 1; j < 8; ++j)
        if (i == j) r = w[j];
    return r;
}

// Value of entry j of a loaded sector.  Block: a u8 minimum then 124 two-bit offsets (3 = at
// least minimum + 3) starting at bit 8.  Base 3: header m | cut << 6, then 155 digits, five per
// byte (digit 0 = at least m, 1 = m + cut + 1, 2 = at least m + cut + 2).
template <int FMT>
__device__ __forceinline__ uint32_t decode_sector(const uint32_t w[8], uint32_t j) {
    if (FMT == FMT_B3) {
        uint32_t q = 1u + j / 5u;
        uint32_t hdr = w[0] & 0xFFu, byte = (pick8(w, q >> 2) >> (8u * (q & 3u))) & 0xFFu;
        uint32_t k = j % 5u;
        uint32_t pw = k == 0 ? 1u : k == 1 ? 3u : k == 2 ? 9u : k == 3 ? 27u : 81u;
        uint32_t d = (byte / pw) % 3u;
        uint32_t m = hdr & 63u;
        return d == 0u ? m : m + (hdr >> 6) + d;
    } else {
        uint32_t pos = 8u + 2u * j;
        return (w[0] & 0xFFu) + ((pick8(w, pos >> 5) >> (pos & 31u)) & 3u);
    }
}

template <int FMT>
struct SectorTraits {
    static constexpr uint32_t PER = FMT == FMT_B3 ? 155u : 124u;  // entries per 32-byte sector
};

// Lower bound of entry idx.
template <int FMT>
__device__ __forceinline__ uint32_t lower_bound_dev(const uint32_t* __restrict__ tab, uint64_t idx) {
    constexpr uint32_t PER = SectorTraits<FMT>::PER;
    uint32_t w[8];
    uint64_t b = idx / PER;
    load_sector(tab + b * 8u, w);
    return decode_sector<FMT>(w, (uint32_t)(idx - b * PER));
}

// Lower bound of entry cls * NE + e (NE edge coordinates per corner class) in 32-bit arithmetic:
// cls * NE = cls * (NE / PER) * PER + cls * (NE % PER), and every term fits 32 bits for the
// kinds built here (at most 9,930 classes, 3,041,280 edge coordinates, 2^32 sectors).
template <int FMT, uint64_t NE>
__device__ __forceinline__ void split_sector(uint32_t cls, uint32_t e, uint32_t& sector, uint32_t& j) {
    constexpr uint32_t PER = SectorTraits<FMT>::PER;
    constexpr uint32_t Q = (uint32_t)(NE / PER), R = (uint32_t)(NE % PER);
    static_assert(NE / PER * 9930ull < (1ull << 32) && R * 9930ull + NE < (1ull << 32), "32-bit sector arithmetic");
    const uint32_t t = cls * R + e;
    const uint32_t tq = t / PER;
    sector = cls * Q + tq;
    j = t - tq * PER;
}

template <int FMT, uint64_t NE>
__device__ __forceinline__ uint32_t lower_bound_split(const uint32_t* __restrict__ tab, uint32_t cls, uint32_t e) {
    uint32_t sector, j, w[8];
    split_sector<FMT, NE>(cls, e, sector, j);
    load_sector(tab + (uint64_t)sector * 8u, w);
    return decode_sector<FMT>(w, j);
}

// One probe of the search: the lower bound of state s, the same value as
// lower_bound_dev(tab, table_index_dev(T, classidx, s, second)) with 32-bit sector arithmetic.
template <int MODE, int NEC, int FMT>
__device__ __forceinline__ uint32_t probe_dev(const DevTables& T, const uint32_t* __restrict__ classidx,
                                              const uint32_t* __restrict__ tab, const State& s, bool second = false) {
    uint32_t packed = __ldg(classidx + corner_raw_dev(T, s));
    return lower_bound_split<FMT, KindTraits<MODE, NEC>::N_EDGE>(tab, packed >> 4,
                                                                 edge_coord_sym<MODE, NEC>(T, s, packed & 15u, second));
}

__device__ __forceinline__ bool is_solved(const State& s) {
    return s.c0 == 0x03020100u && s.c1 == 0x07060504u && s.e0 == 0x03020100u && s.e1 == 0x07060504u &&
           s.e2 == 0x0B0A0908u;
}

// Representative state of entry idx (the BFS expands it): corners from the class
// representative's raw coordinate, edges from the edge coordinate.  Follows kernels.cu:294-379.
template <int MODE, int NEC>
__device__ __forceinline__ void unrank_dev(const DevTables& T, const uint32_t* __restrict__ class_rep, uint64_t idx,
                                           State& s) {
    constexpr uint64_t NE = KindTraits<MODE, NEC>::N_EDGE;
    uint32_t cls = (uint32_t)(idx / NE);
    uint32_t coord = (uint32_t)(idx - (uint64_t)cls * NE);
    uint32_t raw = __ldg(class_rep + cls);
    uint32_t twist = raw / 70u;
    uint32_t dmask = T.ccomb_unrank[raw - twist * 70u];
    uint32_t c[8];
    uint32_t osum = 0, nu = 0, nd = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        uint32_t o;
        if (i < 7) {
            o = twist % 3u;
            twist /= 3u;
            osum += o;
        } else {
            o = (3u - osum % 3u) % 3u;
        }
        uint32_t cp = (dmask >> i) & 1u ? 4u + nd++ : nu++;
        c[i] = cp | (o << 3);
    }
    s.c0 = c[0] | (c[1] << 8) | (c[2] << 16) | (c[3] << 24);
    s.c1 = c[4] | (c[5] << 8) | (c[6] << 16) | (c[7] << 24);
    uint32_t emask, eord, eflips, umask, nflips;
    if (MODE == KIND_304) {
        uint32_t ef = coord % 16u, rest = coord / 16u;
        uint32_t u = rest % 70u;
        emask = T.slice_unrank[rest / 70u];
        eord = 0xE4u;
        eflips = ef;
        umask = T.ccomb_unrank[u];
        nflips = 0;
    } else {
        uint32_t gc = coord % (uint32_t)NEC, grest = coord / (uint32_t)NEC;
        nflips = grest % 256u;
        emask = T.slice_unrank[grest / 256u];
        uint32_t content = T.gen_rep[__popc(nflips) & 1u][gc];
        eord = T.eorder_unrank[content >> 4];
        eflips = content & 15u;
        umask = 0x0Fu;
    }
    uint32_t e[3] = {0, 0, 0};
    uint32_t ne = 0, no = 0, nue = 0, nde = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        uint32_t b, flip;
        if ((emask >> i) & 1u) {
            b = 8u | ((eord >> (2 * ne)) & 3u);
            flip = (eflips >> ne) & 1u;
            ++ne;
        } else {
            b = (umask >> no) & 1u ? nue++ : 4u + nde++;
            flip = (nflips >> no) & 1u;
            ++no;
        }
        e[i >> 2] |= (b | (flip << 4)) << ((i & 3) * 8);
    }
    s.e0 = e[0];
    s.e1 = e[1];
    s.e2 = e[2];
}

// Copy the constant tables into shared memory (whole block).
#ifndef CCS_HOST_EMULATION
__device__ __forceinline__ void stage_tables(DevTables& dst, const DevTables* __restrict__ src) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(DevTables) / 16); i += blockDim.x) d[i] = s[i];
    __syncthreads();
}
#endif

}  // namespace ccs
