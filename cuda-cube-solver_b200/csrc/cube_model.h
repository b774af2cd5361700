// Host-side cube model for libccs: moves, the 16 U-D symmetries, corner classes, table kinds,
// and the constant tables the kernels read (DevTables).
//
// Mirrors the Python host model of this package (cubie.py, geometry.py, coords.py, kinds.py),
// which restates the reference's src/cuda_cube_solver/{cubie,geometry,coords,kinds}.py.  The
// numbering of corner classes, combinations, E-orders and E-content classes is kept identical to
// the reference because it fixes the byte layout of the table files.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ccs {

constexpr int N_MOVES = 18;
constexpr int N_UDSYM = 16;
constexpr uint32_t N_CCOMB = 70;
constexpr uint32_t N_CORNER_RAW = 2187u * 70u;  // 153,090
constexpr uint32_t N_CLASSES = 9930;
constexpr uint32_t N_SLICE = 495;
constexpr uint32_t BLOCK_ENTRIES = 124;  // 2-bit block format: entries per 32-byte sector
constexpr uint32_t B3_ENTRIES = 155;     // base-3 block format: entries per 32-byte sector
constexpr int MAX_DEPTH = 24;

struct Cubie {
    uint8_t cp[8], co[8], ep[12], eo[12];
};

Cubie identity();
Cubie compose(const Cubie& a, const Cubie& b);  // apply b after a
Cubie inverse(const Cubie& a);
const Cubie& move(int m);                      // the 18 HTM moves, U U2 U' R ... B'
void pack(const Cubie& c, uint32_t w[5]);      // corner byte cp|co<<3, edge byte ep|eo<<4
Cubie unpack(const uint32_t w[5]);
bool is_legal(const Cubie& c);

// Action of a symmetry on cubies (positions, labels, orientation).
struct SymAction {
    uint8_t cperm[8], cshift[8];
    bool reflect;
    uint8_t eperm[12], eflip[12];
};
const SymAction& ud_sym(int s);         // the 16 U-D symmetries, identity first (reference order)
const SymAction& axis_rotation();       // 120-degree turn about URF: R -> U -> F
Cubie conjugate(const SymAction& s, const Cubie& c);  // M c M^-1
int ud_sym_mul(int t, int s);           // index of M_t M_s
int frame_move(int k, int m);           // move m seen in axis frame k (0..2)

// Corner classes under the 16 U-D symmetries.
struct CornerClasses {
    std::vector<uint32_t> classidx;  // raw -> class << 4 | first symmetry reaching the representative
    std::vector<uint32_t> rep;       // class -> representative raw
    std::vector<uint16_t> stab;      // class -> mask of symmetries fixing the representative
};
const CornerClasses& corner_classes();
uint32_t corner_raw(const uint8_t corner_bytes[8]);

// Table kinds.  mode KIND_GEN: E content up to a relabelling group (EP 9 / EO 1 in the
// reference's kernel); mode KIND_304: EdgeKind(3, 4).
enum KindMode : int { KIND_GEN = 1, KIND_304 = 2 };

struct KindDesc {
    int mode = KIND_GEN;
    int nec = 1;                   // E-content classes (KIND_GEN)
    uint64_t n_edge = 0;           // edge coordinates per corner class
    uint64_t n_entries = 0;        // 9,930 * n_edge
    uint16_t gen_class[384] = {};  // content (E-order rank * 16 + E flips) -> class
    uint16_t gen_rep[2][384] = {}; // class -> content, by E-flip parity
};

// Group kinds from generator lists (perm[4], flips[4] each); throws std::runtime_error with the
// reference's message if the group is not normalised by the U-D symmetries.
KindDesc make_group_kind(const std::string& name, const std::vector<std::pair<std::vector<int>, std::vector<int>>>& gens);
KindDesc make_304_kind();
bool preset_kind(const std::string& name, KindDesc* out);  // "304", "s4", "d4f", "a4t", "d4t", "d4", "a4"

// Combination / permutation ranks (itertools order, as the reference).
const std::vector<uint16_t>& slice_rank();    // 4096 -> rank or 0xFFFF
const std::vector<uint16_t>& slice_unrank();  // 495
const std::vector<uint16_t>& ccomb_rank();    // 256
const std::vector<uint8_t>& ccomb_unrank();   // 70
const std::vector<uint8_t>& eorder_rank();    // 256 -> rank or 0xFF
const std::vector<uint8_t>& eorder_unrank();  // 24

// Reference CPU index of a packed state (used by the library's self-checks and tests).
uint64_t table_index_host(const KindDesc& k, const uint32_t w[5]);

}  // namespace ccs
