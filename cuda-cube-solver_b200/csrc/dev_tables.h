// Constant tables the kernels stage in shared memory (built on the host by dev_tables.cpp).
//
// Packed state (the reference's format, kernels.cu:1-6): corners in two 32-bit words (byte =
// cp | co << 3), edges in three (byte = ep | eo << 4), position i in byte i of the byte string.
#pragma once

#include <cstdint>

#include "cube_model.h"

namespace ccs {

struct alignas(16) DevTables {
    // Right multiplication s <- s * m: new byte at position i = old byte at the move's source
    // position, orientation added.  Edges: sources below 8 come from (e0, e1), the others from e2.
    uint32_t mv_csel[18][2];
    uint32_t mv_cadd[18][2];
    uint32_t mv_esel[18][3];
    uint32_t mv_esel2[18][3];
    uint32_t mv_emsk[18][3];
    uint32_t mv_eflp[18][3];
    // Left multiplication s <- m * s: every cubie c is renamed to the move's byte for c.
    uint32_t lf_c[18][2];
    uint32_t lf_e[18][3];
    // Conjugation of edges by U-D symmetry s: output word w = prmt of the source words
    // (U/D layers from (e0, e1), E layer from e2), source-position flip, cubie relabel bytes.
    uint32_t sy_psel[16][3];
    uint32_t sy_pflp[16][3];
    uint32_t sy_rel[16][3];
    // What the cubie relabel of a U-D symmetry does to the coordinate: E cubies stay E cubies
    // (labels permuted: sy_lab maps a compacted 2-bit label string to the rank of the relabelled
    // order, 0..23), U cubies all become U or all become D (sy_swap), and the flips of E positions
    // and of E cubies toggle together (sy_fx).
    uint8_t sy_lab[16][256];
    uint8_t sy_fx[16];
    uint8_t sy_swap[16];
    uint16_t slice_rank[4096];   // 12-bit E mask -> 0..494
    uint16_t slice_unrank[496];
    uint16_t genc[384];          // E content (order rank * 16 + E flips) -> class
    uint16_t genc2[384];         // the same for a second resident table of a compatible kind
    uint16_t gen_rep[2][384];    // class -> content (order rank * 16 + flips), by flip parity
    uint8_t cmp4[16][256];       // 2-bit fields of a byte selected by a 4-bit mask, compacted
    uint8_t flp[256];            // (E mask4 << 4 | flip mask4) -> E flips | non-E flips << 4
    uint8_t ump[256];            // (E mask4 << 4 | U mask4) -> U mask over the non-E positions
    uint8_t ccomb_rank[256];
    uint8_t ccomb_unrank[72];
    uint8_t eorder_unrank[24];
    uint8_t eorder_rank[256];
    uint8_t sym_mul[16][16];
    uint8_t inv_move[24];        // inverse of move m (padded)
    uint8_t frame_move[3][24];   // move m seen in axis frame k (padded)
    uint8_t amask_pad[8];
    uint32_t amask[20];          // canonical successors of last move (index last + 1), 18 bits
};

// Fills the tables for a kind (gen tables from KindDesc; unused for KIND_304); genc2 starts as a
// copy of genc.
void build_dev_tables(const KindDesc& kind, DevTables* out);

// The E-content class table of a kind, as genc / genc2 hold it.
void build_genc(const KindDesc& kind, uint16_t genc[384]);

}  // namespace ccs

static_assert(sizeof(ccs::DevTables) % 16 == 0, "DevTables is staged with 16-byte copies");
