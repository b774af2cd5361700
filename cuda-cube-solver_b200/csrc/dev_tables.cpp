// Builds DevTables from the host cube model.
#include "dev_tables.h"

#include <cstring>
#include <stdexcept>

namespace ccs {

namespace {
uint32_t selector(const int src[4]) {
    uint32_t s = 0;
    for (int j = 0; j < 4; ++j) s |= (uint32_t)(src[j] & 7) << (4 * j);
    return s;
}

// Canonical move order: no face twice in a row, opposite faces only in U-D, R-L, F-B order.
bool allowed_after(int last, int m) {
    if (last < 0) return true;
    int lf = last / 3, mf = m / 3;
    return mf != lf && !(lf >= 3 && mf == lf - 3);
}
}  // namespace

void build_genc(const KindDesc& kind, uint16_t genc[384]) {
    for (int c = 0; c < 384; ++c) genc[c] = kind.gen_class[c];
}

void build_dev_tables(const KindDesc& kind, DevTables* T) {
    std::memset(T, 0, sizeof(DevTables));
    for (int m = 0; m < 18; ++m) {
        const Cubie& mv = move(m);
        for (int w = 0; w < 2; ++w) {
            int src[4];
            for (int j = 0; j < 4; ++j) src[j] = mv.cp[4 * w + j];
            T->mv_csel[m][w] = selector(src);
            uint32_t add = 0;
            for (int j = 0; j < 4; ++j) add |= (uint32_t)mv.co[4 * w + j] << (3 + 8 * j);
            T->mv_cadd[m][w] = add;
        }
        for (int w = 0; w < 3; ++w) {
            int lo[4], hi[4];
            uint32_t msk = 0, flp = 0;
            for (int j = 0; j < 4; ++j) {
                int s = mv.ep[4 * w + j];
                lo[j] = s < 8 ? s : 0;
                hi[j] = s >= 8 ? s - 8 : 0;
                if (s >= 8) msk |= 0xFFu << (8 * j);
                flp |= (uint32_t)mv.eo[4 * w + j] << (4 + 8 * j);
            }
            T->mv_esel[m][w] = selector(lo);
            T->mv_esel2[m][w] = selector(hi);
            T->mv_emsk[m][w] = msk;
            T->mv_eflp[m][w] = flp;
        }
        for (int w = 0; w < 2; ++w) {
            uint32_t v = 0;
            for (int j = 0; j < 4; ++j) v |= (uint32_t)(mv.cp[4 * w + j] | (mv.co[4 * w + j] << 3)) << (8 * j);
            T->lf_c[m][w] = v;
        }
        for (int w = 0; w < 3; ++w) {
            uint32_t v = 0;
            for (int j = 0; j < 4; ++j) v |= (uint32_t)(mv.ep[4 * w + j] | (mv.eo[4 * w + j] << 4)) << (8 * j);
            T->lf_e[m][w] = v;
        }
    }
    for (int s = 0; s < 16; ++s) {
        const SymAction& a = ud_sym(s);
        int pinv[12];
        for (int p = 0; p < 12; ++p) pinv[a.eperm[p]] = p;
        for (int w = 0; w < 3; ++w) {
            int src[4];
            uint32_t pf = 0, rel = 0;
            for (int j = 0; j < 4; ++j) {
                int q = 4 * w + j, p = pinv[q];
                // U-D symmetries keep the E layer and map the U and D layers onto themselves.
                if ((q >= 8) != (p >= 8)) throw std::logic_error("U-D symmetry moves the E layer");
                src[j] = p >= 8 ? p - 8 : p;
                pf |= (uint32_t)a.eflip[p] << (4 + 8 * j);
                int c = 4 * w + j;  // relabel table: byte for cubie c
                rel |= (uint32_t)(a.eperm[c] | (a.eflip[c] << 4)) << (8 * j);
            }
            T->sy_psel[s][w] = selector(src);
            T->sy_pflp[s][w] = pf;
            T->sy_rel[s][w] = rel;
        }
        for (int t = 0; t < 16; ++t) T->sym_mul[t][s] = (uint8_t)ud_sym_mul(t, s);
        // The relabel-free edge coordinate relies on these properties of U-D symmetries.
        const int fx = a.eflip[8], swap = a.eperm[0] >= 4;
        for (int p = 0; p < 12; ++p) {
            if ((a.eperm[p] >= 8) != (p >= 8)) throw std::logic_error("U-D symmetry moves an E cubie out of the E layer");
            if (a.eflip[p] != (p >= 8 ? fx : 0)) throw std::logic_error("U-D symmetry flips unevenly");
            if (p < 8 && ((a.eperm[p] >= 4) != ((p >= 4) != (bool)swap))) throw std::logic_error("U-D symmetry splits a layer");
        }
        T->sy_fx[s] = (uint8_t)fx;
        T->sy_swap[s] = (uint8_t)swap;
        for (int v = 0; v < 256; ++v) {
            uint32_t out = 0;
            for (int j = 0; j < 4; ++j) out |= (uint32_t)(a.eperm[8 + ((v >> (2 * j)) & 3)] - 8) << (2 * j);
            const uint8_t r = eorder_rank()[out];
            T->sy_lab[s][v] = r == 0xFF ? 0 : r;  // (label strings that are no order never occur)
        }
    }
    for (int i = 0; i < 4096; ++i) T->slice_rank[i] = slice_rank()[i] == 0xFFFF ? 0 : slice_rank()[i];
    for (int i = 0; i < 495; ++i) T->slice_unrank[i] = slice_unrank()[i];
    for (int i = 0; i < 256; ++i) T->ccomb_rank[i] = (uint8_t)(ccomb_rank()[i] == 0xFFFF ? 0 : ccomb_rank()[i]);
    for (int i = 0; i < 70; ++i) T->ccomb_unrank[i] = ccomb_unrank()[i];
    for (int i = 0; i < 24; ++i) T->eorder_unrank[i] = eorder_unrank()[i];
    for (int i = 0; i < 256; ++i) T->eorder_rank[i] = eorder_rank()[i] == 0xFF ? 0 : eorder_rank()[i];
    if (kind.mode == KIND_GEN) {
        build_genc(kind, T->genc);
        std::memcpy(T->genc2, T->genc, sizeof(T->genc2));
        std::memcpy(T->gen_rep, kind.gen_rep, sizeof(T->gen_rep));
    }
    for (int m4 = 0; m4 < 16; ++m4)
        for (int v = 0; v < 256; ++v) {
            uint32_t out = 0, n = 0;
            for (int j = 0; j < 4; ++j)
                if ((m4 >> j) & 1) out |= ((v >> (2 * j)) & 3u) << (2 * n++);
            T->cmp4[m4][v] = (uint8_t)out;
        }
    for (int em = 0; em < 16; ++em)
        for (int x = 0; x < 16; ++x) {
            uint32_t ef = 0, nf = 0, ne = 0, nn = 0;
            for (int j = 0; j < 4; ++j) {
                if ((em >> j) & 1) ef |= ((x >> j) & 1u) << ne++;
                else nf |= ((x >> j) & 1u) << nn++;
            }
            T->flp[(em << 4) | x] = (uint8_t)(ef | (nf << 4));
            T->ump[(em << 4) | x] = (uint8_t)nf;
        }
    for (int m = 0; m < 18; ++m) T->inv_move[m] = (uint8_t)(3 * (m / 3) + 2 - m % 3);
    for (int k = 0; k < 3; ++k)
        for (int m = 0; m < 18; ++m) T->frame_move[k][m] = (uint8_t)frame_move(k, m);
    for (int last = -1; last < 18; ++last) {
        uint32_t mask = 0;
        for (int m = 0; m < 18; ++m)
            if (allowed_after(last, m)) mask |= 1u << m;
        T->amask[last + 1] = mask;
    }
}

}  // namespace ccs
