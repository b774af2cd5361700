/* CPU oracle for the optimal-solve path.  TEST INFRASTRUCTURE ONLY: tests/, the smoke check and
 * bench.py's CPU baseline call it as the checker or as the CPU reference arm; the product path
 * (libccs) never links or calls it.
 *
 * A plain-C, cubie-level restatement of the reference's algorithms:
 *   - table index and unrank          kernels.cu:134-215, 275-279, 294-379 (EP 9 / EO 1 group
 *                                     kinds, kinds.py:56-96) and EdgeKind(3, 4) = "304"
 *   - BFS (forward / backward passes,  table.py:82-129, kernels.cu:485-611 (the same depths; one
 *     claims with stabiliser images)   byte of exact depth per entry instead of the mod-3 table)
 *   - 2-bit block and base-3 encoding kernels.cu:396-434, 485-503, 1839-1869
 *   - IDA* with six frames, axis rule,  kernels.cu:756-805, 1398-1427, 1507-1783, solver.py:254-320
 *     all-axes-tight prune, inherited
 *     inverse frame, frame order
 * Constant tables (moves, symmetry actions, corner classes, E-content classes) are passed in by
 * the caller from the package's Python host model, which is itself pinned to the reference by
 * tests/golden fixtures, so this file shares no code with libccs.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
    uint8_t cp[8], co[8], ep[12], eo[12];
} cube;

static uint8_t MV_CP[18][8], MV_CO[18][8], MV_EP[18][12], MV_EO[18][12];
static uint8_t SY_EPERM[16][12], SY_EFLIP[16][12], SY_MUL[16][16];
static uint8_t FRAME_MOVE[3][18];
static const uint32_t* CLASSIDX;
static const uint32_t* CLASS_REP;
static const uint16_t* CLASS_STAB;
static uint16_t SLICE_RANK[4096], SLICE_UNRANK[495], CCOMB_RANK[256];
static uint8_t CCOMB_UNRANK[70], EORDER_RANK[256], EORDER_UNRANK[24];

static int K_MODE = 1; /* 1 = group kind (E content up to a group), 2 = EdgeKind(3, 4) */
static uint32_t K_NEC = 1;
static uint64_t K_NEDGE = 0;
static uint16_t GEN_CLASS[384], GEN_REP[2][384];

/* ---- setup ------------------------------------------------------------------------------ */

static void combination_tables(int bits, uint16_t* rank, uint16_t* unrank) {
    /* itertools.combinations(range(bits), 4): lexicographic order of the sorted positions */
    int n = 0;
    for (int a = 0; a < bits; ++a)
        for (int b = a + 1; b < bits; ++b)
            for (int c = b + 1; c < bits; ++c)
                for (int d = c + 1; d < bits; ++d) {
                    uint32_t mask = (1u << a) | (1u << b) | (1u << c) | (1u << d);
                    rank[mask] = (uint16_t)n;
                    unrank[n++] = (uint16_t)mask;
                }
}

int orc_init(const uint8_t* mv_cp, const uint8_t* mv_co, const uint8_t* mv_ep, const uint8_t* mv_eo,
             const uint8_t* sy_eperm, const uint8_t* sy_eflip, const uint8_t* sy_mul, const uint8_t* frame_move,
             const uint32_t* classidx, const uint32_t* class_rep, const uint16_t* class_stab) {
    memcpy(MV_CP, mv_cp, sizeof MV_CP);
    memcpy(MV_CO, mv_co, sizeof MV_CO);
    memcpy(MV_EP, mv_ep, sizeof MV_EP);
    memcpy(MV_EO, mv_eo, sizeof MV_EO);
    memcpy(SY_EPERM, sy_eperm, sizeof SY_EPERM);
    memcpy(SY_EFLIP, sy_eflip, sizeof SY_EFLIP);
    memcpy(SY_MUL, sy_mul, sizeof SY_MUL);
    memcpy(FRAME_MOVE, frame_move, sizeof FRAME_MOVE);
    CLASSIDX = classidx;
    CLASS_REP = class_rep;
    CLASS_STAB = class_stab;
    uint16_t cun[70];
    memset(SLICE_RANK, 0, sizeof SLICE_RANK);
    memset(CCOMB_RANK, 0, sizeof CCOMB_RANK);
    combination_tables(12, SLICE_RANK, SLICE_UNRANK);
    combination_tables(8, CCOMB_RANK, cun);
    for (int i = 0; i < 70; ++i) CCOMB_UNRANK[i] = (uint8_t)cun[i];
    /* itertools.permutations(range(4)); key = labels packed 2 bits each, first in the low bits */
    int n = 0;
    memset(EORDER_RANK, 0xFF, sizeof EORDER_RANK);
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b)
            for (int c = 0; c < 4; ++c)
                for (int d = 0; d < 4; ++d) {
                    if (a == b || a == c || a == d || b == c || b == d || c == d) continue;
                    uint32_t key = a | (b << 2) | (c << 4) | (d << 6);
                    EORDER_RANK[key] = (uint8_t)n;
                    EORDER_UNRANK[n++] = (uint8_t)key;
                }
    return 0;
}

/* mode 1: group kind with nec classes and its gen tables; mode 2: "304". */
int orc_set_kind(int mode, int nec, const uint16_t* gen_class, const uint16_t* gen_rep) {
    K_MODE = mode;
    K_NEC = (uint32_t)nec;
    if (mode == 2) {
        K_NEDGE = 495ull * 70ull * 16ull;
    } else {
        K_NEDGE = 495ull * 256ull * (uint64_t)nec;
        memcpy(GEN_CLASS, gen_class, sizeof GEN_CLASS);
        memcpy(GEN_REP, gen_rep, sizeof GEN_REP);
    }
    return 0;
}

uint64_t orc_n_entries(void) { return 9930ull * K_NEDGE; }

/* ---- cube model ------------------------------------------------------------------------- */

static void from_words(const uint32_t w[5], cube* c) {
    for (int i = 0; i < 20; ++i) {
        uint8_t b = (uint8_t)(w[i >> 2] >> (8 * (i & 3)));
        if (i < 8) c->cp[i] = b & 7, c->co[i] = b >> 3;
        else c->ep[i - 8] = b & 15, c->eo[i - 8] = b >> 4;
    }
}

static void to_words(const cube* c, uint32_t w[5]) {
    uint8_t b[20];
    for (int i = 0; i < 8; ++i) b[i] = (uint8_t)(c->cp[i] | (c->co[i] << 3));
    for (int i = 0; i < 12; ++i) b[8 + i] = (uint8_t)(c->ep[i] | (c->eo[i] << 4));
    for (int j = 0; j < 5; ++j) w[j] = b[4 * j] | (b[4 * j + 1] << 8) | (b[4 * j + 2] << 16) | ((uint32_t)b[4 * j + 3] << 24);
}

/* s <- s * m (apply move m after s) */
static void move_right(cube* s, int m) {
    cube r;
    for (int i = 0; i < 8; ++i) {
        int j = MV_CP[m][i];
        r.cp[i] = s->cp[j];
        r.co[i] = (uint8_t)((s->co[j] + MV_CO[m][i]) % 3);
    }
    for (int i = 0; i < 12; ++i) {
        int j = MV_EP[m][i];
        r.ep[i] = s->ep[j];
        r.eo[i] = (uint8_t)(s->eo[j] ^ MV_EO[m][i]);
    }
    *s = r;
}

/* s <- m * s (rename every cubie through the move) */
static void move_left(cube* s, int m) {
    for (int i = 0; i < 8; ++i) {
        int c = s->cp[i];
        s->co[i] = (uint8_t)((MV_CO[m][c] + s->co[i]) % 3);
        s->cp[i] = MV_CP[m][c];
    }
    for (int i = 0; i < 12; ++i) {
        int c = s->ep[i];
        s->eo[i] = (uint8_t)(MV_EO[m][c] ^ s->eo[i]);
        s->ep[i] = MV_EP[m][c];
    }
}

static int inverse_move(int m) { return 3 * (m / 3) + 2 - m % 3; }

static int is_solved(const cube* c) {
    for (int i = 0; i < 8; ++i)
        if (c->cp[i] != i || c->co[i]) return 0;
    for (int i = 0; i < 12; ++i)
        if (c->ep[i] != i || c->eo[i]) return 0;
    return 1;
}

static uint32_t corner_raw(const cube* c) {
    uint32_t twist = 0, w = 1, dmask = 0;
    for (int i = 0; i < 7; ++i, w *= 3) twist += c->co[i] * w;
    for (int i = 0; i < 8; ++i) dmask |= (uint32_t)(c->cp[i] >= 4) << i;
    return twist * 70u + CCOMB_RANK[dmask];
}

/* Edge coordinate of the edges conjugated by U-D symmetry sym. */
static uint64_t edge_coord(const cube* c, int sym) {
    uint8_t ep[12], eo[12];
    for (int p = 0; p < 12; ++p) {
        int q = SY_EPERM[sym][p], cub = c->ep[p];
        ep[q] = SY_EPERM[sym][cub];
        eo[q] = (uint8_t)(c->eo[p] ^ SY_EFLIP[sym][p] ^ SY_EFLIP[sym][cub]);
    }
    uint32_t emask = 0, eord = 0, eflips = 0, nflips = 0, umask = 0, ne = 0, nn = 0;
    for (int i = 0; i < 12; ++i) {
        if (ep[i] >= 8) {
            emask |= 1u << i;
            eord |= (uint32_t)(ep[i] & 3) << (2 * ne);
            eflips |= (uint32_t)eo[i] << ne;
            ++ne;
        } else {
            nflips |= (uint32_t)eo[i] << nn;
            umask |= (uint32_t)(ep[i] < 4) << nn;
            ++nn;
        }
    }
    if (K_MODE == 2) return ((uint64_t)SLICE_RANK[emask] * 70u + CCOMB_RANK[umask]) * 16u + eflips;
    return ((uint64_t)SLICE_RANK[emask] * 256u + nflips) * K_NEC + GEN_CLASS[EORDER_RANK[eord] * 16u + eflips];
}

static uint64_t table_index(const cube* c) {
    uint32_t packed = CLASSIDX[corner_raw(c)];
    return (uint64_t)(packed >> 4) * K_NEDGE + edge_coord(c, packed & 15);
}

static void unrank(uint64_t idx, cube* s) {
    uint32_t cls = (uint32_t)(idx / K_NEDGE);
    uint64_t coord = idx % K_NEDGE;
    uint32_t raw = CLASS_REP[cls], twist = raw / 70u, dmask = CCOMB_UNRANK[raw % 70u];
    uint32_t sum = 0, nu = 0, nd = 0;
    for (int i = 0; i < 8; ++i) {
        uint32_t o;
        if (i < 7) o = twist % 3, twist /= 3, sum += o;
        else o = (3 - sum % 3) % 3;
        s->co[i] = (uint8_t)o;
        s->cp[i] = (uint8_t)((dmask >> i) & 1 ? 4 + nd++ : nu++);
    }
    uint32_t emask, eord, eflips, umask, nflips;
    if (K_MODE == 2) {
        eflips = (uint32_t)(coord % 16);
        uint64_t rest = coord / 16;
        umask = CCOMB_UNRANK[rest % 70];
        emask = SLICE_UNRANK[rest / 70];
        eord = 0xE4;
        nflips = 0;
    } else {
        uint32_t gc = (uint32_t)(coord % K_NEC);
        uint64_t rest = coord / K_NEC;
        nflips = (uint32_t)(rest % 256);
        emask = SLICE_UNRANK[rest / 256];
        uint32_t content = GEN_REP[__builtin_popcount(nflips) & 1][gc];
        eord = EORDER_UNRANK[content >> 4];
        eflips = content & 15;
        umask = 0x0F;
    }
    uint32_t ne = 0, no = 0, nue = 0, nde = 0;
    for (int i = 0; i < 12; ++i) {
        if ((emask >> i) & 1) {
            s->ep[i] = (uint8_t)(8 | ((eord >> (2 * ne)) & 3));
            s->eo[i] = (uint8_t)((eflips >> ne) & 1);
            ++ne;
        } else {
            s->ep[i] = (uint8_t)((umask >> no) & 1 ? nue++ : 4 + nde++);
            s->eo[i] = (uint8_t)((nflips >> no) & 1);
            ++no;
        }
    }
}

void orc_index(const uint32_t* words, int n, int move, uint64_t* out) {
    for (int i = 0; i < n; ++i) {
        cube c;
        from_words(words + 5 * i, &c);
        if (move >= 0) move_right(&c, move);
        if (move <= -2) move_left(&c, -2 - move);
        out[i] = table_index(&c);
    }
}

void orc_unrank(const uint64_t* idx, int n, uint32_t* out_words) {
    for (int i = 0; i < n; ++i) {
        cube c;
        unrank(idx[i], &c);
        to_words(&c, out_words + 5 * i);
    }
}

/* ---- table decoding / encoding ---------------------------------------------------------- */

static uint32_t lower_bound(const uint8_t* tab, int fmt, uint64_t idx) {
    if (fmt == 1) {
        uint64_t b = idx / 155;
        uint32_t j = (uint32_t)(idx % 155);
        const uint8_t* p = tab + b * 32;
        uint32_t hdr = p[0], byte = p[1 + j / 5], d = byte;
        for (uint32_t k = 0; k < j % 5; ++k) d /= 3;
        d %= 3;
        uint32_t m = hdr & 63;
        return d == 0 ? m : m + (hdr >> 6) + d;
    }
    uint64_t b = idx / 124;
    uint32_t pos = 8 + 2 * (uint32_t)(idx % 124);
    const uint8_t* p = tab + b * 32;
    return p[0] + ((p[pos >> 3] >> (pos & 7)) & 3);
}

void orc_lower_bound(const uint8_t* tab, int fmt, const uint32_t* words, int n, uint32_t* out) {
    for (int i = 0; i < n; ++i) {
        cube c;
        from_words(words + 5 * i, &c);
        out[i] = lower_bound(tab, fmt, table_index(&c));
    }
}

/* 2-bit block file from exact depths: per 124 entries a u8 minimum, then min(depth - min, 3) at bit 8 + 2j. */
void orc_encode_block(const uint8_t* depth, uint64_t n, uint8_t* out) {
    uint64_t nb = (n + 123) / 124;
    for (uint64_t b = 0; b < nb; ++b) {
        uint64_t first = b * 124, cnt = n - first < 124 ? n - first : 124;
        uint32_t mn = 255;
        for (uint64_t j = 0; j < cnt; ++j) mn = depth[first + j] < mn ? depth[first + j] : mn;
        uint8_t* o = out + b * 32;
        memset(o, 0, 32);
        o[0] = (uint8_t)mn;
        for (uint64_t j = 0; j < cnt; ++j) {
            uint32_t off = depth[first + j] - mn;
            off = off > 3 ? 3 : off;
            uint32_t pos = 8 + 2 * (uint32_t)j;
            o[pos >> 3] |= (uint8_t)(off << (pos & 7));
        }
    }
}

/* Base-3 file: the value of entry x is what the reference recovers from its 2-bit block and
 * mod-3 tables (block value, and for offset 3 the smallest value >= min + 3 with the right
 * residue, the minimum read from the 2-bit block file `blk`); per 155 entries the minimum, the
 * cut maximising the encoded sum (lowest on ties), and five base-3 digits per byte. */
void orc_encode_b3(const uint8_t* depth, const uint8_t* blk, uint64_t n, uint8_t* out) {
    uint64_t nb = (n + 154) / 155;
    for (uint64_t b = 0; b < nb; ++b) {
        uint64_t first = b * 155, cnt = n - first < 155 ? n - first : 155;
        uint8_t v[155];
        uint32_t m = 255;
        for (uint64_t j = 0; j < cnt; ++j) {
            uint64_t x = first + j;
            uint32_t m124 = blk[(x / 124) * 32], d = depth[x], val;
            if (d - m124 < 3) val = d;
            else {
                val = m124 + 3;
                while (val % 3 != d % 3) ++val;
            }
            v[j] = (uint8_t)val;
            m = val < m ? val : m;
        }
        uint32_t best = 0, best_score = 0;
        for (uint32_t c = 0; c < 4; ++c) {
            uint32_t score = 0;
            for (uint64_t j = 0; j < cnt; ++j) score += v[j] <= m + c ? m : (v[j] == m + c + 1 ? m + c + 1 : m + c + 2);
            if (score > best_score) best_score = score, best = c;
        }
        uint8_t* o = out + b * 32;
        o[0] = (uint8_t)(m | (best << 6));
        for (uint32_t q = 0; q < 31; ++q) {
            uint32_t x = 0;
            for (int k = 4; k >= 0; --k) {
                uint64_t j = q * 5 + (uint32_t)k;
                uint32_t d = 0;
                if (j < cnt) d = v[j] <= m + best ? 0 : (v[j] == m + best + 1 ? 1 : 2);
                x = x * 3 + d;
            }
            o[1 + q] = (uint8_t)x;
        }
    }
}

/* ---- BFS ---------------------------------------------------------------------------------- */

typedef struct {
    uint8_t* depth;
    uint64_t lo, hi;
    uint32_t d;
    int forward;
    uint64_t found;
} bfs_job;

static uint32_t claim(uint8_t* depth, uint64_t idx, uint8_t value) {
    uint8_t expected = 0xFF;
    if (__atomic_load_n(depth + idx, __ATOMIC_RELAXED) != 0xFF) return 0;
    return __atomic_compare_exchange_n(depth + idx, &expected, value, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
}

/* Claim the coset of n and its images under the symmetries fixing its class representative. */
static uint32_t claim_with_stabilizer(uint8_t* depth, const cube* n, uint8_t value) {
    uint32_t packed = CLASSIDX[corner_raw(n)], cls = packed >> 4, sym = packed & 15, stab = CLASS_STAB[cls];
    uint32_t claimed = 0;
    for (uint32_t t = 0; t < 16; ++t)
        if ((stab >> t) & 1) claimed += claim(depth, (uint64_t)cls * K_NEDGE + edge_coord(n, SY_MUL[t][sym]), value);
    return claimed;
}

static void* bfs_worker(void* arg) {
    bfs_job* j = (bfs_job*)arg;
    uint64_t found = 0;
    for (uint64_t x = j->lo; x < j->hi; ++x) {
        uint8_t v = __atomic_load_n(j->depth + x, __ATOMIC_RELAXED);
        if (j->forward ? v != j->d : v != 0xFF) continue;
        cube s;
        unrank(x, &s);
        for (int m = 0; m < 18; ++m) {
            cube n = s;
            move_right(&n, m);
            if (j->forward) {
                found += claim_with_stabilizer(j->depth, &n, (uint8_t)(j->d + 1));
            } else if (__atomic_load_n(j->depth + table_index(&n), __ATOMIC_RELAXED) == j->d) {
                __atomic_store_n(j->depth + x, (uint8_t)(j->d + 1), __ATOMIC_RELAXED);
                ++found;
                break;
            }
        }
    }
    j->found = found;
    return NULL;
}

/* Exact BFS into depth[n] (0xFF = unvisited); counts[] gets the entries per depth.  Forward
 * passes while the frontier is under a quarter of the unvisited entries (table.py:112). */
int orc_bfs(uint8_t* depth, int threads, uint64_t* counts, int max_depths) {
    uint64_t n = orc_n_entries();
    memset(depth, 0xFF, n);
    cube solved = {{0, 1, 2, 3, 4, 5, 6, 7}, {0}, {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11}, {0}};
    counts[0] = claim_with_stabilizer(depth, &solved, 0);
    uint64_t remaining = n - counts[0];
    int nd = 1;
    pthread_t tid[256];
    bfs_job jobs[256];
    if (threads > 256) threads = 256;
    for (uint32_t d = 0; remaining; ++d) {
        if (nd >= max_depths) return -1;
        int forward = counts[nd - 1] < remaining / 4;
        for (int t = 0; t < threads; ++t) {
            jobs[t] = (bfs_job){depth, n * t / threads, n * (t + 1) / threads, d, forward, 0};
            pthread_create(&tid[t], NULL, bfs_worker, &jobs[t]);
        }
        uint64_t found = 0;
        for (int t = 0; t < threads; ++t) {
            pthread_join(tid[t], NULL);
            found += jobs[t].found;
        }
        if (!found) return -2;
        counts[nd++] = found;
        remaining -= found;
    }
    return nd;
}

/* ---- IDA* ----------------------------------------------------------------------------------- */

typedef struct {
    const uint8_t* tab;
    int fmt;
    uint64_t nodes, probes;
    uint8_t path[24];
    int bound;
    volatile int* stop;
} search;

static int allowed(int last, int m) {
    if (last < 0) return 1;
    int lf = last / 3, mf = m / 3;
    return mf != lf && !(lf >= 3 && mf == lf - 3);
}

static void frame_do(cube* f, int k, int m) {
    if (k < 3) move_right(f, FRAME_MOVE[k][m]);
    else move_left(f, inverse_move(FRAME_MOVE[k - 3][m]));
}

/* Frames at the budget edge first, then one below, then the rest (index order within each). */
static int frame_order(const uint32_t h[6], uint32_t edge, int order[6]) {
    int n = 0;
    for (int cls = 0; cls < 3; ++cls)
        for (int j = 0; j < 6; ++j) {
            int c = h[j] >= edge ? 0 : (h[j] + 1 == edge ? 1 : 2);
            if (c == cls) order[n++] = j;
        }
    return n;
}

static int all_axes_tight(const uint32_t c[6], uint32_t budget) {
    if (budget == 0) return 0;
    return (c[0] == budget && c[1] == budget && c[2] == budget) || (c[3] == budget && c[4] == budget && c[5] == budget);
}

static int dfs(search* S, const cube f[6], const uint32_t h[6], int g, int last) {
    if (g == S->bound) return is_solved(&f[0]);
    if (S->stop && *S->stop) return 0;
    uint32_t budget = (uint32_t)(S->bound - g);
    int order[6];
    frame_order(h, budget, order);
    for (int m = 0; m < 18; ++m) {
        if (!allowed(last, m)) continue;
        int axis = (m / 3) % 3;
        if (h[3 + axis] == budget) continue; /* axis rule: no solution of this length starts on that axis */
        ++S->nodes;
        int inherit = 3 + axis; /* same coset: the inverse frame on the move's axis keeps its value */
        uint32_t c[6];
        memcpy(c, h, sizeof c);
        cube child[6];
        int pruned = 0;
        for (int i = 0; i < 6 && !pruned; ++i) {
            int k = order[i];
            if (k == inherit) continue;
            child[k] = f[k];
            frame_do(&child[k], k, m);
            uint32_t v = lower_bound(S->tab, S->fmt, table_index(&child[k]));
            ++S->probes;
            if (k < 3 && h[k] && v < h[k] - 1) v = h[k] - 1;
            c[k] = v;
            if ((uint32_t)g + 1 + v > (uint32_t)S->bound) pruned = 1;
        }
        if (pruned || all_axes_tight(c, budget - 1)) continue;
        child[inherit] = f[inherit];
        frame_do(&child[inherit], inherit, m);
        if (dfs(S, child, c, g + 1, m)) {
            S->path[g] = (uint8_t)m;
            return 1;
        }
    }
    return 0;
}

/* Solve one cube given its six frames (30 words, g / R g R^-1 / R^2 g R^-2 and inverses).
 * Returns the optimal length (or -1 if stopped); moves[24]; nodes / probes over all bounds. */
int orc_solve_frames(const uint8_t* tab, int fmt, const uint32_t* frames30, uint8_t* moves, uint64_t* nodes,
                     uint64_t* probes, volatile int* stop) {
    cube f[6];
    uint32_t h[6];
    search S = {tab, fmt, 0, 0, {0}, 0, stop};
    uint32_t bound = 0;
    for (int k = 0; k < 6; ++k) {
        from_words(frames30 + 5 * k, &f[k]);
        h[k] = lower_bound(tab, fmt, table_index(&f[k]));
        ++S.probes;
        bound = h[k] > bound ? h[k] : bound;
    }
    int len = -1;
    if (is_solved(&f[0])) len = 0;
    for (uint32_t b = bound ? bound : 1; len < 0 && b <= 22; ++b) {
        S.bound = (int)b;
        if (dfs(&S, f, h, 0, -1)) len = (int)b;
        if (stop && *stop) break;
    }
    if (len > 0) memcpy(moves, S.path, (size_t)len);
    if (nodes) *nodes = S.nodes;
    if (probes) *probes = S.probes;
    return len;
}

/* ---- multi-threaded solving (the CPU baseline) ---------------------------------------------- */

typedef struct {
    const uint8_t* tab;
    int fmt;
    const uint32_t* frames;
    int n;
    int* next;
    int32_t* lengths;
    uint8_t* moves;
    uint64_t* nodes;
    uint64_t* probes;
    volatile int* stop;
    pthread_mutex_t* mu;
} pool_job;

static void* pool_worker(void* arg) {
    pool_job* j = (pool_job*)arg;
    for (;;) {
        pthread_mutex_lock(j->mu);
        int i = (*j->next)++;
        pthread_mutex_unlock(j->mu);
        if (i >= j->n || *j->stop) break;
        j->lengths[i] = orc_solve_frames(j->tab, j->fmt, j->frames + 30ull * i, j->moves + 24ull * i, &j->nodes[i],
                                         &j->probes[i], j->stop);
    }
    return NULL;
}

static volatile int g_stop;

static void* stop_timer(void* arg) {
    double secs = *(double*)arg;
    struct timespec ts = {(time_t)secs, (long)((secs - (double)(time_t)secs) * 1e9)};
    nanosleep(&ts, NULL);
    g_stop = 1;
    return NULL;
}

/* Solve n cubes on `threads` host threads; stop after `budget_s` seconds (0: no limit).
 * lengths[i] = -1 for cubes not finished; nodes / probes count the work done on every cube. */
int orc_solve_many(const uint8_t* tab, int fmt, const uint32_t* frames, int n, int threads, double budget_s,
                   int32_t* lengths, uint8_t* moves, uint64_t* nodes, uint64_t* probes) {
    pthread_t tid[512], timer;
    pool_job job;
    pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
    int next = 0;
    g_stop = 0;
    for (int i = 0; i < n; ++i) lengths[i] = -1, nodes[i] = 0, probes[i] = 0;
    job = (pool_job){tab, fmt, frames, n, &next, lengths, moves, nodes, probes, &g_stop, &mu};
    if (threads > 512) threads = 512;
    int timed = budget_s > 0;
    if (timed) pthread_create(&timer, NULL, stop_timer, &budget_s);
    for (int t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, pool_worker, &job);
    for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
    if (timed) {
        g_stop = 1;
        pthread_cancel(timer);
        pthread_join(timer, NULL);
    }
    int done = 0;
    for (int i = 0; i < n; ++i) done += lengths[i] >= 0;
    return done;
}
