// Host-side cube model for libccs (see cube_model.h).  Everything is derived from 3D geometry:
// face turns rotate the cubies of a layer by -90 degrees about the face normal, symmetries are
// signed permutation matrices acting on sticker slots.
#include "cube_model.h"

#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <set>
#include <stdexcept>

namespace ccs {
namespace {

using V3 = std::array<int, 3>;

const char* CORNER_NAMES[8] = {"URF", "UFL", "ULB", "UBR", "DFR", "DLF", "DBL", "DRB"};
const char* EDGE_NAMES[12] = {"UR", "UF", "UL", "UB", "DR", "DF", "DL", "DB", "FR", "FL", "BL", "BR"};
const char FACES[6] = {'U', 'R', 'F', 'D', 'L', 'B'};

V3 normal(char f) {
    switch (f) {
        case 'U': return {0, 1, 0};
        case 'R': return {1, 0, 0};
        case 'F': return {0, 0, 1};
        case 'D': return {0, -1, 0};
        case 'L': return {-1, 0, 0};
        default: return {0, 0, -1};  // B
    }
}

char face_of(const V3& n) {
    for (char f : FACES)
        if (normal(f) == n) return f;
    throw std::logic_error("not a face normal");
}

V3 center(const char* name) {
    V3 c{0, 0, 0};
    for (const char* p = name; *p; ++p) {
        V3 n = normal(*p);
        for (int a = 0; a < 3; ++a) c[a] += n[a];
    }
    return c;
}

// Clockwise quarter turn of face f seen from outside: rotation by -90 degrees about n,
// v -> (v . n) n + v x n.
V3 rotate_cw(char f, const V3& v) {
    V3 n = normal(f);
    int dot = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
    V3 cr{v[1] * n[2] - v[2] * n[1], v[2] * n[0] - v[0] * n[2], v[0] * n[1] - v[1] * n[0]};
    return {dot * n[0] + cr[0], dot * n[1] + cr[1], dot * n[2] + cr[2]};
}

template <int N>
void face_turn_part(char f, const char* const (&names)[N], int modulus, uint8_t* perm, uint8_t* orient) {
    V3 n = normal(f);
    for (int i = 0; i < N; ++i) perm[i] = (uint8_t)i, orient[i] = 0;
    for (int p = 0; p < N; ++p) {
        V3 c = center(names[p]);
        if (c[0] * n[0] + c[1] * n[1] + c[2] * n[2] <= 0) continue;
        V3 qc = rotate_cw(f, c);
        int q = -1;
        for (int j = 0; j < N; ++j)
            if (center(names[j]) == qc) q = j;
        perm[q] = (uint8_t)p;
        char lands = face_of(rotate_cw(f, normal(names[p][0])));
        const char* qn = names[q];
        int idx = (int)(std::find(qn, qn + std::char_traits<char>::length(qn), lands) - qn);
        orient[q] = (uint8_t)(idx % modulus);
    }
}

Cubie face_turn(char f) {
    Cubie c;
    face_turn_part(f, CORNER_NAMES, 3, c.cp, c.co);
    face_turn_part(f, EDGE_NAMES, 2, c.ep, c.eo);
    return c;
}

struct Mat {
    int m[3][3];
    V3 apply(const V3& v) const {
        V3 r{0, 0, 0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) r[i] += m[i][j] * v[j];
        return r;
    }
    int det() const {
        return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
               m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    }
    bool operator==(const Mat& o) const {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                if (m[i][j] != o.m[i][j]) return false;
        return true;
    }
    Mat operator*(const Mat& o) const {
        Mat r{};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                r.m[i][j] = 0;
                for (int k = 0; k < 3; ++k) r.m[i][j] += m[i][k] * o.m[k][j];
            }
        return r;
    }
};

// Cubie-level action of a matrix: position p (centre) goes to the position at M centre; slot 0
// of p (its first face) goes to slot cshift[p] / eflip[p] of the image.
template <int N>
void slot_action(const Mat& M, const char* const (&names)[N], uint8_t* perm, uint8_t* shift) {
    for (int p = 0; p < N; ++p) {
        V3 qc = M.apply(center(names[p]));
        int q = -1;
        for (int j = 0; j < N; ++j)
            if (center(names[j]) == qc) q = j;
        perm[p] = (uint8_t)q;
        char f = face_of(M.apply(normal(names[p][0])));
        const char* qn = names[q];
        shift[p] = (uint8_t)(std::find(qn, qn + std::char_traits<char>::length(qn), f) - qn);
    }
}

SymAction make_action(const Mat& M) {
    SymAction a;
    slot_action(M, CORNER_NAMES, a.cperm, a.cshift);
    slot_action(M, EDGE_NAMES, a.eperm, a.eflip);
    a.reflect = M.det() < 0;
    return a;
}

struct SymData {
    std::vector<Mat> ud;  // 16 U-D symmetries, reference order
    std::vector<SymAction> ud_act;
    SymAction rot;
    int mul[16][16];
    int fmove[3][18];
};

const SymData& syms() {
    static SymData* d = [] {
        auto* s = new SymData;
        std::vector<Mat> all;
        int perm[3] = {0, 1, 2};
        do {  // itertools.permutations order
            for (int signs = 0; signs < 8; ++signs) {  // itertools.product((1, -1), repeat=3)
                Mat m{};
                for (int r = 0; r < 3; ++r) m.m[r][perm[r]] = (signs >> (2 - r)) & 1 ? -1 : 1;
                all.push_back(m);
            }
        } while (std::next_permutation(perm, perm + 3));
        Mat eye{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
        auto it = std::find(all.begin(), all.end(), eye);
        Mat e = *it;
        all.erase(it);
        all.insert(all.begin(), e);
        for (const Mat& m : all)
            if (m.m[1][1] == 1 || m.m[1][1] == -1) s->ud.push_back(m);
        if (s->ud.size() != 16) throw std::logic_error("expected 16 U-D symmetries");
        for (const Mat& m : s->ud) s->ud_act.push_back(make_action(m));
        s->rot = make_action(Mat{{{0, 0, 1}, {1, 0, 0}, {0, 1, 0}}});
        for (int t = 0; t < 16; ++t)
            for (int u = 0; u < 16; ++u) {
                Mat p = s->ud[t] * s->ud[u];
                s->mul[t][u] = (int)(std::find(s->ud.begin(), s->ud.end(), p) - s->ud.begin());
            }
        return s;
    }();
    return *d;
}

std::vector<Cubie>& moves_vec() {
    static std::vector<Cubie>* mv = [] {
        auto* v = new std::vector<Cubie>;
        for (char f : FACES) {
            Cubie q = face_turn(f), p = identity();
            for (int t = 1; t <= 3; ++t) {
                p = compose(p, q);
                v->push_back(p);
            }
        }
        return v;
    }();
    return *mv;
}

template <typename T>
std::pair<std::vector<T>, std::vector<T>> combination_tables(int bits, int choose, T fill) {
    std::vector<T> rank(1u << bits, fill), unrank;
    // itertools.combinations order: lexicographic in the sorted positions.
    std::vector<int> c(choose);
    for (int i = 0; i < choose; ++i) c[i] = i;
    for (;;) {
        uint32_t mask = 0;
        for (int x : c) mask |= 1u << x;
        rank[mask] = (T)unrank.size();
        unrank.push_back((T)mask);
        int i = choose - 1;
        while (i >= 0 && c[i] == bits - choose + i) --i;
        if (i < 0) break;
        ++c[i];
        for (int j = i + 1; j < choose; ++j) c[j] = c[j - 1] + 1;
    }
    return {rank, unrank};
}

struct Ranks {
    std::vector<uint16_t> srank, sunrank, crank;
    std::vector<uint8_t> cunrank, erank, eunrank;
};

const Ranks& ranks() {
    static Ranks* r = [] {
        auto* x = new Ranks;
        auto s = combination_tables<uint16_t>(12, 4, 0xFFFF);
        x->srank = s.first;
        x->sunrank = s.second;
        auto c = combination_tables<uint16_t>(8, 4, 0xFFFF);
        x->crank = c.first;
        for (uint16_t v : c.second) x->cunrank.push_back((uint8_t)v);
        x->erank.assign(256, 0xFF);
        int p[4] = {0, 1, 2, 3};
        do {
            uint32_t key = 0;
            for (int j = 0; j < 4; ++j) key |= (uint32_t)p[j] << (2 * j);
            x->erank[key] = (uint8_t)x->eunrank.size();
            x->eunrank.push_back((uint8_t)key);
        } while (std::next_permutation(p, p + 4));
        return x;
    }();
    return *r;
}

}  // namespace

Cubie identity() {
    Cubie c;
    for (int i = 0; i < 8; ++i) c.cp[i] = (uint8_t)i, c.co[i] = 0;
    for (int i = 0; i < 12; ++i) c.ep[i] = (uint8_t)i, c.eo[i] = 0;
    return c;
}

Cubie compose(const Cubie& a, const Cubie& b) {
    Cubie r;
    for (int i = 0; i < 8; ++i) r.cp[i] = a.cp[b.cp[i]], r.co[i] = (uint8_t)((a.co[b.cp[i]] + b.co[i]) % 3);
    for (int i = 0; i < 12; ++i) r.ep[i] = a.ep[b.ep[i]], r.eo[i] = (uint8_t)((a.eo[b.ep[i]] + b.eo[i]) & 1);
    return r;
}

Cubie inverse(const Cubie& a) {
    Cubie r;
    for (int i = 0; i < 8; ++i) r.cp[a.cp[i]] = (uint8_t)i;
    for (int i = 0; i < 8; ++i) r.co[i] = (uint8_t)((3 - a.co[r.cp[i]]) % 3);
    for (int i = 0; i < 12; ++i) r.ep[a.ep[i]] = (uint8_t)i;
    for (int i = 0; i < 12; ++i) r.eo[i] = a.eo[r.ep[i]];
    return r;
}

const Cubie& move(int m) { return moves_vec().at(m); }

void pack(const Cubie& c, uint32_t w[5]) {
    uint8_t b[20];
    for (int i = 0; i < 8; ++i) b[i] = (uint8_t)(c.cp[i] | (c.co[i] << 3));
    for (int i = 0; i < 12; ++i) b[8 + i] = (uint8_t)(c.ep[i] | (c.eo[i] << 4));
    for (int j = 0; j < 5; ++j) w[j] = b[4 * j] | (b[4 * j + 1] << 8) | (b[4 * j + 2] << 16) | ((uint32_t)b[4 * j + 3] << 24);
}

Cubie unpack(const uint32_t w[5]) {
    Cubie c;
    for (int i = 0; i < 20; ++i) {
        uint8_t b = (uint8_t)(w[i >> 2] >> (8 * (i & 3)));
        if (i < 8) c.cp[i] = b & 7, c.co[i] = b >> 3;
        else c.ep[i - 8] = b & 15, c.eo[i - 8] = b >> 4;
    }
    return c;
}

bool is_legal(const Cubie& c) {
    uint32_t seen_c = 0, seen_e = 0;
    int cs = 0, es = 0;
    for (int i = 0; i < 8; ++i) {
        if (c.cp[i] > 7 || c.co[i] > 2) return false;
        seen_c |= 1u << c.cp[i];
        cs += c.co[i];
    }
    for (int i = 0; i < 12; ++i) {
        if (c.ep[i] > 11 || c.eo[i] > 1) return false;
        seen_e |= 1u << c.ep[i];
        es += c.eo[i];
    }
    if (seen_c != 0xFFu || seen_e != 0xFFFu || cs % 3 || es % 2) return false;
    int pc = 0, pe = 0;
    for (int i = 0; i < 8; ++i)
        for (int j = i + 1; j < 8; ++j) pc ^= c.cp[i] > c.cp[j];
    for (int i = 0; i < 12; ++i)
        for (int j = i + 1; j < 12; ++j) pe ^= c.ep[i] > c.ep[j];
    return pc == pe;
}

const SymAction& ud_sym(int s) { return syms().ud_act.at(s); }
const SymAction& axis_rotation() { return syms().rot; }
int ud_sym_mul(int t, int s) { return syms().mul[t][s]; }

Cubie conjugate(const SymAction& s, const Cubie& c) {
    Cubie r;
    int sign = s.reflect ? -1 : 1;
    for (int p = 0; p < 8; ++p) {
        int q = s.cperm[p], cub = c.cp[p];
        r.cp[q] = s.cperm[cub];
        r.co[q] = (uint8_t)(((s.cshift[p] + sign * c.co[p] - s.cshift[cub]) % 3 + 3) % 3);
    }
    for (int p = 0; p < 12; ++p) {
        int q = s.eperm[p], cub = c.ep[p];
        r.ep[q] = s.eperm[cub];
        r.eo[q] = (uint8_t)(c.eo[p] ^ s.eflip[p] ^ s.eflip[cub]);
    }
    return r;
}

int frame_move(int k, int m) {
    static std::array<std::array<int, 18>, 3>* fm = [] {
        auto* t = new std::array<std::array<int, 18>, 3>;
        std::map<std::vector<uint8_t>, int> lookup;
        auto key = [](const Cubie& c) {
            std::vector<uint8_t> v(c.cp, c.cp + 8);
            v.insert(v.end(), c.co, c.co + 8);
            v.insert(v.end(), c.ep, c.ep + 12);
            v.insert(v.end(), c.eo, c.eo + 12);
            return v;
        };
        for (int i = 0; i < 18; ++i) lookup[key(move(i))] = i;
        std::array<int, 18> rot{};
        for (int i = 0; i < 18; ++i) rot[i] = lookup.at(key(conjugate(axis_rotation(), move(i))));
        for (int i = 0; i < 18; ++i) {
            (*t)[0][i] = i;
            (*t)[1][i] = rot[i];
            (*t)[2][i] = rot[rot[i]];
        }
        return t;
    }();
    return (*fm)[k][m];
}

const std::vector<uint16_t>& slice_rank() { return ranks().srank; }
const std::vector<uint16_t>& slice_unrank() { return ranks().sunrank; }
const std::vector<uint16_t>& ccomb_rank() { return ranks().crank; }
const std::vector<uint8_t>& ccomb_unrank() { return ranks().cunrank; }
const std::vector<uint8_t>& eorder_rank() { return ranks().erank; }
const std::vector<uint8_t>& eorder_unrank() { return ranks().eunrank; }

uint32_t corner_raw(const uint8_t b[8]) {
    uint32_t twist = 0, w = 1, dmask = 0;
    for (int i = 0; i < 7; ++i, w *= 3) twist += (uint32_t)(b[i] >> 3) * w;
    for (int i = 0; i < 8; ++i) dmask |= (uint32_t)((b[i] >> 2) & 1) << i;
    return twist * N_CCOMB + ccomb_rank()[dmask];
}

namespace {
// Representative corner bytes of a raw coordinate (twist digits, the last closing the sum; U
// cubies 0..3 in non-D positions and D cubies 4..7 in D positions, each in position order).
void corners_from_raw(uint32_t raw, uint8_t b[8]) {
    uint32_t twist = raw / N_CCOMB, dmask = ccomb_unrank()[raw % N_CCOMB];
    uint32_t sum = 0, nu = 0, nd = 0;
    for (int i = 0; i < 8; ++i) {
        uint32_t o;
        if (i < 7) o = twist % 3, twist /= 3, sum += o;
        else o = (3 - sum % 3) % 3;
        uint32_t cp = (dmask >> i) & 1 ? 4 + nd++ : nu++;
        b[i] = (uint8_t)(cp | (o << 3));
    }
}

uint32_t conj_raw(const SymAction& s, uint32_t raw) {
    uint8_t b[8], r[8];
    corners_from_raw(raw, b);
    int sign = s.reflect ? -1 : 1;
    for (int p = 0; p < 8; ++p) {
        int cub = b[p] & 7, o = b[p] >> 3;
        int q = s.cperm[p];
        r[q] = (uint8_t)(s.cperm[cub] | ((((s.cshift[p] + sign * o - s.cshift[cub]) % 3 + 3) % 3) << 3));
    }
    return corner_raw(r);
}
}  // namespace

const CornerClasses& corner_classes() {
    static CornerClasses* cc = [] {
        auto* c = new CornerClasses;
        std::vector<uint32_t> omin(N_CORNER_RAW), first(N_CORNER_RAW);
        std::vector<std::array<uint32_t, 16>> img(N_CORNER_RAW);
        for (uint32_t raw = 0; raw < N_CORNER_RAW; ++raw) {
            uint32_t mn = UINT32_MAX, fs = 0;
            for (int s = 0; s < 16; ++s) {
                uint32_t v = conj_raw(ud_sym(s), raw);
                img[raw][s] = v;
                if (v < mn) mn = v, fs = (uint32_t)s;
            }
            omin[raw] = mn;
            first[raw] = fs;
        }
        std::vector<uint32_t> reps(omin);
        std::sort(reps.begin(), reps.end());
        reps.erase(std::unique(reps.begin(), reps.end()), reps.end());
        std::vector<int32_t> cls_of(N_CORNER_RAW, -1);
        for (size_t i = 0; i < reps.size(); ++i) cls_of[reps[i]] = (int32_t)i;
        c->classidx.resize(N_CORNER_RAW);
        for (uint32_t raw = 0; raw < N_CORNER_RAW; ++raw) c->classidx[raw] = ((uint32_t)cls_of[omin[raw]] << 4) | first[raw];
        c->rep = reps;
        c->stab.resize(reps.size());
        for (size_t i = 0; i < reps.size(); ++i) {
            uint16_t m = 0;
            for (int s = 0; s < 16; ++s)
                if (img[reps[i]][s] == reps[i]) m |= (uint16_t)(1u << s);
            c->stab[i] = m;
        }
        if (reps.size() != N_CLASSES) throw std::logic_error("expected 9,930 corner classes");
        return c;
    }();
    return *cc;
}

// ---- group kinds ------------------------------------------------------------------------

namespace {
struct Elem {
    std::array<int, 4> p, f;
    bool operator<(const Elem& o) const { return std::tie(p, f) < std::tie(o.p, o.f); }
    bool operator==(const Elem& o) const { return p == o.p && f == o.f; }
};
// a after b: label x -> a.p[b.p[x]], flip f_b[x] ^ f_a[b.p[x]]
Elem mul(const Elem& a, const Elem& b) {
    Elem r;
    for (int x = 0; x < 4; ++x) r.p[x] = a.p[b.p[x]], r.f[x] = b.f[x] ^ a.f[b.p[x]];
    return r;
}
Elem inv(const Elem& a) {
    Elem r;
    for (int z = 0; z < 4; ++z) r.p[a.p[z]] = z;
    for (int z = 0; z < 4; ++z) r.f[z] = a.f[r.p[z]];
    return r;
}
int perm_rank(const std::array<int, 4>& p) {
    uint32_t key = 0;
    for (int j = 0; j < 4; ++j) key |= (uint32_t)p[j] << (2 * j);
    return eorder_rank()[key];
}
}  // namespace

KindDesc make_group_kind(const std::string& name, const std::vector<std::pair<std::vector<int>, std::vector<int>>>& gens) {
    std::vector<Elem> g;
    for (auto& pr : gens) {
        Elem e;
        for (int x = 0; x < 4; ++x) e.p[x] = pr.first.at(x), e.f[x] = pr.second.at(x);
        g.push_back(e);
    }
    std::set<Elem> group{Elem{{0, 1, 2, 3}, {0, 0, 0, 0}}};
    std::vector<Elem> frontier(group.begin(), group.end());
    while (!frontier.empty()) {
        std::vector<Elem> next;
        for (auto& x : frontier)
            for (auto& y : g) {
                Elem z = mul(y, x);
                if (group.insert(z).second) next.push_back(z);
            }
        frontier = next;
    }
    // The relabellings of the E cubies (8..11) that the U-D symmetries induce.
    for (int s = 0; s < 16; ++s) {
        const SymAction& a = ud_sym(s);
        Elem se;
        for (int x = 0; x < 4; ++x) se.p[x] = a.eperm[8 + x] - 8, se.f[x] = a.eflip[8 + x];
        for (auto& x : group)
            if (!group.count(mul(mul(se, x), inv(se))))
                throw std::runtime_error(name + ": group not normalised by the UD symmetries; symmetry reduction would be wrong");
    }
    KindDesc k;
    k.mode = KIND_GEN;
    std::vector<int> cls(384, -1), reps;
    const auto& eun = eorder_unrank();
    for (int c = 0; c < 384; ++c) {
        if (cls[c] >= 0) continue;
        std::array<int, 4> q;
        for (int i = 0; i < 4; ++i) q[i] = (eun[c >> 4] >> (2 * i)) & 3;
        for (auto& e : group) {
            std::array<int, 4> np;
            int nf = 0;
            for (int i = 0; i < 4; ++i) np[i] = e.p[q[i]], nf |= ((((c >> i) & 1) ^ e.f[q[i]]) << i);
            cls[perm_rank(np) * 16 + nf] = (int)reps.size();
        }
        reps.push_back(c);
    }
    auto parity = [](int c) { return __builtin_popcount(c & 15) & 1; };
    bool even = true;
    for (auto& e : group) even &= ((e.f[0] + e.f[1] + e.f[2] + e.f[3]) % 2 == 0);
    if (even) {
        std::vector<int> within;
        int count[2] = {0, 0};
        for (int r : reps) {
            int p = parity(r);
            within.push_back(count[p]);
            k.gen_rep[p][count[p]] = (uint16_t)r;
            ++count[p];
        }
        k.nec = (int)reps.size() / 2;
        for (int c = 0; c < 384; ++c) k.gen_class[c] = (uint16_t)within[cls[c]];
    } else {
        k.nec = (int)reps.size();
        for (int c = 0; c < 384; ++c) k.gen_class[c] = (uint16_t)cls[c], k.gen_rep[parity(c)][cls[c]] = (uint16_t)c;
    }
    k.n_edge = (uint64_t)N_SLICE * 256u * (uint64_t)k.nec;
    k.n_entries = (uint64_t)N_CLASSES * k.n_edge;
    return k;
}

KindDesc make_304_kind() {
    KindDesc k;
    k.mode = KIND_304;
    k.nec = 1;
    k.n_edge = (uint64_t)N_SLICE * 70u * 16u;
    k.n_entries = (uint64_t)N_CLASSES * k.n_edge;
    return k;
}

bool preset_kind(const std::string& name, KindDesc* out) {
    using G = std::vector<std::pair<std::vector<int>, std::vector<int>>>;
    static const std::map<std::string, G> groups = {
        {"s4", {{{0, 1, 3, 2}, {0, 0, 0, 0}}, {{0, 2, 1, 3}, {0, 0, 0, 0}}, {{1, 0, 2, 3}, {0, 0, 0, 0}}}},
        {"d4f", {{{0, 1, 2, 3}, {1, 1, 1, 1}}, {{0, 3, 2, 1}, {0, 0, 0, 0}}, {{1, 0, 3, 2}, {0, 0, 0, 0}}}},
        {"a4t", {{{0, 2, 3, 1}, {0, 1, 1, 0}}, {{1, 0, 3, 2}, {1, 1, 1, 1}}}},
        {"d4t", {{{0, 3, 2, 1}, {0, 0, 0, 0}}, {{1, 0, 3, 2}, {1, 1, 1, 1}}}},
        {"d4", {{{1, 2, 3, 0}, {0, 0, 0, 0}}, {{0, 3, 2, 1}, {0, 0, 0, 0}}}},
        {"a4", {{{0, 2, 3, 1}, {0, 0, 0, 0}}, {{1, 0, 3, 2}, {0, 0, 0, 0}}}},
    };
    if (name == "304") {
        *out = make_304_kind();
        return true;
    }
    auto it = groups.find(name);
    if (it == groups.end()) return false;
    *out = make_group_kind(name, it->second);
    return true;
}

uint64_t table_index_host(const KindDesc& k, const uint32_t w[5]) {
    Cubie c = unpack(w);
    uint8_t cb[8];
    for (int i = 0; i < 8; ++i) cb[i] = (uint8_t)(c.cp[i] | (c.co[i] << 3));
    uint32_t packed = corner_classes().classidx[corner_raw(cb)];
    Cubie e = conjugate(ud_sym(packed & 15), c);
    uint32_t emask = 0, eord = 0, eflips = 0, nflips = 0, umask = 0, ne = 0, nn = 0;
    for (int i = 0; i < 12; ++i) {
        if (e.ep[i] >= 8) {
            emask |= 1u << i;
            eord |= (uint32_t)(e.ep[i] & 3) << (2 * ne);
            eflips |= (uint32_t)e.eo[i] << ne;
            ++ne;
        } else {
            nflips |= (uint32_t)e.eo[i] << nn;
            umask |= (uint32_t)(e.ep[i] < 4) << nn;
            ++nn;
        }
    }
    uint64_t coord;
    if (k.mode == KIND_304) {
        coord = ((uint64_t)slice_rank()[emask] * 70u + ccomb_rank()[umask]) * 16u + eflips;
    } else {
        uint32_t cl = k.gen_class[eorder_rank()[eord] * 16u + eflips];
        coord = ((uint64_t)slice_rank()[emask] * 256u + nflips) * (uint64_t)k.nec + cl;
    }
    return (uint64_t)(packed >> 4) * k.n_edge + coord;
}

}  // namespace ccs
