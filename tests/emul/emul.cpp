// Host build of libccs's device cube math (csrc/cube_dev.cuh), for CPU tests only: the CUDA
// qualifiers are defined away and the integer intrinsics it uses are written out in plain C++,
// so the exact kernel arithmetic (moves, table index, unrank, table decoding) can be checked
// against the CPU oracle without a GPU.  Not part of the product: libccs never links it.
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>

#define __device__
#define __host__
#define __forceinline__ inline
#define __global__
#define __restrict__
#define CCS_HOST_EMULATION 1

static inline uint32_t __byte_perm(uint32_t a, uint32_t b, uint32_t s) {
    uint64_t x = ((uint64_t)b << 32) | a;
    uint32_t r = 0;
    for (int i = 0; i < 4; ++i) {
        uint32_t sel = (s >> (4 * i)) & 7u;
        r |= (uint32_t)((x >> (8 * sel)) & 0xFFu) << (8 * i);
    }
    return r;
}
static inline int __popc(uint32_t v) { return __builtin_popcount(v); }
static inline int __ffs(uint32_t v) { return v ? __builtin_ctz(v) + 1 : 0; }
static inline uint32_t __dp4a(uint32_t a, uint32_t b, uint32_t c) {
    for (int i = 0; i < 4; ++i) c += ((a >> (8 * i)) & 0xFFu) * ((b >> (8 * i)) & 0xFFu);
    return c;
}
template <typename T>
static inline T __ldg(const T* p) { return *p; }

#include "../../cuda-cube-solver_b200/csrc/cube_dev.cuh"
#include "../../cuda-cube-solver_b200/csrc/dev_tables.h"

using namespace ccs;

namespace {
struct Kind {
    KindDesc desc;
    std::unique_ptr<DevTables> T;
};
std::map<std::string, Kind> kinds_;

Kind* kind(const char* name) {
    auto it = kinds_.find(name);
    if (it == kinds_.end()) {
        Kind k;
        if (!preset_kind(name, &k.desc)) return nullptr;
        k.T = std::make_unique<DevTables>();
        build_dev_tables(k.desc, k.T.get());
        it = kinds_.emplace(name, std::move(k)).first;
    }
    return &it->second;
}

template <typename F>
int with_kind(const KindDesc& d, F&& f) {
    if (d.mode == KIND_304) return f(std::integral_constant<int, KIND_304>{}, std::integral_constant<int, 1>{});
    switch (d.nec) {
        case 8: return f(std::integral_constant<int, KIND_GEN>{}, std::integral_constant<int, 8>{});
        case 12: return f(std::integral_constant<int, KIND_GEN>{}, std::integral_constant<int, 12>{});
        case 16: return f(std::integral_constant<int, KIND_GEN>{}, std::integral_constant<int, 16>{});
        case 24: return f(std::integral_constant<int, KIND_GEN>{}, std::integral_constant<int, 24>{});
    }
    return -1;
}
}  // namespace

extern "C" {

// move >= 0: right multiply first; move <= -2: left multiply by -2 - move.
int emul_index(const char* name, const uint32_t* w, int n, int move, uint64_t* out, uint32_t* out_w) {
    Kind* k = kind(name);
    if (!k) return -1;
    const uint32_t* classidx = corner_classes().classidx.data();
    return with_kind(k->desc, [&](auto M, auto N) {
        for (int i = 0; i < n; ++i) {
            State s{w[5 * i], w[5 * i + 1], w[5 * i + 2], w[5 * i + 3], w[5 * i + 4]};
            if (move >= 0) move_right(*k->T, s, move);
            if (move <= -2) move_left(*k->T, s, -2 - move);
            out[i] = table_index_dev<decltype(M)::value, decltype(N)::value>(*k->T, classidx, s);
            uint32_t o[5] = {s.c0, s.c1, s.e0, s.e1, s.e2};
            std::memcpy(out_w + 5 * i, o, sizeof o);
        }
        return 0;
    });
}

int emul_unrank(const char* name, const uint64_t* idx, int n, uint32_t* out_w) {
    Kind* k = kind(name);
    if (!k) return -1;
    const uint32_t* rep = corner_classes().rep.data();
    return with_kind(k->desc, [&](auto M, auto N) {
        for (int i = 0; i < n; ++i) {
            State s;
            unrank_dev<decltype(M)::value, decltype(N)::value>(*k->T, rep, idx[i], s);
            uint32_t o[5] = {s.c0, s.c1, s.e0, s.e1, s.e2};
            std::memcpy(out_w + 5 * i, o, sizeof o);
        }
        return 0;
    });
}

// Sector and entry of cls * NE + e by the search's 32-bit arithmetic (split_sector).
int emul_split_sector(const char* name, int fmt, const uint32_t* cls, const uint32_t* e, int n, uint64_t* out) {
    Kind* k = kind(name);
    if (!k) return -1;
    return with_kind(k->desc, [&](auto M, auto N) {
        constexpr uint64_t NE = KindTraits<decltype(M)::value, decltype(N)::value>::N_EDGE;
        for (int i = 0; i < n; ++i) {
            uint32_t sector, j;
            if (fmt) split_sector<FMT_B3, NE>(cls[i], e[i], sector, j);
            else split_sector<FMT_BLOCK, NE>(cls[i], e[i], sector, j);
            out[2 * i] = sector;
            out[2 * i + 1] = j;
        }
        return 0;
    });
}

int emul_lower_bound(const uint32_t* table, int fmt, const uint64_t* idx, int n, uint32_t* out) {
    for (int i = 0; i < n; ++i) out[i] = fmt ? lower_bound_dev<FMT_B3>(table, idx[i]) : lower_bound_dev<FMT_BLOCK>(table, idx[i]);
    return 0;
}
}
