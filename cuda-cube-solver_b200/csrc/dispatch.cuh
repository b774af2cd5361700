// Compile-time dispatch over the table kinds and formats libccs is built for.
#pragma once

#include <type_traits>

#include "ccs_internal.h"
#include "cube_dev.cuh"

namespace ccs {

// Calls f(integral_constant<MODE>, integral_constant<NEC>) for a supported kind.
template <typename F>
inline int dispatch_kind(const KindDesc& k, F&& f) {
    using std::integral_constant;
    if (k.mode == KIND_304) return f(integral_constant<int, KIND_304>{}, integral_constant<int, 1>{});
    switch (k.nec) {
        case 8: return f(integral_constant<int, KIND_GEN>{}, integral_constant<int, 8>{});
        case 12: return f(integral_constant<int, KIND_GEN>{}, integral_constant<int, 12>{});
        case 16: return f(integral_constant<int, KIND_GEN>{}, integral_constant<int, 16>{});
        case 24: return f(integral_constant<int, KIND_GEN>{}, integral_constant<int, 24>{});
    }
    return fail(CCS_E_ARG, "kinds with %d E-content classes are not compiled in (8, 12, 16, 24 are)", k.nec);
}

template <typename F>
inline int dispatch_fmt(int fmt, F&& f) {
    using std::integral_constant;
    if (fmt == CCS_FMT_BLOCK) return f(integral_constant<int, FMT_BLOCK>{});
    if (fmt == CCS_FMT_B3) return f(integral_constant<int, FMT_B3>{});
    return fail(CCS_E_ARG, "unknown table format %d", fmt);
}

}  // namespace ccs
