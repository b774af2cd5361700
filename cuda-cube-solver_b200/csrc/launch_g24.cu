// Search kernels of group kinds of 24 E-content classes (d4t, d4).
#include "search_launch.cuh"

namespace ccs {
template int launch_kind<KIND_GEN, 24>(ccs_handle*, const SearchParams&, int, cudaStream_t, int);
template int kernel_footprint_kind<KIND_GEN, 24>(ccs_handle*, int, size_t*, int*);
}  // namespace ccs
