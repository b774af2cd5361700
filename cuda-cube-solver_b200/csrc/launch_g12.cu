// Search kernels of group kinds of 12 E-content classes (d4f).
#include "search_launch.cuh"

namespace ccs {
template int launch_kind<KIND_GEN, 12>(ccs_handle*, const SearchParams&, int, cudaStream_t, int);
template int kernel_footprint_kind<KIND_GEN, 12>(ccs_handle*, int, size_t*, int*);
}  // namespace ccs
