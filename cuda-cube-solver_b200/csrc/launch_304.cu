// Search kernels of the 304 edge kind.
#include "search_launch.cuh"

namespace ccs {
template int launch_kind<KIND_304, 1>(ccs_handle*, const SearchParams&, int, cudaStream_t, int);
template int kernel_footprint_kind<KIND_304, 1>(ccs_handle*, int, size_t*, int*);
}  // namespace ccs
