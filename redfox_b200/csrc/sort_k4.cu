// sort_k4.cu -- radix sort instantiations for 4-byte keys.
#include "sort_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SORT(4)
}  // namespace rfx
