// sort_k2.cu -- radix sort instantiations for 2-byte keys.
#include "sort_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SORT(2)
}  // namespace rfx
