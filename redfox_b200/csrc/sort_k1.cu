// sort_k1.cu -- radix sort instantiations for 1-byte keys.
#include "sort_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SORT(1)
}  // namespace rfx
