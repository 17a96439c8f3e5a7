// sort_k8.cu -- radix sort instantiations for 8-byte keys.
#include "sort_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SORT(8)
}  // namespace rfx
