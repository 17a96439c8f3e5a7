// scan_w8.cu -- scan kernel instantiations for 8-byte input rows.
#include "scan_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SCAN(8)
}  // namespace rfx
