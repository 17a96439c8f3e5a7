// scan_w64.cu -- scan kernel instantiations for 64-byte input rows.
#include "scan_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SCAN(64)
}  // namespace rfx
