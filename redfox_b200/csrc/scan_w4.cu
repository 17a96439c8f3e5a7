// scan_w4.cu -- scan kernel instantiations for 4-byte input rows.
#include "scan_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SCAN(4)
}  // namespace rfx
