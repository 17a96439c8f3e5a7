// scan_w1.cu -- scan kernel instantiations for 1-byte input rows.
#include "scan_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SCAN(1)
}  // namespace rfx
