// scan_w16.cu -- scan kernel instantiations for 16-byte input rows.
#include "scan_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SCAN(16)
}  // namespace rfx
