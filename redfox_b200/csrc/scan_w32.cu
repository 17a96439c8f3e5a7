// scan_w32.cu -- scan kernel instantiations for 32-byte input rows.
#include "scan_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SCAN(32)
}  // namespace rfx
