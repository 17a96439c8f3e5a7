// scan_w2.cu -- scan kernel instantiations for 2-byte input rows.
#include "scan_launch.cuh"
namespace rfx {
RFX_INSTANTIATE_SCAN(2)
}  // namespace rfx
