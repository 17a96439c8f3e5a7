// shim_common.h -- shared by the redfox:: shim libraries: the reference's entries return
// void and abort on a CUDA error; the shims log a non-OK rfx_status instead and leave the
// outputs untouched (what the rfx_*_compat entries guarantee on a host-detected error).
#pragma once

#include <cstdio>

#include "rfx/rfx.h"

namespace redfox_shim {

inline void report(const char* entry, rfx_status st) {
  if (st != RFX_OK) std::fprintf(stderr, "redfox::%s: rfx status %d\n", entry, (int)st);
}

}  // namespace redfox_shim
