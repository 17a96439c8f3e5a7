// jit.h -- in-process runtime compilation of plan-specialised kernels.
//
// The reference generates CUDA source per RA operator and compiles it with nvcc
// (RelationalAlgebraKernel.cpp:849-909, CudaCompilerInterface.cpp:126-404).  Here the
// scan kernels are generated from the compiled ScanProgram and compiled with NVRTC for
// sm_100a, loaded with cudaLibraryLoadData and cached per (source, device).  NVRTC is
// opened with dlopen on first use, so the library loads on hosts without it.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "rfx/rfx.h"

namespace rfx {

// Compiles (or fetches from the cache) `source` and returns the kernel `name`.
// Returns RFX_ERR_UNSUPPORTED when runtime compilation is unavailable or disabled
// (environment RFX_JIT=0); the caller then uses the interpreting kernels.
rfx_status jit_kernel(const std::string& source, const char* name, cudaKernel_t* out);

// Whether runtime compilation is enabled and NVRTC could be opened.
bool jit_available();

}  // namespace rfx
