// jit.cpp -- NVRTC front end for the plan-specialised kernels (see jit.h).
#include "jit.h"

#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

namespace rfx {

namespace {

struct Nvrtc {
  bool tried = false;
  bool ok = false;
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
};

std::mutex g_mu;
Nvrtc g_nv;
std::map<std::pair<int, std::string>, cudaKernel_t> g_cache;

bool env_disabled() {
  const char* e = std::getenv("RFX_JIT");
  return e && (std::strcmp(e, "0") == 0 || std::strcmp(e, "off") == 0);
}

bool open_nvrtc() {
  if (g_nv.tried) return g_nv.ok;
  g_nv.tried = true;
  const char* names[] = {"/usr/local/cuda/lib64/libnvrtc.so.12", "libnvrtc.so.12", "libnvrtc.so"};
  void* h = nullptr;
  for (const char* n : names)
    if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
  if (!h) return false;
#define RFX_SYM(field, sym) g_nv.field = reinterpret_cast<decltype(g_nv.field)>(dlsym(h, #sym))
  RFX_SYM(create, nvrtcCreateProgram);
  RFX_SYM(compile, nvrtcCompileProgram);
  RFX_SYM(cubin_size, nvrtcGetCUBINSize);
  RFX_SYM(cubin, nvrtcGetCUBIN);
  RFX_SYM(log_size, nvrtcGetProgramLogSize);
  RFX_SYM(log, nvrtcGetProgramLog);
  RFX_SYM(destroy, nvrtcDestroyProgram);
#undef RFX_SYM
  g_nv.ok = g_nv.create && g_nv.compile && g_nv.cubin_size && g_nv.cubin && g_nv.log_size && g_nv.log && g_nv.destroy;
  return g_nv.ok;
}

}  // namespace

bool jit_available() {
  if (env_disabled()) return false;
  std::lock_guard<std::mutex> lk(g_mu);
  return open_nvrtc();
}

rfx_status jit_kernel(const std::string& source, const char* name, cudaKernel_t* out) {
  if (env_disabled()) return RFX_ERR_UNSUPPORTED;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return RFX_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  auto key = std::make_pair(dev, source);
  auto it = g_cache.find(key);
  if (it != g_cache.end()) {
    *out = it->second;
    return RFX_OK;
  }
  if (!open_nvrtc()) return RFX_ERR_UNSUPPORTED;
  nvrtcProgram prog;
  if (g_nv.create(&prog, source.c_str(), "rfx_plan.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) return RFX_ERR_UNSUPPORTED;
  const char* opts[] = {"-arch=sm_100a", "-std=c++17", "-default-device", "-lineinfo"};
  nvrtcResult r = g_nv.compile(prog, 4, opts);
  if (r != NVRTC_SUCCESS) {
    size_t ls = 0;
    g_nv.log_size(prog, &ls);
    std::vector<char> logbuf(ls + 1, 0);
    g_nv.log(prog, logbuf.data());
    std::fprintf(stderr, "rfx: runtime compilation failed:\n%s\n", logbuf.data());
    g_nv.destroy(&prog);
    return RFX_ERR_UNSUPPORTED;
  }
  size_t cs = 0;
  g_nv.cubin_size(prog, &cs);
  std::vector<char> cubin(cs);
  g_nv.cubin(prog, cubin.data());
  g_nv.destroy(&prog);
  cudaLibrary_t lib;
  if (cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    return RFX_ERR_CUDA;
  }
  cudaKernel_t k;
  if (cudaLibraryGetKernel(&k, lib, name) != cudaSuccess) {
    (void)cudaGetLastError();
    return RFX_ERR_CUDA;
  }
  g_cache[key] = k;
  *out = k;
  return RFX_OK;
}

}  // namespace rfx
