// host_common.cpp -- see host_common.h.
#include "host_common.h"

#include <cstring>
#include <mutex>
#include <unordered_map>

#include <cudaTypedefs.h>

namespace rfx {

rfx_status cuda_fail(cudaError_t e) {
  (void)cudaGetLastError();  // clear a non-sticky error so the next call starts clean
  return e == cudaSuccess ? RFX_OK : RFX_ERR_CUDA;
}

namespace {
std::mutex g_mu;
std::unordered_map<int, int> g_sms;
std::unordered_map<int, uint32_t*> g_err;
struct OccKey {
  const void* k;
  int threads;
  size_t smem;
  bool operator==(const OccKey& o) const { return k == o.k && threads == o.threads && smem == o.smem; }
};
struct OccHash {
  size_t operator()(const OccKey& o) const {
    return std::hash<const void*>()(o.k) ^ (o.smem * 131) ^ ((size_t)o.threads << 20);
  }
};
std::unordered_map<OccKey, int, OccHash> g_occ;
// cudaFuncSetAttribute applies to the current device only: the opt-in is remembered per
// (device, kernel)
struct SmemKey {
  int dev;
  const void* k;
  bool operator==(const SmemKey& o) const { return dev == o.dev && k == o.k; }
};
struct SmemHash {
  size_t operator()(const SmemKey& o) const { return std::hash<const void*>()(o.k) ^ ((size_t)o.dev << 40); }
};
std::unordered_map<SmemKey, size_t, SmemHash> g_smem_set;
}  // namespace

int device_sms() {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_sms.find(dev);
  if (it != g_sms.end()) return it->second;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  g_sms[dev] = sms;
  return sms;
}

uint32_t* device_error_word() {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_err.find(dev);
  if (it != g_err.end()) return it->second;
  uint32_t* p = nullptr;
  if (cudaMalloc(&p, sizeof(uint32_t)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, sizeof(uint32_t));
  cudaDeviceSynchronize();
  g_err[dev] = p;
  return p;
}

cudaError_t allow_smem(const void* kernel, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_mu);
  const SmemKey key{dev, kernel};
  auto it = g_smem_set.find(key);
  if (it != g_smem_set.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) g_smem_set[key] = bytes;
  return e;
}

int persistent_grid(const void* kernel, int threads, size_t dyn_smem, uint64_t work_blocks) {
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_occ.find(OccKey{kernel, threads, dyn_smem});
    if (it != g_occ.end()) per_sm = it->second;
  }
  if (per_sm == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, dyn_smem) != cudaSuccess || per_sm <= 0)
      per_sm = 1;
    std::lock_guard<std::mutex> lk(g_mu);
    g_occ[OccKey{kernel, threads, dyn_smem}] = per_sm;
  }
  uint64_t cap = (uint64_t)device_sms() * (uint64_t)per_sm;
  uint64_t g = work_blocks < cap ? work_blocks : cap;
  return (int)(g ? g : 1);
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}
}  // namespace

bool encode_line_map(CUtensorMap* map, const void* base, uint64_t lines, uint32_t box_lines) {
  std::memset(map, 0, sizeof(*map));
  if (!base || lines == 0 || lines > (1ull << 31) || (reinterpret_cast<uintptr_t>(base) & 15u) || box_lines == 0 ||
      box_lines > 256)
    return false;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {128, lines};
  cuuint64_t strides[1] = {128};
  cuuint32_t box[2] = {128, box_lines};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    std::memset(map, 0, sizeof(*map));
    return false;
  }
  return true;
}

}  // namespace rfx

extern "C" rfx_status rfx_device_status(void* stream) {
  uint32_t* w = rfx::device_error_word();
  if (!w) return RFX_ERR_CUDA;
  uint32_t v = 0;
  RFX_CUDA_TRY(cudaStreamSynchronize(rfx::as_stream(stream)));
  RFX_CUDA_TRY(cudaMemcpy(&v, w, sizeof(v), cudaMemcpyDeviceToHost));
  if (v) RFX_CUDA_TRY(cudaMemset(w, 0, sizeof(uint32_t)));
  return static_cast<rfx_status>(v);
}

extern "C" const char* rfx_version(void) { return "redfox_b200 0.1 (sm_100a)"; }
