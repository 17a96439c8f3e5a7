// tune.cpp -- see tune.h.
#include "tune.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

namespace rfx {
namespace {

struct Entry {
  int variant;
  float ms[8];
  int ncand;
};

std::mutex g_mu;
int g_mode = -1;  // -1: not read from the environment yet
std::map<uint32_t, int> g_force;  // op -> pinned variant
std::map<std::tuple<int, uint32_t, uint64_t, uint32_t>, Entry> g_table;  // (device, op, shape, class)

int mode_locked() {
  if (g_mode < 0) {
    const char* e = std::getenv("RFX_TUNE");
    g_mode = (e && e[0] == '1') ? 1 : 0;
  }
  return g_mode;
}

}  // namespace

uint32_t size_class(uint64_t n) {
  uint32_t l = 0;
  while (n > 1) {
    n >>= 1;
    ++l;
  }
  return l / 2;
}

bool tune_enabled() {
  std::lock_guard<std::mutex> lk(g_mu);
  return mode_locked() == 1;
}

int tune_pick(uint32_t op, uint64_t shape, uint64_t n, int ncand, const std::function<rfx_status(int)>& run,
              cudaStream_t stream) {
  if (ncand <= 1) return 0;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto f = g_force.find(op);
    if (f != g_force.end() && f->second < ncand) return f->second;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, op, shape, size_class(n));
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (mode_locked() != 1) return 0;
    auto it = g_table.find(key);
    if (it != g_table.end()) return it->second.variant;
  }
  Entry e;
  e.ncand = ncand < 8 ? ncand : 8;
  e.variant = 0;
  float best = 1e30f;
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess) return 0;
  if (cudaEventCreate(&b) != cudaSuccess) {
    cudaEventDestroy(a);
    return 0;
  }
  for (int v = 0; v < e.ncand; ++v) {
    e.ms[v] = -1.0f;
    if (run(v) != RFX_OK) continue;  // untimed first run (compiles, caches launch shapes)
    float mv = 1e30f;
    for (int r = 0; r < 3; ++r) {
      cudaEventRecord(a, stream);
      const rfx_status st = run(v);
      cudaEventRecord(b, stream);
      if (st != RFX_OK || cudaEventSynchronize(b) != cudaSuccess) {
        mv = 1e30f;
        break;
      }
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      if (ms < mv) mv = ms;
    }
    e.ms[v] = mv < 1e30f ? mv : -1.0f;
    if (mv < best) {
      best = mv;
      e.variant = v;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  (void)cudaGetLastError();
  std::lock_guard<std::mutex> lk(g_mu);
  g_table[key] = e;
  return e.variant;
}

}  // namespace rfx

// 0: defaults (no tuning), 1: tune each (operator, shape, size class) on first use.
extern "C" void rfx_tune_set(int mode) {
  std::lock_guard<std::mutex> lk(rfx::g_mu);
  rfx::g_mode = mode == 1 ? 1 : 0;
}

// Pins operator `op` to `variant` (ahead of tuning and the default); variant < 0 unpins.
extern "C" void rfx_tune_force(uint32_t op, int variant) {
  std::lock_guard<std::mutex> lk(rfx::g_mu);
  if (variant < 0)
    rfx::g_force.erase(op);
  else
    rfx::g_force[op] = variant;
}

extern "C" void rfx_tune_reset(void) {
  std::lock_guard<std::mutex> lk(rfx::g_mu);
  rfx::g_table.clear();
}

// The tuning table as text, one line per entry:
// "op=<op> shape=<hex> class=<c> variant=<v> ms=<t0>,<t1>,..."; returns the bytes needed.
extern "C" size_t rfx_tune_dump(char* buf, size_t cap) {
  std::string s;
  {
    std::lock_guard<std::mutex> lk(rfx::g_mu);
    for (const auto& kv : rfx::g_table) {
      char line[256];
      int k = std::snprintf(line, sizeof(line), "op=%u shape=%llx class=%u variant=%d ms=", std::get<1>(kv.first),
                            (unsigned long long)std::get<2>(kv.first), std::get<3>(kv.first), kv.second.variant);
      for (int v = 0; v < kv.second.ncand && k < (int)sizeof(line) - 16; ++v)
        k += std::snprintf(line + k, sizeof(line) - k, v ? ",%.4f" : "%.4f", kv.second.ms[v]);
      s += line;
      s += '\n';
    }
  }
  if (buf && cap) {
    const size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return s.size() + 1;
}
