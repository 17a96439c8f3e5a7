// tune.h -- per-size-class choice of a kernel variant (tile shape, items per thread).
//
// Operators with more than one compiled variant ask `tune_pick` which one to run.  With
// tuning off (the default) the answer is variant 0, the hand-picked default.  With tuning
// on (rfx_tune_set(1) or RFX_TUNE=1 in the environment) the first call for a given
// (operator, shape, size class) runs every candidate on the caller's own inputs and
// stream, times each with CUDA events (one untimed run, then the best of three), and
// remembers the fastest; later calls of the same class reuse it without timing.  Only
// out-of-place operators are tuned, so repeated runs leave the same outputs.  Tuning
// synchronises the stream and must not be used while a stream is being captured.
#pragma once

#include <cstdint>
#include <functional>

#include "host_common.h"

namespace rfx {

enum TuneOp : uint32_t {
  TUNE_REDUCE_ROWS = 1,   // rfx_reduce_tuples, TMA-staged: chunked, or look-back per 256- / 128-line tile
  TUNE_SET_FILTER = 2,    // set intersection / difference / union's B - A: warp segments (bounds, mark,
                          // compact) with 16 or 8 items per thread, two passes with 16 or 8, or one pass
                          // with 8, 4 or 16
  TUNE_SCAN_COMPACT = 3,  // plan-specialised select / project: items per thread
  TUNE_SCAN_AGGREGATE = 4,  // plan-specialised filter-aggregate: rows per thread per iteration
  TUNE_SORT_PASS = 5,     // radix sort pass: per tile; onesweep (TMA stages + look-back warp; 3 tile sizes);
                          // per tile ranking with match_any
  TUNE_JOIN_EMIT = 6,     // fused join emit: operands staged in shared memory by bulk copies, or gathered
};

// Size class of n: floor(log2(n)) / 2 (classes of 4x).
uint32_t size_class(uint64_t n);

bool tune_enabled();

// Returns the variant to run (0 .. ncand-1).  `run(v)` launches variant v on `stream`
// and returns RFX_OK or an error (a failing candidate is skipped).
int tune_pick(uint32_t op, uint64_t shape, uint64_t n, int ncand, const std::function<rfx_status(int)>& run,
              cudaStream_t stream);

}  // namespace rfx
