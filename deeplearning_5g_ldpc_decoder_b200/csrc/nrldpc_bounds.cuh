// nrldpc_bounds.cuh — device-side index checks of the debug build.
//
// libnrldpc_b200_debug.so is compiled with -DNRLDPC_BOUNDS_CHECK.  In it every
// gather and scatter index of the decode kernels is checked before the access:
// shared-memory belief words, base-graph edge entries, message-scratch words,
// rate-matched LLR reads and CRC table entries.  A violation never traps the
// GPU.  The first one is recorded (kind, index, limit, CTA) in the status
// words of the translation unit whose kernel made it.  The access is skipped:
// a load reads 0 and a store is dropped.  The host reads the record with
// nrldpc_bounds_check_status().  In the release library the checks compile
// to nothing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nrldpc {

enum BoundsKind : uint32_t {
  kBoundsLq = 1,        // shared-memory belief word (byte or element offset)
  kBoundsEdge = 2,      // base-graph edge index
  kBoundsScratch = 3,   // message scratch word of the CTA
  kBoundsLlr = 4,       // rate-matched LLR index of a code block
  kBoundsCrc = 5,       // CRC position-table entry
};

#ifdef NRLDPC_BOUNDS_CHECK
namespace {
// kind, index, limit, CTA of the first violation (one record per translation unit)
__device__ uint32_t g_bounds_record[4];
}  // namespace

__device__ __forceinline__ bool bounds_ok(bool ok, uint32_t kind, uint64_t index, uint64_t limit) {
  if (ok) return true;
  if (atomicCAS(&g_bounds_record[0], 0u, kind) == 0u) {
    g_bounds_record[1] = (uint32_t)index;
    g_bounds_record[2] = (uint32_t)limit;
    g_bounds_record[3] = blockIdx.x;
  }
  return false;
}
#define NRLDPC_INBOUNDS(idx, lim, kind) \
  (::nrldpc::bounds_ok((uint64_t)(idx) < (uint64_t)(lim), (kind), (uint64_t)(idx), (uint64_t)(lim)))

// Host side: copy this translation unit's record to out[4], optionally clear it.
static inline int bounds_read_tu(uint32_t* out, bool reset) {
  if (cudaMemcpyFromSymbol(out, g_bounds_record, 4 * sizeof(uint32_t)) != cudaSuccess) return -1;
  if (reset) {
    const uint32_t zero[4] = {0u, 0u, 0u, 0u};
    if (cudaMemcpyToSymbol(g_bounds_record, zero, sizeof(zero)) != cudaSuccess) return -1;
  }
  return 0;
}
constexpr bool kBoundsChecked = true;
#else
#define NRLDPC_INBOUNDS(idx, lim, kind) true
static inline int bounds_read_tu(uint32_t* out, bool) {
  out[0] = out[1] = out[2] = out[3] = 0u;
  return 0;
}
constexpr bool kBoundsChecked = false;
#endif

// One reader per translation unit with kernels (defined there).
int bounds_read_fixed(uint32_t* out, bool reset);
int bounds_read_float(uint32_t* out, bool reset);
int bounds_read_mixed(uint32_t* out, bool reset);

}  // namespace nrldpc
