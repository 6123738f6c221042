// nrldpc_decode_common.cuh — device helpers shared by the decode kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "nrldpc_bounds.cuh"
#include "nrldpc_internal.h"

namespace nrldpc {

// Stage one code block's circular-buffer LLRs into decoder order (HARQ index).
//
// Restates nr_ldpc_rate_recover_harq_combine (c_lib/ldpc_rate_recovery.c:24-65)
// in gather form.  HARQ index i in [0, N+2Zc):
//   * i <  2Zc          punctured systematic bits: receive no LLR;
//   * i in [B, K)       filler bits: set to filling_bit_value (overrides HARQ);
//   * otherwise         circular-buffer position pos = i - 2Zc, compacted to
//                       c = pos (pos < B-2Zc) or pos - F (pos >= K-2Zc).
// The k-th de-interleaved LLR lands on compact position (c0 + k) mod Nv, and
// LLR k is read from rate-matched index (k mod E/Qm)*Qm + k/(E/Qm).  All
// repetitions k = kf, kf+Nv, ... < E are summed; the reference adds them
// one by one into int16_t, which is the same sum modulo 2^16.
// Returns the recovered value as a 32-bit sum (caller truncates to int16).
__device__ __forceinline__ int32_t recover_position(const DecodeParams& p, const int16_t* __restrict__ in,
                                                    int i, int32_t init) {
  const int twoZ = 2 * p.Zc;
  if (i >= p.B && i < p.K) return p.fill;
  int32_t s = init;
  if (i < twoZ) return s;
  const int pos = i - twoZ;
  const int c = pos < p.B - twoZ ? pos : pos - p.F;
  int kf = c - p.c0;
  if (kf < 0) kf += p.Nv;
  for (int k = kf; k < p.E; k += p.Nv) {
    const int b = k / p.symbols;
    const int sidx = k - b * p.symbols;
    const int64_t idx = (int64_t)sidx * p.Qm + b;
    if (NRLDPC_INBOUNDS(idx, p.E, kBoundsLlr)) s += __ldg(in + idx);
  }
  return s;
}

// CRC remainder contribution of one hard bit: T[B-1-i] if bit i is set.
__device__ __forceinline__ uint32_t crc_term(const DecodeParams& p, int i) {
  return NRLDPC_INBOUNDS(p.B - 1 - i, kMaxB, kBoundsCrc) ? __ldg(p.crc_tab + (p.B - 1 - i)) : 0u;
}

}  // namespace nrldpc
