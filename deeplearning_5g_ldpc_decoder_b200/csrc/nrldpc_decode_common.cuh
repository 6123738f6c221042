// nrldpc_decode_common.cuh — device helpers shared by the decode kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "nrldpc_bounds.cuh"
#include "nrldpc_internal.h"

namespace nrldpc {

// Largest dynamic shared memory of a decode launch: G * (N + 2Zc) words with
// G * Zc <= 384 lifted rows, i.e. 384 * 68 words.
constexpr int kMaxDecodeSmem = kThreadsTarget * kMaxCols * 4;

// Set a decode kernel's dynamic shared-memory limit to `limit` (by default
// kMaxDecodeSmem, at least what any of its launches asks for) once per device;
// `done` holds one bit per device, per kernel.  The limit is never lowered, so
// launches and occupancy queries of any size can share it, and the attribute
// call is not paid on every launch.
template <typename K>
int raise_smem_limit_once(K kernel, std::atomic<uint32_t>* done, int limit = kMaxDecodeSmem) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  const uint32_t bit = dev < 32 ? 1u << dev : 0u;
  if (bit && (done->load(std::memory_order_acquire) & bit)) return 0;
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
  if (e != cudaSuccess) return (int)e;
  if (bit) done->fetch_or(bit, std::memory_order_release);
  return 0;
}

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

// Soft-buffer position of rate-matched LLR e (the inverse of the gather form
// above, for E <= Nv where every LLR lands on its own position): symbol
// s = e / Qm and bit b = e mod Qm give k = b (E/Qm) + s (the de-interleave of
// c_lib/ldpc_rate_recovery.c:47-64), compact position (c0 + k) mod Nv, then the
// filler gap and the 2Zc punctured columns.
// e / Qm for e < 2^16, Qm in {1, 2, 4, 6, 8}: the high word of e * ceil(2^32 / Qm).
// For Qm = 1 that constant is 2^32, which does not fit 32 bits: the quotient is e.
__device__ __forceinline__ uint32_t div_qm(uint32_t e, uint32_t qm, uint32_t magic) {
  return qm == 1u ? e : __umulhi(e, magic);
}

__device__ __forceinline__ int scatter_position(const DecodeParams& p, uint32_t e) {
  const uint32_t s = div_qm(e, (uint32_t)p.Qm, p.qm_magic);
  const uint32_t b = e - s * (uint32_t)p.Qm;
  int c = p.c0 + (int)(b * (uint32_t)p.symbols + s);
  c -= c >= p.Nv ? p.Nv : 0;
  const int twoZ = 2 * p.Zc;
  return (c < p.B - twoZ ? c : c + p.F) + twoZ;
}

// Rate recovery of the halves of the group's LQ words selected by r0 / r1
// (half h gets code block cw_h, zeros when cw_h < 0), with the soft buffers;
// the other half keeps its bits.  Scatter form for E <= Nv: (A) every position
// starts from its base value (filler, else the stored soft buffer with HARQ_on,
// else 0), (B) each LLR, read with coalesced 16-byte loads, is added to its own
// position (int16 wrap-around as the reference's +=), (C) the soft buffers are
// written back.  The same values as recover_position at every position.  Called
// by every thread of the CTA (it holds CTA barriers); `active` selects the
// threads that own a group.
static __device__ void recover_scatter(const DecodeParams& p, uint32_t* lq, int zx, bool active, int cw0, int cw1, bool r0,
                                bool r1) {
  const bool v0 = active && r0 && cw0 >= 0, v1 = active && r1 && cw1 >= 0;
  const uint32_t keep = (r0 ? 0u : 0x0000FFFFu) | (r1 ? 0u : 0xFFFF0000u);
  int16_t* h0 = (p.harq && v0) ? p.harq + (int64_t)cw0 * p.harq_stride : nullptr;
  int16_t* h1 = (p.harq && v1) ? p.harq + (int64_t)cw1 * p.harq_stride : nullptr;
  if (active && (r0 || r1)) {
    for (int i = zx; i < p.lq_len; i += p.Zc) {
      uint32_t w = keep ? (lq[i] & keep) : 0u;
      const bool filler = i >= p.B && i < p.K;
      if (v0) w |= (uint32_t)(uint16_t)(filler ? p.fill : (p.harq_on && h0) ? h0[i] : 0);
      if (v1) w |= (uint32_t)(uint16_t)(filler ? p.fill : (p.harq_on && h1) ? h1[i] : 0) << 16;
      lq[i] = w;
    }
  }
  __syncthreads();
  int16_t* lq16 = reinterpret_cast<int16_t*>(lq);
  for (int h = 0; h < 2; ++h) {
    if (!(h ? v1 : v0)) continue;
    const int16_t* in = p.llr + (int64_t)(h ? cw1 : cw0) * p.llr_stride;
    const uint32_t E = (uint32_t)p.E;
    uint32_t e = 8u * (uint32_t)zx;
    if (p.rr_vec) {
      for (; e + 8u <= E; e += 8u * (uint32_t)p.Zc) {
        const int4 v = __ldg(reinterpret_cast<const int4*>(in + e));
        const uint32_t w4[4] = {(uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z, (uint32_t)v.w};
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int pos = scatter_position(p, e + (uint32_t)q);
          if (NRLDPC_INBOUNDS(pos, p.lq_len, kBoundsLq)) {
            const int16_t x = (int16_t)(w4[q >> 1] >> (16 * (q & 1)));
            lq16[2 * pos + h] = (int16_t)(lq16[2 * pos + h] + x);
          }
        }
      }
    }
    for (; e < E; e += 8u * (uint32_t)p.Zc) {   // unaligned rows, and the tail of 8 LLRs
      for (uint32_t q = e; q < e + 8u && q < E; ++q) {
        const int pos = scatter_position(p, q);
        if (NRLDPC_INBOUNDS(pos, p.lq_len, kBoundsLq)) lq16[2 * pos + h] = (int16_t)(lq16[2 * pos + h] + __ldg(in + q));
      }
    }
  }
  __syncthreads();
  if (h0 || h1) {
    for (int i = zx; i < p.lq_len; i += p.Zc) {
      const uint32_t w = lq[i];
      if (h0) h0[i] = (int16_t)(w & 0xFFFFu);
      if (h1) h1[i] = (int16_t)(w >> 16);
    }
  }
}

// CRC remainder contribution of one hard bit: T[B-1-i] if bit i is set.
__device__ __forceinline__ uint32_t crc_term(const DecodeParams& p, int i) {
  return NRLDPC_INBOUNDS(p.B - 1 - i, kMaxB, kBoundsCrc) ? __ldg(p.crc_tab + (p.B - 1 - i)) : 0u;
}

// Group index k / Bp of the hard-decision loops without an integer divide:
// the multiply-high by magic = ceil(2^32 / Bp) is exact while
// k * (magic * Bp - 2^32) < 2^32.  Bp = roundup32(K) <= 8480 and
// k < G * Bp <= 14400 (G = floor(384 / Zc), K <= 22 Zc), so the product
// stays below 1.3e8.
__device__ __forceinline__ uint32_t bp_magic(int Bp) { return 0xFFFFFFFFu / (uint32_t)Bp + 1u; }
__device__ __forceinline__ int div_bp(int k, uint32_t magic) { return (int)__umulhi((uint32_t)k, magic); }

// Per-layer descriptor staged in shared memory at kernel start, one 16-byte
// load per layer instead of several dynamically indexed parameter reads:
// x = the layer's word offset in the CTA's message scratch,
// y = first edge | degree << 16 | (five message planes) << 24,
// z = the layer's packed alpha | beta << 16 (unused with per-iteration weights).
__device__ __forceinline__ uint4 row_descriptor(const DecodeParams& p, int r) {
  const uint32_t e0 = p.row_off[r], deg = (uint32_t)p.row_off[r + 1] - e0;
  const uint32_t five = p.lr_off[r + 1] - p.lr_off[r] > 4u * kThreadsTarget ? 1u : 0u;
  return make_uint4(p.lr_off[r], e0 | (deg << 16) | (five << 24), p.w_inline[r], 0u);
}
__device__ __forceinline__ int row_e0(uint32_t y) { return (int)(y & 0xFFFFu); }
__device__ __forceinline__ int row_deg(uint32_t y) { return (int)((y >> 16) & 0xFFu); }
__device__ __forceinline__ bool row_five(uint32_t y) { return (y >> 24) != 0u; }

}  // namespace nrldpc
