// nrldpc_mixed.cu — one persistent fixed-point decode kernel for batches that
// mix base graphs, lifting sizes, rates, modulations, redundancy versions and
// CRC types (algos 1, 2, 3).
//
// Same arithmetic as the uniform kernel (nrldpc_fixed_row.cuh, bit-exact with
// c_lib/fixedpoint_ldpc_decoder.c).  Differences:
//  * work items (G pairs of one (BG, Zc)) come from a device work queue
//    (atomic counter), so CTAs stay busy whatever the size mix;
//  * the item's base-graph tables (per-edge shared-memory offsets, row offsets,
//    scratch layout) are staged into shared memory per item;
//  * the two code blocks of a pair share (BG, Zc) but may differ in every other
//    parameter: rate recovery, the CRC check and the outputs use each block's
//    own B, E, Qm, rv and CRC type.
#include <cuda_runtime.h>
#include <stdint.h>

#include "nrldpc_fixed_row.cuh"
#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

using namespace fixedrow;

// Rate recovery of soft-buffer position i of one block (c_lib/ldpc_rate_recovery.c:24-65,
// gather form; see recover_position in nrldpc_decode_common.cuh), starting from
// `init` (the stored soft buffer when combining a retransmission).  With a
// limited circular buffer (ncb < N) positions at or beyond ncb take no coded
// bits and the compacted buffer has ncb - F positions (TS 38.212 5.4.2.1).
__device__ __forceinline__ int32_t mixed_recover(const MixedGraph& g, const MixedCw& c, const int16_t* __restrict__ in,
                                                 int i, int32_t fill, int32_t init) {
  const int twoZ = 2 * g.Zc;
  if (i >= c.B && i < g.K) return fill;
  int32_t s = init;
  if (i < twoZ) return s;
  const int pos = i - twoZ;
  if (pos >= c.ncb) return s;
  const int cc = pos < c.B - twoZ ? pos : pos - c.F;
  int kf = cc - c.c0;
  if (kf < 0) kf += c.Nv;
  for (int k = kf; k < c.E; k += c.Nv) {
    const int b = k / c.symbols;
    const int sidx = k - b * c.symbols;
    s += __ldg(in + (int64_t)sidx * c.Qm + b);
  }
  return s;
}

__device__ void mixed_emit(const MixedParams& p, const uint32_t* lq, int zx, int Zc, int cw, const MixedCw& c, int h,
                           int status, int iters) {
  const int shift = 16 * h;
  if (iters > 0 && p.bits) {
    const int nbytes = (c.B + 7) >> 3;
    uint8_t* out = p.bits + c.bits_off;
    for (int byte = zx; byte < nbytes; byte += Zc) {
      uint32_t v = 0u;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int i = byte * 8 + b;
        v = (v << 1) | (i < c.B ? (lq[i] >> (shift + 15)) & 1u : 0u);
      }
      out[byte] = (uint8_t)v;
    }
  }
  if (zx == 0) {
    if (p.status) p.status[cw] = status;
    if (p.iters) p.iters[cw] = iters;
  }
}

template <bool kDegenClip>
__global__ void __launch_bounds__(kThreadsTarget, 2) fixed_mixed_kernel(const __grid_constant__ MixedParams p) {
  extern __shared__ __align__(16) uint32_t s_lq[];
  __shared__ uint32_t s_crc[2 * kMaxGroups];
  __shared__ MixedGraph s_g;
  __shared__ int4 s_grp[kMaxGroups];      // per pair: B0, B1, CRC table offsets of both halves
  __shared__ int s_item;

  const int tid = threadIdx.x;
  uint32_t* scratch = p.scratch + (int64_t)blockIdx.x * p.scratch_words;
  const int num_items = p.num_items_dev ? *p.num_items_dev : p.num_items;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(p.counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= num_items) break;
    const MixedItem desc = p.items[item];
    {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(p.graphs + desc.graph);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&s_g);
      for (int w = tid; w < (int)(sizeof(MixedGraph) / 4); w += blockDim.x) dst[w] = __ldg(src + w);
    }
    __syncthreads();
    const int Zc = s_g.Zc, G = s_g.G, lq_len = s_g.lq_len;
    const int g = tid / Zc;
    const int zx = tid - g * Zc;
    const bool active = g < G;
    uint32_t* lq = s_lq + (active ? g : 0) * lq_len;
    const int cw0 = active ? p.slots[desc.slot_base + 2 * g] : -1;
    const int cw1 = active ? p.slots[desc.slot_base + 2 * g + 1] : -1;
    const bool v0 = cw0 >= 0, v1 = cw1 >= 0;
    MixedCw c0 = {}, c1 = {};
    if (v0) c0 = p.cws[cw0];
    if (v1) c1 = p.cws[cw1];
    if (active && zx == 0)
      s_grp[g] = make_int4(v0 ? c0.B : 0, v1 ? c1.B : 0, c0.crctype * kMaxB, c1.crctype * kMaxB);

    if (active) {
      const int16_t* in0 = p.llr + c0.llr_off;
      const int16_t* in1 = p.llr + c1.llr_off;
      int16_t* h0 = (v0 && c0.harq_mode && p.harq) ? p.harq + c0.harq_off : nullptr;
      int16_t* h1 = (v1 && c1.harq_mode && p.harq) ? p.harq + c1.harq_off : nullptr;
      for (int i = zx; i < lq_len; i += Zc) {
        const int32_t i0 = (h0 && (c0.harq_mode & 1)) ? h0[i] : 0;
        const int32_t i1 = (h1 && (c1.harq_mode & 1)) ? h1[i] : 0;
        const int32_t a0 = v0 ? mixed_recover(s_g, c0, in0, i, p.fill, i0) : 0;
        const int32_t a1 = v1 ? mixed_recover(s_g, c1, in1, i, p.fill, i1) : 0;
        if (h0 && (c0.harq_mode & 2)) h0[i] = (int16_t)a0;
        if (h1 && (c1.harq_mode & 2)) h1[i] = (int16_t)a1;
        lq[i] = ((uint32_t)a0 & 0xFFFFu) | ((uint32_t)a1 << 16);
      }
    }
    if (tid < 2 * kMaxGroups) s_crc[tid] = 0u;
    bool done0 = !v0, done1 = !v1;
    __syncthreads();

    const int bi = s_g.bgn == 1 ? 0 : 1;
    const uint32_t zx4 = 4u * (uint32_t)zx;
    const uint32_t zxm4 = zx4 - 4u * (uint32_t)Zc;
    const uint32_t gb4 = 4u * (uint32_t)((active ? g : 0) * lq_len);
    const int Bp = desc.bmax_pad;
    int it = 0;
    for (; it < p.max_it; ++it) {
      for (int row = 0; row < s_g.R; ++row) {
        if (active) {
          const int e0 = s_g.row_off[row];
          const int deg = s_g.row_off[row + 1] - e0;
          const uint32_t ab = p.weights_T[bi] > 0
                                  ? __ldg(p.weights[bi] + (min(it, p.weights_T[bi] - 1) * s_g.R + row))
                                  : p.w_inline[bi][row];
          const int32_t alpha = (int32_t)(int16_t)(ab & 0xFFFFu);
          const int32_t beta = ((int32_t)ab) >> 16;
          layer_dispatch<kDegenClip, true>(deg, p, s_g.edges, reinterpret_cast<char*>(s_lq), zx4, zxm4, gb4, e0, alpha,
                                           beta, it == 0, scratch + s_g.lr_off[row] + tid);
        }
        __syncthreads();
      }
      // Hard decisions + CRC of both halves of every pair (each with its own B and CRC type).
      for (int k = tid; k < G * Bp; k += blockDim.x) {
        const int gg = k / Bp;
        const int i = k - gg * Bp;
        const int4 gr = s_grp[gg];
        uint32_t r0 = 0u, r1 = 0u;
        const uint32_t w = i < lq_len ? s_lq[gg * lq_len + i] : 0u;
        if (i < gr.x && (w & 0x8000u)) r0 = __ldg(p.crc_tab + gr.z + (gr.x - 1 - i));
        if (i < gr.y && (w & 0x80000000u)) r1 = __ldg(p.crc_tab + gr.w + (gr.y - 1 - i));
        r0 = __reduce_xor_sync(0xFFFFFFFFu, r0);
        r1 = __reduce_xor_sync(0xFFFFFFFFu, r1);
        if ((tid & 31) == 0) {
          if (r0) atomicXor(&s_crc[2 * gg], r0);
          if (r1) atomicXor(&s_crc[2 * gg + 1], r1);
        }
      }
      __syncthreads();
      if (active) {
        const bool pass0 = !done0 && s_crc[2 * g] == 0u;
        const bool pass1 = !done1 && s_crc[2 * g + 1] == 0u;
        if (pass0) mixed_emit(p, lq, zx, Zc, cw0, c0, 0, 0, it + 1);
        if (pass1) mixed_emit(p, lq, zx, Zc, cw1, c1, 1, 0, it + 1);
        done0 = done0 || pass0;
        done1 = done1 || pass1;
      }
      const bool all_done = __syncthreads_and(done0 && done1);
      if (tid < 2 * kMaxGroups) s_crc[tid] = 0u;
      if (all_done) {
        ++it;
        break;
      }
    }
    if (active) {
      if (!done0) mixed_emit(p, lq, zx, Zc, cw0, c0, 0, 1, it);
      if (!done1) mixed_emit(p, lq, zx, Zc, cw1, c1, 1, 1, it);
    }
    __syncthreads();   // shared state is reused by the next item
  }
}

}  // namespace

int launch_mixed(const MixedParams& p, int grid, bool degen_clip, void* stream) {
  const int smem = kThreadsTarget * kMaxCols * 4;   // largest G * (N + 2Zc) words of any (BG, Zc)
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t err;
  if (degen_clip) {
    err = cudaFuncSetAttribute(fixed_mixed_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (err != cudaSuccess) return (int)err;
    fixed_mixed_kernel<true><<<grid, kThreadsTarget, smem, s>>>(p);
  } else {
    err = cudaFuncSetAttribute(fixed_mixed_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (err != cudaSuccess) return (int)err;
    fixed_mixed_kernel<false><<<grid, kThreadsTarget, smem, s>>>(p);
  }
  count_launch();
  return (int)cudaGetLastError();
}

int prepare_mixed(bool degen_clip) {
  const int smem = kThreadsTarget * kMaxCols * 4;
  cudaError_t err = degen_clip
                        ? cudaFuncSetAttribute(fixed_mixed_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
                        : cudaFuncSetAttribute(fixed_mixed_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  return (int)err;
}

int occupancy_mixed(bool degen_clip) {
  const int smem = kThreadsTarget * kMaxCols * 4;
  int n = 0;
  prepare_mixed(degen_clip);
  if (degen_clip) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fixed_mixed_kernel<true>, kThreadsTarget, smem);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fixed_mixed_kernel<false>, kThreadsTarget, smem);
  }
  return n;
}

}  // namespace nrldpc
