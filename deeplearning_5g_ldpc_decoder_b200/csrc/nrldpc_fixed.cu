// nrldpc_fixed.cu — fixed-point layered min-sum decoder (algos 1, 2, 3) for sm_100a.
//
// Semantics: bit-exact restatement of the reference's int16 layered min-sum
// (c_lib/fixedpoint_ldpc_decoder.c:103-222; the trained-table and degree
// variants c_lib/neural_fixedpoint_ldpc_decoder.c:223-281 and
// c_lib/degree_fixedpoint_ldpc_decoder.c:379-447 differ only in where alpha
// and beta come from, which the host resolves into a per-(iteration, row)
// table).
//
// Mapping (B200-first, not the reference's <<<1, Zc>>> launch):
//  * Two code blocks of the same (BG, Zc) are interleaved as int16x2 in every
//    32-bit word, so each check-node step is one packed dual-int16 SIMD op for
//    both code blocks (__vsub2 / __vmaxs2 / __vibmin_u16x2 / __vadd2 ..., see
//    nrldpc_fixed_row.cuh).
//  * Lifted row zx of every layer is owned by one thread; a CTA holds G pairs
//    (up to floor(384 / Zc); fewer when a small batch is spread over the SMs)
//    so small lifting sizes still fill the CTA.
//  * The beliefs LQ of all G pairs live in shared memory for the whole decode.
//    Circulant shifts are resolved as shared-memory word addresses
//    col*Zc + (V_ij mod Zc + zx) mod Zc.
//  * Check-to-variable messages are kept compressed per lifted check row and
//    pair (two scaled minima, the position of the minimum, one sign bit per
//    edge: 16 or 20 bytes for both code blocks instead of 4*degree) in a
//    per-CTA global scratch that stays resident in L2.
//  * The grid is persistent.  With a block cursor (DecodeParams::cursor: the
//    queue head and a count of finished CTAs, both zero at launch and rewound
//    by the last CTA to finish) every int16 half lane takes code blocks from one
//    device queue: as soon as its block passes the CRC or reaches
//    max_iterations the block's outputs are written and the half lane
//    restarts on the next block (zero messages through the `fresh` mask, its
//    own iteration count), so each block costs its own iterations.  Without a
//    cursor (launches of one wave or less, and the no-allocation entry point)
//    each CTA loops over fixed work items of G pairs until every block of the
//    item has finished.
//  * Each row's compressed message words are loaded while the row before it
//    computes (load_row_msg), hiding their L2 latency.
//  * Per-layer descriptors (scratch offset, first edge, degree, plane count,
//    alpha|beta) are staged in shared memory at kernel start: one 16-byte
//    shared load per layer replaces six dynamically indexed parameter reads.
//  * CRC early termination runs every iteration inside the kernel: each hard
//    bit i contributes x^(B-1-i+W) mod g(x) (a precomputed table), the
//    contributions are XOR-reduced with warp reductions and shared atomics.
#include <cuda_runtime.h>
#include <stdint.h>

#include "nrldpc_decode_common.cuh"
#include "nrldpc_fixed_row.cuh"
#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

using namespace fixedrow;


// Write the results of code block `cw` (half h of the pair in `lq`) using the
// Zc threads of its group.
__device__ void emit_block(const DecodeParams& p, const uint32_t* lq, int zx, int cw, int h, int status,
                           int iters) {
  const int shift = 16 * h;
  if (iters > 0 && p.bits) {
    const int nbytes = (p.B + 7) >> 3;
    uint8_t* out = p.bits + (int64_t)cw * p.bits_stride;
    for (int byte = zx; byte < nbytes; byte += p.Zc) {
      uint32_t v = 0u;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int i = byte * 8 + b;
        const uint32_t bit = i < p.B ? (lq[i] >> (shift + 15)) & 1u : 0u;
        v = (v << 1) | bit;
      }
      out[byte] = (uint8_t)v;
    }
  }
  if (p.app) {
    int16_t* out = reinterpret_cast<int16_t*>(p.app) + (int64_t)cw * p.app_stride;
    for (int i = zx; i < p.lq_len; i += p.Zc) out[i] = (int16_t)(lq[i] >> shift);
  }
  if (zx == 0) {
    if (p.status) p.status[cw] = status;
    if (p.iters) p.iters[cw] = iters;
  }
}

// XOR of the warp's partial remainders of slot gg into s_crc.
__device__ __forceinline__ void crc_flush(uint32_t* s_crc, int gg, uint32_t r0, uint32_t r1) {
  r0 = __reduce_xor_sync(0xFFFFFFFFu, r0);
  r1 = __reduce_xor_sync(0xFFFFFFFFu, r1);
  if ((threadIdx.x & 31) == 0) {
    if (r0) atomicXor(&s_crc[2 * gg], r0);
    if (r1) atomicXor(&s_crc[2 * gg + 1], r1);
  }
}

// Hard decisions + CRC remainder of both halves of every group into s_crc
// (zero for a block whose CRC passes).
// With B a multiple of 4 each thread takes four consecutive positions per
// step: one 16-byte shared load of their LQ words and one 16-byte load of
// their table entries T[B-4-i0 .. B-1-i0] (16-byte aligned because B and i0
// are multiples of 4 and each type's table starts 16-byte aligned), and per
// position one sign mask and one three-input XOR-AND per half.  A slot spans
// Bq = roundup(B, 128) positions, so a warp's 32 steps (128 positions) share
// one slot and the warp reduces once per slot.  Otherwise one position per
// step over Bp = roundup(B, 32) positions per slot.
__device__ __forceinline__ void crc_pass(const DecodeParams& p, const uint32_t* s_lq, uint32_t* s_crc) {
  uint32_t r0 = 0u, r1 = 0u;
  int cur = -1;
  if ((p.B & 3) == 0) {
    const int Bq4 = ((p.B + 127) & ~127) >> 2;   // four-position steps per slot
    const uint32_t magic = bp_magic(Bq4);
    for (int k = threadIdx.x; k < p.G * Bq4; k += blockDim.x) {
      const int gg = div_bp(k, magic);
      if (gg != cur) {
        if (cur >= 0) crc_flush(s_crc, cur, r0, r1);
        r0 = r1 = 0u;
        cur = gg;
      }
      const int i0 = 4 * (k - gg * Bq4);
      if (i0 < p.B && NRLDPC_INBOUNDS(p.B - 1 - i0, kMaxB, kBoundsCrc)) {   // i0 + 4 <= B
        const uint4 w = *reinterpret_cast<const uint4*>(s_lq + gg * p.lq_len + i0);
        const uint4 t = __ldg(reinterpret_cast<const uint4*>(p.crc_tab + (p.B - 4 - i0)));
        // position i0 + j pairs with T[B-1-i0-j]: t.w, t.z, t.y, t.x
        r0 ^= (t.w & sign_of_byte1(w.x)) ^ (t.z & sign_of_byte1(w.y)) ^ (t.y & sign_of_byte1(w.z)) ^
              (t.x & sign_of_byte1(w.w));
        r1 ^= (t.w & sign_of_byte3(w.x)) ^ (t.z & sign_of_byte3(w.y)) ^ (t.y & sign_of_byte3(w.z)) ^
              (t.x & sign_of_byte3(w.w));
      }
    }
  } else {
    const int Bp = (p.B + 31) & ~31;
    const uint32_t magic = bp_magic(Bp);
    for (int k = threadIdx.x; k < p.G * Bp; k += blockDim.x) {
      const int gg = div_bp(k, magic);
      if (gg != cur) {
        if (cur >= 0) crc_flush(s_crc, cur, r0, r1);
        r0 = r1 = 0u;
        cur = gg;
      }
      const int i = k - gg * Bp;
      if (i < p.B) {
        const uint32_t w = s_lq[gg * p.lq_len + i];
        const uint32_t tv = crc_term(p, i);
        r0 ^= tv & sign_of_byte1(w);
        r1 ^= tv & sign_of_byte3(w);
      }
    }
  }
  if (cur >= 0) crc_flush(s_crc, cur, r0, r1);
}

// Rate recovery into the halves of the group's LQ words selected by r0 / r1
// (half h gets code block cw_h, zeros when cw_h < 0), with the soft buffers;
// the other half keeps its bits.  One pass for both halves.
__device__ __forceinline__ void recover_halves(const DecodeParams& p, uint32_t* lq, int zx, int cw0, int cw1,
                                               bool r0, bool r1) {
  const uint32_t keep = (r0 ? 0u : 0x0000FFFFu) | (r1 ? 0u : 0xFFFF0000u);
  const bool v0 = r0 && cw0 >= 0, v1 = r1 && cw1 >= 0;
  const int16_t* in0 = p.llr + (int64_t)(v0 ? cw0 : 0) * p.llr_stride;
  const int16_t* in1 = p.llr + (int64_t)(v1 ? cw1 : 0) * p.llr_stride;
  int16_t* h0 = (p.harq && v0) ? p.harq + (int64_t)cw0 * p.harq_stride : nullptr;
  int16_t* h1 = (p.harq && v1) ? p.harq + (int64_t)cw1 * p.harq_stride : nullptr;
  for (int i = zx; i < p.lq_len; i += p.Zc) {
    uint32_t w = keep ? (lq[i] & keep) : 0u;
    if (v0) {
      const int32_t a = recover_position(p, in0, i, (p.harq_on && h0) ? h0[i] : 0);
      if (h0) h0[i] = (int16_t)a;
      w |= (uint32_t)a & 0xFFFFu;
    }
    if (v1) {
      const int32_t a = recover_position(p, in1, i, (p.harq_on && h1) ? h1[i] : 0);
      if (h1) h1[i] = (int16_t)a;
      w |= (uint32_t)a << 16;
    }
    lq[i] = w;
  }
}

// Next code blocks of the queue for the half lanes that ask (q0 / q1: this
// thread asks for half 0 / half 1), one atomic per warp.  Called by whole
// warps; returns -1 past the end of the queue.
__device__ __forceinline__ void take_blocks(const DecodeParams& p, bool q0, bool q1, int* cw0, int* cw1) {
  const unsigned b0 = __ballot_sync(0xFFFFFFFFu, q0);
  const unsigned b1 = __ballot_sync(0xFFFFFFFFu, q1);
  const int n0 = __popc(b0), total = n0 + __popc(b1);
  if (total == 0) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(b0 | b1) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(p.cursor, total);
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  const unsigned lt = (1u << lane) - 1u;
  if (q0) {
    const int i = base + __popc(b0 & lt);
    *cw0 = i < p.num_cw ? i : -1;
  }
  if (q1) {
    const int i = base + n0 + __popc(b1 & lt);
    *cw1 = i < p.num_cw ? i : -1;
  }
}

// kG1: one lane pair per CTA (G = 1: Zc >= 193, or a batch small enough to
// give every pair its own CTA), so the group index and its
// shared-memory base are compile-time zeros and free registers in the layer loop.
template <int kClip, bool kRefill, bool kG1>
__global__ void __launch_bounds__(kThreadsTarget, 2) fixed_pair_kernel(const __grid_constant__ DecodeParams p) {
  extern __shared__ __align__(16) uint32_t s_lq[];        // [G][lq_len] int16x2
  __shared__ uint32_t s_crc[2 * kMaxGroups];
  __shared__ uint2 s_edges[kMaxNnz];   // per-edge (col*Zc*4, (V mod Zc)*4), read with warp-uniform indices
  __shared__ uint4 s_rows[kMaxRows];   // per-layer descriptors (row_descriptor)
  for (int e = threadIdx.x; e < kMaxNnz; e += blockDim.x) s_edges[e] = p.edge_cs4[e];
  for (int r = threadIdx.x; r < p.R; r += blockDim.x) s_rows[r] = row_descriptor(p, r);

  const int tid = threadIdx.x;
  const int g = kG1 ? 0 : tid / p.Zc;
  const int zx = kG1 ? tid : tid - g * p.Zc;
  const bool active = kG1 ? tid < p.Zc : g < p.G;
  uint32_t* lq = s_lq + (active ? g : 0) * p.lq_len;
  uint32_t* scratch = p.scratch + (int64_t)blockIdx.x * p.scratch_words;
  // debug build: every message word of the CTA (planes of kThreadsTarget words,
  // ending at lr_off[R]) lies inside its scratch
  if (!NRLDPC_INBOUNDS(p.lr_off[p.R] - 1u, p.scratch_words, kBoundsScratch) ||
      !NRLDPC_INBOUNDS(blockDim.x - 1u, kThreadsTarget, kBoundsScratch))
    return;
  const uint32_t zx4 = 4u * (uint32_t)zx;
  const uint32_t zxm4 = zx4 - 4u * (uint32_t)p.Zc;     // wraps: min(zx4+s, zxm4+s) = ((zx+V) mod Zc)*4
  const uint32_t gb4 = kG1 ? 0u : 4u * (uint32_t)((active ? g : 0) * p.lq_len);
  const uint32_t lq_limit = 4u * (uint32_t)(p.G * p.lq_len);   // bytes of s_lq in use

  if constexpr (kRefill) {
    __shared__ int s_cw[2 * kMaxGroups];   // block in each half lane, -1 when idle
    __shared__ int s_base;
    // The half lanes' blocks live in s_cw, not in registers: the layer loop
    // needs every register it can get.
    if (tid == 0) s_base = atomicAdd(p.cursor, 2 * p.G);
    __syncthreads();
    if (active && zx == 0) {
      s_cw[2 * g] = s_base + 2 * g < p.num_cw ? s_base + 2 * g : -1;
      s_cw[2 * g + 1] = s_base + 2 * g + 1 < p.num_cw ? s_base + 2 * g + 1 : -1;
    }
    __syncthreads();
    bool idle;
    {
      const int c0 = active ? s_cw[2 * g] : -1, c1 = active ? s_cw[2 * g + 1] : -1;
      if (active && !p.rr_scatter) recover_halves(p, lq, zx, c0, c1, true, true);
      if (p.rr_scatter) recover_scatter(p, lq, zx, active, c0, c1, true, true);
      if (tid < 2 * kMaxGroups) s_crc[tid] = 0u;
      idle = __syncthreads_and(!active || (c0 < 0 && c1 < 0));
    }
    uint32_t itv = 0u;   // iterations of half 0 in bits 0-15, half 1 in bits 16-31
    uint32_t fresh = 0xFFFFFFFFu;   // both halves start their first iteration
    const bool run = p.max_it > 0;   // max_iterations == 0: rate recovery only, status 1
    RowMsg nxt{};
    while (!idle) {
      for (int row = 0; run && row < p.R; ++row) {
        if (active) {
          const RowMsg cur = nxt;
          const uint4 d = s_rows[row];
          const int rn = row + 1 < p.R ? row + 1 : 0;
          const uint2 dn = *reinterpret_cast<const uint2*>(&s_rows[rn]);
          nxt = load_row_msg(scratch + dn.x + tid, row_five(dn.y));
          uint32_t ab0, ab1;
          if (p.weights_T > 0) {
            ab0 = __ldg(p.weights + (min((int)(itv & 0xFFFFu), p.weights_T - 1) * p.R + row));
            ab1 = __ldg(p.weights + (min((int)(itv >> 16), p.weights_T - 1) * p.R + row));
          } else {
            ab0 = ab1 = d.z;
          }
          layer_dispatch<kClip, true, kG1>(row_deg(d.y), p, s_edges, reinterpret_cast<char*>(s_lq), zx4, zxm4, gb4,
                                           lq_limit, row_e0(d.y), (int32_t)(int16_t)(ab0 & 0xFFFFu), ((int32_t)ab0) >> 16,
                                           (int32_t)(int16_t)(ab1 & 0xFFFFu), ((int32_t)ab1) >> 16, cur, fresh,
                                           scratch + d.x + tid);
        }
        __syncthreads();
      }
      fresh = 0u;
      if (run) crc_pass(p, s_lq, s_crc);
      __syncthreads();
      bool fin[2] = {false, false};
      if (active) {
        for (int h = 0; h < 2; ++h) {
          const int c = s_cw[2 * g + h];
          if (c < 0) continue;
          if (run) itv += h ? 0x10000u : 1u;
          const int ith = (int)(h ? itv >> 16 : itv & 0xFFFFu);
          const bool pass = run && s_crc[2 * g + h] == 0u;
          if (pass || ith >= p.max_it) {
            emit_block(p, lq, zx, c, h, pass ? 0 : 1, ith);
            fin[h] = true;
          }
        }
      }
      // s_crc read and the finished blocks emitted before anything is reused
      const bool any = __syncthreads_or(fin[0] || fin[1]);
      if (tid < 2 * kMaxGroups) s_crc[tid] = 0u;
      if (!any) continue;
      int nc0 = -1, nc1 = -1;
      take_blocks(p, fin[0] && zx == 0, fin[1] && zx == 0, &nc0, &nc1);
      if (zx == 0) {
        if (fin[0]) s_cw[2 * g] = nc0;
        if (fin[1]) s_cw[2 * g + 1] = nc1;
      }
      __syncthreads();
      const int c0 = active ? s_cw[2 * g] : -1, c1 = active ? s_cw[2 * g + 1] : -1;
      if (active && (fin[0] || fin[1])) {
        for (int h = 0; h < 2; ++h) {
          if (!fin[h]) continue;
          itv &= h ? 0x0000FFFFu : 0xFFFF0000u;
          if ((h ? c1 : c0) >= 0) fresh |= h ? 0xFFFF0000u : 0x0000FFFFu;
        }
        if (!p.rr_scatter) recover_halves(p, lq, zx, c0, c1, fin[0], fin[1]);
      }
      // `any` is uniform here, so every thread of the CTA reaches the barriers inside
      if (p.rr_scatter) recover_scatter(p, lq, zx, active, c0, c1, fin[0], fin[1]);
      idle = __syncthreads_and(!active || (c0 < 0 && c1 < 0));
    }
    // Every take of this CTA is done (the last barrier above).  The CTA that
    // finishes last rewinds the queue for the next launch on the stream.
    if (tid == 0) {
      __threadfence();
      if (atomicAdd(p.cursor + 1, 1) == (int)gridDim.x - 1) {
        atomicExch(p.cursor, 0);
        atomicExch(p.cursor + 1, 0);
      }
    }
  } else {
    for (int item = blockIdx.x; item < p.num_items; item += gridDim.x) {
      const int pair = item * p.G + g;
      const int cw0 = 2 * pair, cw1 = 2 * pair + 1;
      const bool v0 = active && cw0 < p.num_cw;
      const bool v1 = active && cw1 < p.num_cw;

      // ---- rate recovery into LQ (and the soft buffers) ----
      if (p.rr_scatter) recover_scatter(p, lq, zx, active, v0 ? cw0 : -1, v1 ? cw1 : -1, true, true);
      if (active && !p.rr_scatter) {
        const int16_t* in0 = p.llr + (int64_t)(v0 ? cw0 : 0) * p.llr_stride;
        const int16_t* in1 = p.llr + (int64_t)(v1 ? cw1 : 0) * p.llr_stride;
        int16_t* h0 = (p.harq && v0) ? p.harq + (int64_t)cw0 * p.harq_stride : nullptr;
        int16_t* h1 = (p.harq && v1) ? p.harq + (int64_t)cw1 * p.harq_stride : nullptr;
        for (int i = zx; i < p.lq_len; i += p.Zc) {
          int32_t a0 = 0, a1 = 0;
          if (p.harq_on) {
            if (h0) a0 = h0[i];
            if (h1) a1 = h1[i];
          }
          a0 = v0 ? recover_position(p, in0, i, a0) : 0;
          a1 = v1 ? recover_position(p, in1, i, a1) : 0;
          if (h0) h0[i] = (int16_t)a0;
          if (h1) h1[i] = (int16_t)a1;
          lq[i] = ((uint32_t)a0 & 0xFFFFu) | ((uint32_t)a1 << 16);
        }
      }
      if (tid < 2 * kMaxGroups) s_crc[tid] = 0u;
      // Padding slots count as finished so they never hold the CTA back.
      bool done0 = !v0, done1 = !v1;
      __syncthreads();

      int it = 0;
      RowMsg nxt{};
      for (; it < p.max_it; ++it) {
        for (int row = 0; row < p.R; ++row) {
          if (active) {
            const RowMsg cur = nxt;
            const uint4 d = s_rows[row];
            const int rn = row + 1 < p.R ? row + 1 : 0;
            const uint2 dn = *reinterpret_cast<const uint2*>(&s_rows[rn]);
            nxt = load_row_msg(scratch + dn.x + tid, row_five(dn.y));
            const uint32_t ab = p.weights_T > 0 ? __ldg(p.weights + (min(it, p.weights_T - 1) * p.R + row)) : d.z;
            const int32_t alpha = (int32_t)(int16_t)(ab & 0xFFFFu);
            const int32_t beta = ((int32_t)ab) >> 16;
            layer_dispatch<kClip, true, kG1>(row_deg(d.y), p, s_edges, reinterpret_cast<char*>(s_lq), zx4, zxm4, gb4,
                                             lq_limit, row_e0(d.y), alpha, beta, alpha, beta, cur,
                                             it == 0 ? 0xFFFFFFFFu : 0u, scratch + d.x + tid);
          }
          __syncthreads();
        }

        // ---- hard decisions + CRC of every code block in the CTA ----
        crc_pass(p, s_lq, s_crc);
        __syncthreads();
        bool pass0 = false, pass1 = false;
        if (active) {
          pass0 = !done0 && s_crc[2 * g] == 0u;
          pass1 = !done1 && s_crc[2 * g + 1] == 0u;
          if (pass0) emit_block(p, lq, zx, cw0, 0, 0, it + 1);
          if (pass1) emit_block(p, lq, zx, cw1, 1, 0, it + 1);
          done0 = done0 || pass0;
          done1 = done1 || pass1;
        }
        // Everyone has read s_crc before it is cleared for the next iteration.
        const bool all_done = __syncthreads_and(done0 && done1);
        if (tid < 2 * kMaxGroups) s_crc[tid] = 0u;
        if (all_done) {
          ++it;
          break;
        }
      }
      if (active) {
        if (!done0) emit_block(p, lq, zx, cw0, 0, 1, it);
        if (!done1) emit_block(p, lq, zx, cw1, 1, 1, it);
      }
      __syncthreads();   // LQ and s_crc are reused by the next work item
    }
  }
}

template <int kClip, bool kRefill, bool kG1>
int launch_fixed_t(const DecodeParams& p, int grid, int block, int smem, cudaStream_t s) {
  static std::atomic<uint32_t> attr_done{0};
  const int err = raise_smem_limit_once(fixed_pair_kernel<kClip, kRefill, kG1>, &attr_done);
  if (err != 0) return err;
  fixed_pair_kernel<kClip, kRefill, kG1><<<grid, block, smem, s>>>(p);
  return (int)cudaSuccess;
}

template <int kClip>
int launch_fixed_c(const DecodeParams& p, int grid, int block, int smem, cudaStream_t s) {
  const bool refill = p.cursor != nullptr;
  if (p.G == 1)   // one-pair specialisation
    return refill ? launch_fixed_t<kClip, true, true>(p, grid, block, smem, s)
                  : launch_fixed_t<kClip, false, true>(p, grid, block, smem, s);
  return refill ? launch_fixed_t<kClip, true, false>(p, grid, block, smem, s)
                : launch_fixed_t<kClip, false, false>(p, grid, block, smem, s);
}

template <int kClip, bool kRefill>
int occupancy_fixed_t(int block, int smem) {
  int n = 0;
  static std::atomic<uint32_t> attr_done{0};
  if (raise_smem_limit_once(fixed_pair_kernel<kClip, kRefill, false>, &attr_done) != 0) return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fixed_pair_kernel<kClip, kRefill, false>, block, smem);
  return n;
}

}  // namespace

int launch_fixed(const DecodeParams& p, int grid, int block, int smem, int clip_mode, void* stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int err;
  switch (clip_mode) {
    case kClipDegen: err = launch_fixed_c<kClipDegen>(p, grid, block, smem, s); break;
    case kClipOpenMax: err = launch_fixed_c<kClipOpenMax>(p, grid, block, smem, s); break;
    default: err = launch_fixed_c<kClipClamp>(p, grid, block, smem, s); break;
  }
  if (err != (int)cudaSuccess) return err;
  count_launch();
  return (int)cudaGetLastError();
}

int bounds_read_fixed(uint32_t* out, bool reset) { return bounds_read_tu(out, reset); }

int occupancy_fixed(int block, int smem, int clip_mode, bool refill) {
  switch (clip_mode) {
    case kClipDegen: return refill ? occupancy_fixed_t<kClipDegen, true>(block, smem) : occupancy_fixed_t<kClipDegen, false>(block, smem);
    case kClipOpenMax:
      return refill ? occupancy_fixed_t<kClipOpenMax, true>(block, smem) : occupancy_fixed_t<kClipOpenMax, false>(block, smem);
    default: return refill ? occupancy_fixed_t<kClipClamp, true>(block, smem) : occupancy_fixed_t<kClipClamp, false>(block, smem);
  }
}

}  // namespace nrldpc
