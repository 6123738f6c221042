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
//    both code blocks (__vsub2 / __vabsss2 / __vibmin_s16x2 / __vaddss2 ...).
//  * Lifted row zx of every layer is owned by one thread; a CTA holds G pairs
//    (G = floor(384 / Zc)) so small lifting sizes still fill the CTA.
//  * The beliefs LQ of all G pairs live in shared memory for the whole decode.
//    Circulant shifts are resolved as shared-memory word addresses
//    col*Zc + (V_ij mod Zc + zx) mod Zc.
//  * Check-to-variable messages are kept compressed per lifted check row and
//    pair (two scaled minima, the position of the minimum, one sign bit per
//    edge: 16 or 20 bytes for both code blocks instead of 4*degree) in a
//    per-CTA global scratch that stays resident in L2.
//  * The grid is persistent: each CTA loops over work items of G pairs.
//  * CRC early termination runs every iteration inside the kernel: each hard
//    bit i contributes x^(B-1-i+W) mod g(x) (a precomputed table), the
//    contributions are XOR-reduced with warp reductions and shared atomics.
//    A code block that passes stops being reported (its outputs are written at
//    that iteration); the CTA leaves the iteration loop once every code block
//    in it has passed.
#include <cuda_runtime.h>
#include <stdint.h>

#include "nrldpc_decode_common.cuh"
#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

// 0xFFFF in each half whose sign bit (bit 15 / bit 31) is set.  prmt's generic
// mode replicates the sign of the selected byte when the selector nibble has
// bit 3 set (__byte_perm masks that bit off, so it cannot be used here).
__device__ __forceinline__ uint32_t sign_mask(uint32_t x) {
  uint32_t r;
  asm("prmt.b32 %0, %1, 0, 0xBB99;" : "=r"(r) : "r"(x));
  return r;
}
// m ? a : b, bitwise.
__device__ __forceinline__ uint32_t bsel(uint32_t m, uint32_t a, uint32_t b) { return (a & m) | (b & ~m); }

// Offset-then-normalise of one int16 magnitude (c_lib/fixedpoint_ldpc_decoder.c:38-46):
// (int16)((alpha * max(m - beta, 0) + 2^14) >> 15), in int32 like the reference.
__device__ __forceinline__ uint32_t scale_half(int32_t m, int32_t alpha, int32_t beta) {
  int32_t off = m - beta;
  off = off < 0 ? 0 : off;
  const int32_t s = (alpha * off + (1 << 14)) >> 15;
  return (uint32_t)s & 0xFFFFu;
}
__device__ __forceinline__ uint32_t scale_pair(uint32_t c, int32_t alpha, int32_t beta) {
  const int32_t lo = (int32_t)(int16_t)(c & 0xFFFFu);
  const int32_t hi = ((int32_t)c) >> 16;
  return scale_half(lo, alpha, beta) | (scale_half(hi, alpha, beta) << 16);
}

// clip_llr (c_lib/fixedpoint_ldpc_decoder.c:28-36) of the exact int32 sum, for
// configurations with min_llr > max_llr where clamping is not a min/max pair.
__device__ __forceinline__ uint32_t clip_half_degen(int32_t v, int32_t mx, int32_t mn) {
  const int32_t r = v > mx ? mx : (v < mn ? mn : v);
  return (uint32_t)r & 0xFFFFu;
}

// |x| of each int16 half as an unsigned 16-bit value: max(x, -x) with the
// native packed subtract and signed max.  |-32768| comes out as 32768; in the
// unsigned minimum search below (which starts at 32767) that value never
// becomes a minimum, exactly like the reference's saturated 32767
// (c_lib/fixedpoint_ldpc_decoder.c:48-66), so no saturation step is needed.
__device__ __forceinline__ uint32_t abs_u16x2(uint32_t x) { return __vmaxs2(x, __vsub2(0u, x)); }

// m ? -v : v per half (two's complement, wrapping like the reference's int16
// store of sign * new_val): (v ^ m) - m.
__device__ __forceinline__ uint32_t cond_neg16x2(uint32_t v, uint32_t m) { return __vsub2(v ^ m, m); }

// One layer step of one lifted check row, for both code blocks of a pair.
//
// Compressed old message of the row (planes of the CTA scratch, kThreadsTarget
// words apart), with J = min(D, 16):
//   w0 = new_min1 pair, w1 = new_min2 pair,
//   w2 = sign flip of edge j < 16 at bit 15-(J-1-j) (block 0) and 31-(J-1-j)
//        (block 1),
//   w3 = "edge j carries new_min2" for j < 16 at bits j (block 0) / 16+j (block 1),
//   w4 (degree 19 only) = flips of edges 16..18 at bits j-3 / j+13 and their
//        "carries new_min2" bits at bits j-12 / j+4.
// Edge j's message is  flip ? -v : v  with  v = carries_min2 ? new_min2 : new_min1,
// which is exactly the reference's sel_lr[j] = (int16)(+-sign * new_val).
//
// Instruction budget: packed add/sub run on the FMA pipe, packed min/max,
// PRMT and LOP3 on the ALU pipe (the bottleneck); the emulated saturating
// packed ops are kept off the common path.
template <int D, bool kDegenClip>
__device__ __forceinline__ void row_update(const DecodeParams& p, char* __restrict__ lqs, uint32_t zx4,
                                           uint32_t zxm4, uint32_t gb4, int e0, int32_t alpha, int32_t beta,
                                           bool first, uint32_t* __restrict__ lrp) {
  constexpr int J = D < 16 ? D : 16;
  constexpr int S = kThreadsTarget;    // plane stride (words)
  uint32_t n1 = 0u, n2 = 0u, xf = 0u, xi = 0u, y = 0u;
  if (!first) {
    n1 = lrp[0];
    n2 = lrp[S];
    xf = lrp[2 * S];
    xi = lrp[3 * S];
    if (D > 16) y = lrp[4 * S];
  }

  uint32_t rel[D];
  uint32_t addr[D];
  uint32_t sg = 0u;                       // XOR of all inputs: sign parity per half
  uint32_t m1 = 0x7FFF7FFFu, m2 = 0x7FFF7FFFu;
  uint32_t oh0 = 0u, oh1 = 0u;            // last edge reaching the running minimum

  // Pass 1: extrinsic inputs rel = LQ - old message (int16 wrap-around, as the
  // reference's int16 assignment at c_lib/fixedpoint_ldpc_decoder.c:203),
  // sign parity, and the two smallest magnitudes.
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const uint2 cs = p.edge_cs4[e0 + j];              // (col*Zc*4, (V mod Zc)*4)
    const uint32_t t = min(zx4 + cs.y, zxm4 + cs.y);   // ((zx + V) mod Zc) * 4
    addr[j] = t + cs.x + gb4;
    const uint32_t q = *reinterpret_cast<const uint32_t*>(lqs + addr[j]);
    uint32_t mf, mi;
    if (j < 16) {
      mf = sign_mask(xf << (J - 1 - j));
      mi = sign_mask(xi << (15 - j));
    } else {
      mf = sign_mask(y << (18 - j));
      mi = sign_mask(y << (11 - (j - 16)));
    }
    const uint32_t r = cond_neg16x2(bsel(mi, n2, n1), mf);
    const uint32_t x = __vsub2(q, r);
    rel[j] = x;
    sg ^= x;
    const uint32_t a = abs_u16x2(x);
    bool ph, pl;
    const uint32_t nm1 = __vibmin_u16x2(a, m1, &ph, &pl);   // per half: a <= m1
    m2 = __vmaxu2(m1, __vminu2(m2, a));
    m1 = nm1;
    oh0 = pl ? (1u << j) : oh0;
    oh1 = ph ? (1u << j) : oh1;
  }
  // With ties at the minimum both minima are equal, so which tied edge is
  // marked does not change any message; the strict "<" of the reference
  // (c_lib/fixedpoint_ldpc_decoder.c:57-66) and "<=" give the same output.

  // Clip the minima (both <= 32767) to max_llr, then offset/normalise (:121-126).
  const uint32_t maxp = ((uint32_t)(uint16_t)p.max_llr) * 0x10001u;
  const uint32_t minp = ((uint32_t)(uint16_t)p.min_llr) * 0x10001u;
  const uint32_t s1 = scale_pair(__vmins2(m1, maxp), alpha, beta);
  const uint32_t s2 = scale_pair(__vmins2(m2, maxp), alpha, beta);
  const uint32_t XI = (oh0 & 0xFFFFu) | (oh1 << 16);
  uint32_t XF = 0u;
  uint32_t Y = 0u;
  if (D > 16) Y = ((oh0 >> 16) << 4) | ((oh1 >> 16) << 20);

  // Pass 2: new messages and new beliefs LQ = clip(rel + msg) (:129-143).
  // Common path: wrap-around sum, clamp, and a flag if any sum overflowed
  // int16 (then the row is redone below with the exact saturating sum).
  uint32_t ovf = 0u;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const uint32_t f = sg ^ rel[j];       // sign bit set: message is negated
    const uint32_t mf = sign_mask(f);
    uint32_t mi;
    if (j < 16) {
      mi = sign_mask(XI << (15 - j));
      XF = __umulhi(XF, 0x80000000u) | (f & 0x80008000u);     // XF >> 1, new flip on top
    } else {
      mi = sign_mask(Y << (11 - (j - 16)));
      Y |= (f >> (18 - j)) & (0x00010001u << (j - 3));
    }
    const uint32_t lr = cond_neg16x2(bsel(mi, s2, s1), mf);
    uint32_t nq;
    if (!kDegenClip) {
      const uint32_t sum = __vadd2(rel[j], lr);
      ovf |= (sum ^ rel[j]) & ~(rel[j] ^ lr);
      nq = __vmins2(__vmaxs2(sum, minp), maxp);
    } else {
      const int32_t lo = (int32_t)(int16_t)(rel[j] & 0xFFFFu) + (int32_t)(int16_t)(lr & 0xFFFFu);
      const int32_t hi = (((int32_t)rel[j]) >> 16) + (((int32_t)lr) >> 16);
      nq = clip_half_degen(lo, p.max_llr, p.min_llr) | (clip_half_degen(hi, p.max_llr, p.min_llr) << 16);
    }
    *reinterpret_cast<uint32_t*>(lqs + addr[j]) = nq;
  }
  if (!kDegenClip && (ovf & 0x80008000u) != 0u) {
    // Rare: some rel + msg left the int16 range.  Saturating add then clamp
    // equals clamping the exact sum when min_llr <= max_llr.
#pragma unroll
    for (int j = 0; j < D; ++j) {
      uint32_t mf, mi;
      if (j < 16) {
        mf = sign_mask(XF << (J - 1 - j));
        mi = sign_mask(XI << (15 - j));
      } else {
        mf = sign_mask(Y << (18 - j));
        mi = sign_mask(Y << (11 - (j - 16)));
      }
      const uint32_t lr = cond_neg16x2(bsel(mi, s2, s1), mf);
      *reinterpret_cast<uint32_t*>(lqs + addr[j]) = __vmins2(__vmaxs2(__vaddss2(rel[j], lr), minp), maxp);
    }
  }
  lrp[0] = s1;
  lrp[S] = s2;
  lrp[2 * S] = XF;
  lrp[3 * S] = XI;
  if (D > 16) lrp[4 * S] = Y;
}

template <bool kDegenClip>
__device__ __forceinline__ void layer_dispatch(int deg, const DecodeParams& p, char* lqs, uint32_t zx4, uint32_t zxm4,
                                               uint32_t gb4, int e0, int32_t alpha, int32_t beta, bool first,
                                               uint32_t* lrp) {
  switch (deg) {
#define NRLDPC_ROW(D) \
  case D: row_update<D, kDegenClip>(p, lqs, zx4, zxm4, gb4, e0, alpha, beta, first, lrp); break;
    NRLDPC_ROW(3)
    NRLDPC_ROW(4)
    NRLDPC_ROW(5)
    NRLDPC_ROW(6)
    NRLDPC_ROW(7)
    NRLDPC_ROW(8)
    NRLDPC_ROW(9)
    NRLDPC_ROW(10)
#undef NRLDPC_ROW
    default: row_update<19, kDegenClip>(p, lqs, zx4, zxm4, gb4, e0, alpha, beta, first, lrp); break;
  }
}

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

template <bool kDegenClip>
__global__ void __launch_bounds__(kThreadsTarget, 2) fixed_pair_kernel(const __grid_constant__ DecodeParams p) {
  extern __shared__ __align__(16) uint32_t s_lq[];        // [G][lq_len] int16x2
  __shared__ uint32_t s_crc[2 * kMaxGroups];

  const int tid = threadIdx.x;
  const int g = tid / p.Zc;
  const int zx = tid - g * p.Zc;
  const bool active = g < p.G;
  uint32_t* lq = s_lq + (active ? g : 0) * p.lq_len;
  uint32_t* scratch = p.scratch + (int64_t)blockIdx.x * p.scratch_words;
  const int Bp = (p.B + 31) & ~31;
  const uint32_t zx4 = 4u * (uint32_t)zx;
  const uint32_t zxm4 = zx4 - 4u * (uint32_t)p.Zc;     // wraps: min(zx4+s, zxm4+s) = ((zx+V) mod Zc)*4
  const uint32_t gb4 = 4u * (uint32_t)((active ? g : 0) * p.lq_len);

  for (int item = blockIdx.x; item < p.num_items; item += gridDim.x) {
    const int pair = item * p.G + g;
    const int cw0 = 2 * pair, cw1 = 2 * pair + 1;
    const bool v0 = active && cw0 < p.num_cw;
    const bool v1 = active && cw1 < p.num_cw;

    // ---- rate recovery into LQ (and the soft buffers) ----
    if (active) {
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
    for (; it < p.max_it; ++it) {
      for (int row = 0; row < p.R; ++row) {
        if (active) {
          const int e0 = p.row_off[row];
          const int deg = p.row_off[row + 1] - e0;
          const uint32_t ab = p.weights_T > 0 ? __ldg(p.weights + (min(it, p.weights_T - 1) * p.R + row))
                                              : p.w_inline[row];
          const int32_t alpha = (int32_t)(int16_t)(ab & 0xFFFFu);
          const int32_t beta = ((int32_t)ab) >> 16;
          layer_dispatch<kDegenClip>(deg, p, reinterpret_cast<char*>(s_lq), zx4, zxm4, gb4, e0, alpha, beta,
                                     it == 0, scratch + p.lr_off[row] + tid);
        }
        __syncthreads();
      }

      // ---- hard decisions + CRC of every code block in the CTA ----
      for (int k = tid; k < p.G * Bp; k += blockDim.x) {
        const int gg = k / Bp;          // warp-uniform: Bp and blockDim are multiples of 32
        const int i = k - gg * Bp;
        uint32_t r0 = 0u, r1 = 0u;
        if (i < p.B) {
          const uint32_t w = s_lq[gg * p.lq_len + i];
          const uint32_t tv = crc_term(p, i);
          r0 = (w & 0x8000u) ? tv : 0u;
          r1 = (w & 0x80000000u) ? tv : 0u;
        }
        r0 = __reduce_xor_sync(0xFFFFFFFFu, r0);
        r1 = __reduce_xor_sync(0xFFFFFFFFu, r1);
        if ((tid & 31) == 0) {
          if (r0) atomicXor(&s_crc[2 * gg], r0);
          if (r1) atomicXor(&s_crc[2 * gg + 1], r1);
        }
      }
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

}  // namespace

int launch_fixed(const DecodeParams& p, int grid, int block, int smem, bool degen_clip, void* stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t err;
  if (degen_clip) {
    err = cudaFuncSetAttribute(fixed_pair_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (err != cudaSuccess) return (int)err;
    fixed_pair_kernel<true><<<grid, block, smem, s>>>(p);
  } else {
    err = cudaFuncSetAttribute(fixed_pair_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (err != cudaSuccess) return (int)err;
    fixed_pair_kernel<false><<<grid, block, smem, s>>>(p);
  }
  count_launch();
  return (int)cudaGetLastError();
}

int occupancy_fixed(int block, int smem, bool degen_clip) {
  int n = 0;
  if (degen_clip) {
    cudaFuncSetAttribute(fixed_pair_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fixed_pair_kernel<true>, block, smem);
  } else {
    cudaFuncSetAttribute(fixed_pair_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fixed_pair_kernel<false>, block, smem);
  }
  return n;
}

}  // namespace nrldpc
