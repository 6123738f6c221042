// nrldpc_fixed_row.cuh — the int16x2 layered min-sum check-node step shared by
// the uniform-batch and mixed-batch fixed-point kernels (algos 1, 2, 3).
// Bit-exact restatement of c_lib/fixedpoint_ldpc_decoder.c:103-144.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "nrldpc_bounds.cuh"
#include "nrldpc_internal.h"

namespace nrldpc {
namespace fixedrow {

// 0xFFFF in each half whose sign bit (bit 15 / bit 31) is set.  prmt's generic
// mode replicates the sign of the selected byte when the selector nibble has
// bit 3 set (__byte_perm masks that bit off, so it cannot be used here).
__device__ __forceinline__ uint32_t sign_mask(uint32_t x) {
  uint32_t r;
  asm("prmt.b32 %0, %1, 0, 0xBB99;" : "=r"(r) : "r"(x));
  return r;
}
// a + b as a multiply-add by the launch parameter p.one (== 1): the compiler
// cannot fold it back into an add, so it issues on the FMA pipe, which has
// room, instead of the integer ALU pipe that bounds these kernels.
template <typename P>
__device__ __forceinline__ uint32_t add_fma(const P& p, uint32_t a, uint32_t b) { return a * p.one + b; }

// Hard-decision masks: all ones when the sign bit of byte b of w is set (prmt's sign-replicating
// selector nibbles 8 | b): byte 1 holds the sign of half 0, byte 3 that of half 1.
__device__ __forceinline__ uint32_t sign_of_byte1(uint32_t w) {
  uint32_t r;
  asm("prmt.b32 %0, %1, 0, 0x9999;" : "=r"(r) : "r"(w));
  return r;
}
__device__ __forceinline__ uint32_t sign_of_byte3(uint32_t w) {
  uint32_t r;
  asm("prmt.b32 %0, %1, 0, 0xBBBB;" : "=r"(r) : "r"(w));
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
// Both halves, each with its own (alpha, beta): the two code blocks of a lane
// pair may be at different iterations of an iteration-dependent table (algo 2).
__device__ __forceinline__ uint32_t scale_pair(uint32_t c, int32_t alpha0, int32_t beta0, int32_t alpha1,
                                               int32_t beta1) {
  const int32_t lo = (int32_t)(int16_t)(c & 0xFFFFu);
  const int32_t hi = ((int32_t)c) >> 16;
  return scale_half(lo, alpha0, beta0) | (scale_half(hi, alpha1, beta1) << 16);
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
// Every word keeps block 0's fields in bits 0-15 and block 1's in bits 16-31,
// so `fresh` (0xFFFF per half that starts its first iteration) clears one
// block's old message without touching the other's.
//
// Instruction budget: packed add/sub run on the FMA pipe, packed min/max,
// PRMT and LOP3 on the ALU pipe (the bottleneck); the emulated saturating
// packed ops are kept off the common path.
// The compressed old message words of one lifted row (w0..w4 below), loaded
// by the kernels one row ahead so that their L2 latency overlaps the row
// before.
struct RowMsg {
  uint32_t n1, n2, xf, xi, y;
};
__device__ __forceinline__ RowMsg load_row_msg(const uint32_t* lrp, bool five) {
  constexpr int S = kThreadsTarget;
  RowMsg m;
  m.n1 = lrp[0];
  m.n2 = lrp[S];
  m.xf = lrp[2 * S];
  m.xi = lrp[3 * S];
  m.y = five ? lrp[4 * S] : 0u;
  return m;
}

template <int D, int kClip, bool kSmemEdges, bool kG1, typename P>
__device__ __forceinline__ void row_update(const P& p, const uint2* __restrict__ sedges, char* __restrict__ lqs, uint32_t zx4,
                                           uint32_t zxm4, uint32_t gb4, uint32_t lq_limit, int e0, int32_t alpha, int32_t beta,
                                           int32_t alpha1, int32_t beta1, const RowMsg& old, uint32_t fresh,
                                           uint32_t* __restrict__ lrp) {
  constexpr int J = D < 16 ? D : 16;
  constexpr int S = kThreadsTarget;    // plane stride (words)
  uint32_t n1 = 0u, n2 = 0u, xf = 0u, xi = 0u, y = 0u;
  if (fresh != 0xFFFFFFFFu) {
    n1 = old.n1;
    n2 = old.n2;
    xf = old.xf;
    xi = old.xi;
    if (D > 16) y = old.y;
    if (fresh) {
      const uint32_t keep = ~fresh;
      n1 &= keep;
      n2 &= keep;
      xf &= keep;
      xi &= keep;
      y &= keep;
    }
  }

  uint32_t rel[D];
  uint32_t addr[D];
  uint32_t sg = 0u;                       // XOR of all inputs: sign parity per half
  uint32_t m1 = 0x7FFF7FFFu, m2 = 0x7FFF7FFFu;
  uint32_t oh0 = 0u, oh1 = 0u;            // last edge reaching the running minimum
  // debug build: the row's edge entries and (below) every belief word it touches
  if (!NRLDPC_INBOUNDS(e0 + D - 1, kMaxNnz, kBoundsEdge)) return;

  // Pass 1: extrinsic inputs rel = LQ - old message (int16 wrap-around, as the
  // reference's int16 assignment at c_lib/fixedpoint_ldpc_decoder.c:203),
  // sign parity, and the two smallest magnitudes.
#pragma unroll
  for (int j = 0; j < D; ++j) {
    uint2 cs;                                          // (col*Zc*4, (V mod Zc)*4)
    if constexpr (kSmemEdges) {
      cs = sedges[e0 + j];
    } else {
      cs = p.edge_cs4[e0 + j];
    }
    if constexpr (kClip == kClipOpenMax) {
      // the adds as multiply-adds on the FMA pipe (measured: 10.02 -> 9.30 ms
      // for 8192 BG1 Zc=384 blocks together with the open-max arithmetic; on
      // the clamp path, whose extra registers spill, it measured 1 % slower)
      const uint32_t a4 = add_fma(p, cs.y, zx4);                // (zx + V mod Zc) * 4
      const uint32_t t = __viaddmin_u32(a4, zxm4 - zx4, a4);    // ((zx + V) mod Zc) * 4
      addr[j] = kG1 ? add_fma(p, t, cs.x) : add_fma(p, t, cs.x) + gb4;
    } else {
      const uint32_t t = min(zx4 + cs.y, zxm4 + cs.y);          // ((zx + V) mod Zc) * 4
      addr[j] = t + cs.x + gb4;
    }
    const uint32_t q = NRLDPC_INBOUNDS(addr[j], lq_limit, kBoundsLq) ? *reinterpret_cast<const uint32_t*>(lqs + addr[j])
                                                                      : 0u;
    uint32_t mf, mi;
    if (j < 16) {
      mf = sign_mask(xf << (J - 1 - j));
      mi = sign_mask(xi << (15 - j));
    } else {
      mf = sign_mask(y << (18 - j));
      mi = sign_mask(y << (11 - (j - 16)));
    }
    // x = q - r with r = mf ? -v : v, as additions: -r = (v ^ ~mf) + (~mf & 1)
    // per half (the complement of v plus one where the message is not negated)
    const uint32_t nmf = ~mf;
    const uint32_t x = __vadd2(__vadd2(q, bsel(mi, n2, n1) ^ nmf), nmf & 0x00010001u);
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
  uint32_t s1, s2;
  if constexpr (kClip == kClipOpenMax) {
    // Both minima lie in [0, 32767] = [0, max_llr], beta = 0 and both halves
    // have the same alpha >= 0: each half is (alpha * m + 2^14) >> 15.
    const int32_t l1 = (int32_t)(m1 & 0xFFFFu) * alpha + (1 << 14), h1 = (int32_t)(m1 >> 16) * alpha + (1 << 14);
    const int32_t l2 = (int32_t)(m2 & 0xFFFFu) * alpha + (1 << 14), h2 = (int32_t)(m2 >> 16) * alpha + (1 << 14);
    s1 = __byte_perm((uint32_t)(l1 >> 15), (uint32_t)(h1 >> 15), 0x5410);
    s2 = __byte_perm((uint32_t)(l2 >> 15), (uint32_t)(h2 >> 15), 0x5410);
  } else {
    s1 = scale_pair(__vmins2(m1, maxp), alpha, beta, alpha1, beta1);
    s2 = scale_pair(__vmins2(m2, maxp), alpha, beta, alpha1, beta1);
  }
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
    uint32_t nq;
    if constexpr (kClip != kClipDegen) {
      // rel + lr with lr = mf ? -v : v = (v ^ mf) + (mf & 1) per half.  An
      // int16 overflow is a sum whose sign differs from rel's where rel and lr
      // agree in sign.
      const uint32_t t = bsel(mi, s2, s1) ^ mf;
      uint32_t sum;
      if constexpr (kClip == kClipOpenMax) {
        // Here alpha >= 0, so the scaled minima lie in [0, 32766] and lr has
        // mf's sign, except lr = 0 when v = 0 (the sum is rel then, and no
        // overflow is flagged either way).  Testing mf instead of lr keeps
        // lr out of registers: 8.76 vs 9.06 ms per 8192-block step (testing
        // t = v ^ mf measured 9.41 ms).
        sum = __vadd2(__vadd2(rel[j], t), mf & 0x00010001u);
        ovf |= (sum ^ rel[j]) & ~(rel[j] ^ mf);
      } else {
        // Scaled minima may be negative here (a negative alpha): neither mf
        // (an unflipped v < 0) nor t (a flipped v = -32768, which stays
        // -32768) always has lr's sign, so test lr itself
        // (tests/test_row_arithmetic_identities.py).
        const uint32_t lr = __vadd2(t, mf & 0x00010001u);
        sum = __vadd2(rel[j], lr);
        ovf |= (sum ^ rel[j]) & ~(rel[j] ^ lr);
      }
      // with max_llr = 32767 the upper clamp of an int16 is the identity
      nq = kClip == kClipOpenMax ? __vmaxs2(sum, minp) : __vmins2(__vmaxs2(sum, minp), maxp);
    } else {
      const uint32_t lr = cond_neg16x2(bsel(mi, s2, s1), mf);
      const int32_t lo = (int32_t)(int16_t)(rel[j] & 0xFFFFu) + (int32_t)(int16_t)(lr & 0xFFFFu);
      const int32_t hi = (((int32_t)rel[j]) >> 16) + (((int32_t)lr) >> 16);
      nq = clip_half_degen(lo, p.max_llr, p.min_llr) | (clip_half_degen(hi, p.max_llr, p.min_llr) << 16);
    }
    if (NRLDPC_INBOUNDS(addr[j], lq_limit, kBoundsLq)) *reinterpret_cast<uint32_t*>(lqs + addr[j]) = nq;
  }
  if (kClip != kClipDegen && (ovf & 0x80008000u) != 0u) {
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
      if (NRLDPC_INBOUNDS(addr[j], lq_limit, kBoundsLq))
        *reinterpret_cast<uint32_t*>(lqs + addr[j]) = __vmins2(__vmaxs2(__vaddss2(rel[j], lr), minp), maxp);
    }
  }
  lrp[0] = s1;
  lrp[S] = s2;
  lrp[2 * S] = XF;
  lrp[3 * S] = XI;
  if (D > 16) lrp[4 * S] = Y;
}

template <int kClip, bool kSmemEdges, bool kG1, typename P>
__device__ __forceinline__ void layer_dispatch(int deg, const P& p, const uint2* sedges, char* lqs, uint32_t zx4, uint32_t zxm4,
                                               uint32_t gb4, uint32_t lq_limit, int e0, int32_t alpha, int32_t beta,
                                               int32_t alpha1, int32_t beta1, const RowMsg& old, uint32_t fresh,
                                               uint32_t* lrp) {
  switch (deg) {
#define NRLDPC_ROW(D) \
  case D: row_update<D, kClip, kSmemEdges, kG1>(p, sedges, lqs, zx4, zxm4, gb4, lq_limit, e0, alpha, beta, alpha1, beta1, old, fresh, lrp); break;
    NRLDPC_ROW(3)
    NRLDPC_ROW(4)
    NRLDPC_ROW(5)
    NRLDPC_ROW(6)
    NRLDPC_ROW(7)
    NRLDPC_ROW(8)
    NRLDPC_ROW(9)
    NRLDPC_ROW(10)
#undef NRLDPC_ROW
    default: row_update<19, kClip, kSmemEdges, kG1>(p, sedges, lqs, zx4, zxm4, gb4, lq_limit, e0, alpha, beta, alpha1, beta1, old, fresh, lrp); break;
  }
}

}  // namespace fixedrow
}  // namespace nrldpc
