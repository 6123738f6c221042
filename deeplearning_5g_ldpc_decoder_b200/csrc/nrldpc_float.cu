// nrldpc_float.cu — FP32 layered decoders for sm_100a: float min-sum (algo 4)
// and belief propagation (algo 0).
//
// Semantics follow c_lib/floatpoint_ldpc_decoder.c.  Float min-sum
// (:163-220, :307-366) is reproduced operation for operation with
// round-to-nearest intrinsics (no FMA contraction), so it is bit-exact.  BP
// (:53-151, :237-298) calls tanhf/atanhf; on the device those are CUDA's float
// functions, which differ from the host libm's by an ulp or two now and then
// (the reference's own CUDA decoder has the same difference), so BP matches
// the C reference to a tolerance.  Evaluating them in double precision instead
// (nearly always the correctly rounded float) costs 3x the decode time.
//
// Mapping: one code block per group of Zc threads, up to G = floor(384 / Zc) groups
// per CTA, FP32 beliefs in shared memory, persistent grid.  Min-sum messages
// are stored compressed per lifted check row (two minima, flip bits, the
// minimum's position: 16 bytes); BP messages are stored per edge.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>

#include "nrldpc_decode_common.cuh"
#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

constexpr float kBpAtanhClip = 19.07f;   // c_lib/floatpoint_ldpc_decoder.c:31

__device__ __forceinline__ float clipf(float v, float mx, float mn) {
  // clip_float_llr (c_lib/floatpoint_ldpc_decoder.c:153-161)
  return v > mx ? mx : (v < mn ? mn : v);
}

// The code's edge table, staged into shared memory at kernel start: the rows
// read it twice per edge, and a shared load is cheaper than a dynamically
// indexed parameter read (BP: 39.0 -> 37.4 ms for 8192 BG1 Zc=384 blocks).
__shared__ uint32_t s_fedge[kMaxNnz];

__device__ __forceinline__ uint32_t edge_addr(const DecodeParams& p, int e, uint32_t zx) {
  const uint32_t ed = s_fedge[e];
  uint32_t t = zx + (ed >> 16);
  t = min(t, t - (uint32_t)p.Zc);
  return (ed & 0xFFFFu) + t;
}

// Belief word a of the code block's LQ (debug build: a < lq_len, else the load
// reads 0 and the store is dropped).
__device__ __forceinline__ float ld_lq(const DecodeParams& p, const float* lq, uint32_t a) {
  return NRLDPC_INBOUNDS(a, p.lq_len, kBoundsLq) ? lq[a] : 0.0f;
}
__device__ __forceinline__ void st_lq(const DecodeParams& p, float* lq, uint32_t a, float v) {
  if (NRLDPC_INBOUNDS(a, p.lq_len, kBoundsLq)) lq[a] = v;
}

// ---------------------------------------------------------------- float min-sum
// Stored message of a lifted check row (4 planes): new_min1, new_min2 (float
// bits), bit j = message of edge j negated, bit j = edge j carries new_min2.
template <int D>
__device__ __forceinline__ void fms_row(const DecodeParams& p, float* __restrict__ lq, uint32_t zx, int e0,
                                        bool first, uint32_t* __restrict__ lrp, int NT) {
  float n1 = 0.f, n2 = 0.f;
  uint32_t xf = 0u, xi = 0u;
  if (!first) {
    n1 = __uint_as_float(lrp[0]);
    n2 = __uint_as_float(lrp[NT]);
    xf = lrp[2 * NT];
    xi = lrp[3 * NT];
  }
  if (!NRLDPC_INBOUNDS(e0 + D - 1, kMaxNnz, kBoundsEdge)) return;   // debug build
  float rel[D];
  uint32_t addr[D];
  float m1 = FLT_MAX, m2 = FLT_MAX;
  int idx = 0;
  bool neg = false;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    addr[j] = edge_addr(p, e0 + j, zx);
    float r = ((xi >> j) & 1u) ? n2 : n1;
    r = ((xf >> j) & 1u) ? -r : r;
    const float v = __fsub_rn(ld_lq(p, lq, addr[j]), r);
    rel[j] = v;
    neg ^= (v < 0.0f);
    const float a = fabsf(v);
    // float_update_two_minima (:171-180): strict <, first index wins.
    if (a < m1) {
      m2 = m1;
      m1 = a;
      idx = j;
    } else if (a < m2) {
      m2 = a;
    }
  }
  const float c1 = clipf(m1, p.f_max, 0.0f);
  const float c2 = clipf(m2, p.f_max, 0.0f);
  float o1 = __fsub_rn(c1, p.f_beta);
  float o2 = __fsub_rn(c2, p.f_beta);
  o1 = o1 < 0.0f ? 0.0f : o1;
  o2 = o2 < 0.0f ? 0.0f : o2;
  const float s1 = __fmul_rn(p.f_alpha, o1);
  const float s2 = __fmul_rn(p.f_alpha, o2);
  uint32_t XF = 0u;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const float nv = (j == idx) ? s2 : s1;
    const bool flip = (rel[j] < 0.0f) != neg;
    const float msg = flip ? -nv : nv;      // edge_sign * new_val, edge_sign = +-1
    XF |= (flip ? 1u : 0u) << j;
    st_lq(p, lq, addr[j], clipf(__fadd_rn(rel[j], msg), p.f_max, p.f_min));
  }
  lrp[0] = __float_as_uint(s1);
  lrp[NT] = __float_as_uint(s2);
  lrp[2 * NT] = XF;
  lrp[3 * NT] = 1u << idx;
}

__device__ __forceinline__ void fms_dispatch(int deg, const DecodeParams& p, float* lq, uint32_t zx, int e0,
                                             bool first, uint32_t* lrp, int NT) {
  switch (deg) {
    case 3: fms_row<3>(p, lq, zx, e0, first, lrp, NT); break;
    case 4: fms_row<4>(p, lq, zx, e0, first, lrp, NT); break;
    case 5: fms_row<5>(p, lq, zx, e0, first, lrp, NT); break;
    case 6: fms_row<6>(p, lq, zx, e0, first, lrp, NT); break;
    case 7: fms_row<7>(p, lq, zx, e0, first, lrp, NT); break;
    case 8: fms_row<8>(p, lq, zx, e0, first, lrp, NT); break;
    case 9: fms_row<9>(p, lq, zx, e0, first, lrp, NT); break;
    case 10: fms_row<10>(p, lq, zx, e0, first, lrp, NT); break;
    default: fms_row<19>(p, lq, zx, e0, first, lrp, NT); break;
  }
}

// --------------------------------------------------------------------- BP
// cp.async.bulk.prefetch.L2: bring `bytes` (a multiple of 16, 16-byte-aligned
// start) of global memory toward L2; a hint, nothing waits for it.
__device__ __forceinline__ void bulk_prefetch_l2(const void* a, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(bytes));
}

__device__ __forceinline__ float bp_message(float prod) {
  // bp_message_from_product (:54-62)
  if (prod >= 1.0f) return 2.0f * kBpAtanhClip;
  if (prod <= -1.0f) return -2.0f * kBpAtanhClip;
  return __fmul_rn(2.0f, atanhf(prod));
}

// Registers are what limits this kernel's occupancy, so the row keeps only
// tanh values and suffix products live: rel = LQ - old message is parked in
// LQ's own shared-memory word until the update (a row's edges are distinct
// words that no other thread touches during the layer), edge addresses are
// recomputed from the constant-cache table, and the prefix product runs as a
// scalar.  The arithmetic and its order are unchanged.
template <int D>
__device__ __forceinline__ void bp_row(const DecodeParams& p, float* __restrict__ lq, uint32_t zx, int e0,
                                       bool first, uint32_t* __restrict__ lrp, int NT) {
  if (!NRLDPC_INBOUNDS(e0 + D - 1, kMaxNnz, kBoundsEdge)) return;   // debug build
  float th[D];
  int nz = 0, zidx = -1;
  float nzprod = 1.0f;
  // compute_tanh_values (:65-82): tanh(rel/2), zero count, product of non-zeros.
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const uint32_t a = edge_addr(p, e0 + j, zx);
    const float old = first ? 0.0f : __uint_as_float(lrp[j * NT]);
    const float v = __fsub_rn(ld_lq(p, lq, a), old);
    st_lq(p, lq, a, v);
    if (v == 0.0f) {
      ++nz;
      zidx = j;
      th[j] = 0.0f;
    } else {
      th[j] = tanhf(__fmul_rn(v, 0.5f));
      nzprod = __fmul_rn(nzprod, th[j]);
    }
  }
  if (nz == 0) {
    // prefix/suffix products (:85-96, :135-145), same multiplication order:
    // sf[j] = th[D-1] * ... * th[j+1] accumulated right to left (sf[D-1] = 1),
    // the prefix th[0] * ... * th[j-1] left to right.
    float sf[D];
    sf[D - 1] = 1.0f;
#pragma unroll
    for (int j = D - 2; j >= 0; --j) sf[j] = __fmul_rn(sf[j + 1], th[j + 1]);
    float pre = 1.0f;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const float m = bp_message(__fmul_rn(pre, sf[j]));
      pre = __fmul_rn(pre, th[j]);
      const uint32_t a = edge_addr(p, e0 + j, zx);
      lrp[j * NT] = __float_as_uint(m);
      st_lq(p, lq, a, __fadd_rn(ld_lq(p, lq, a), m));   // no clipping in BP (:148-150)
    }
  } else {
    // one zero input: only its edge gets a message (the product of the
    // others); two or more: every message is zero
    const float mz = nz == 1 ? bp_message(nzprod) : 0.0f;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const float m = j == zidx && nz == 1 ? mz : 0.0f;
      const uint32_t a = edge_addr(p, e0 + j, zx);
      lrp[j * NT] = __float_as_uint(m);
      st_lq(p, lq, a, __fadd_rn(ld_lq(p, lq, a), m));
    }
  }
}

__device__ __forceinline__ void bp_dispatch(int deg, const DecodeParams& p, float* lq, uint32_t zx, int e0,
                                            bool first, uint32_t* lrp, int NT) {
  switch (deg) {
    case 3: bp_row<3>(p, lq, zx, e0, first, lrp, NT); break;
    case 4: bp_row<4>(p, lq, zx, e0, first, lrp, NT); break;
    case 5: bp_row<5>(p, lq, zx, e0, first, lrp, NT); break;
    case 6: bp_row<6>(p, lq, zx, e0, first, lrp, NT); break;
    case 7: bp_row<7>(p, lq, zx, e0, first, lrp, NT); break;
    case 8: bp_row<8>(p, lq, zx, e0, first, lrp, NT); break;
    case 9: bp_row<9>(p, lq, zx, e0, first, lrp, NT); break;
    case 10: bp_row<10>(p, lq, zx, e0, first, lrp, NT); break;
    default: bp_row<19>(p, lq, zx, e0, first, lrp, NT); break;
  }
}

// Rate recovery of the CTA's code blocks into float LQ in scatter form (E <= Nv:
// every LLR lands on its own position), as the fixed-point kernel's
// recover_scatter: (A) each position's LQ word holds its int32 base value
// (filler, else the stored soft buffer with HARQ_on, else 0), (B) each LLR,
// read with coalesced 16-byte loads where the rows allow, is added at its
// closed-form position, (C) the sum, truncated to int16 like the reference's
// int16 soft buffer, is stored back to the soft buffer and dequantised to
// float (c_lib/tx_rx_process.c:42-44: exact).  Called by every thread of the
// CTA (it holds CTA barriers); `valid` selects the threads whose group has a
// block, `active` those that own a group.
static __device__ void recover_scatter_f(const DecodeParams& p, float* lq, int zx, bool active, bool valid, int cw) {
  int32_t* lqi = reinterpret_cast<int32_t*>(lq);
  int16_t* hq = (p.harq && valid) ? p.harq + (int64_t)cw * p.harq_stride : nullptr;
  if (active) {
    for (int i = zx; i < p.lq_len; i += p.Zc) {
      const bool filler = i >= p.B && i < p.K;
      lqi[i] = !valid ? 0 : filler ? p.fill : (p.harq_on && hq) ? (int32_t)hq[i] : 0;
    }
  }
  __syncthreads();
  if (valid) {
    const int16_t* in = p.llr + (int64_t)cw * p.llr_stride;
    const uint32_t E = (uint32_t)p.E;
    uint32_t e = 8u * (uint32_t)zx;
    if (p.rr_vec) {
      for (; e + 8u <= E; e += 8u * (uint32_t)p.Zc) {
        const int4 v = __ldg(reinterpret_cast<const int4*>(in + e));
        const uint32_t w4[4] = {(uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z, (uint32_t)v.w};
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int pos = scatter_position(p, e + (uint32_t)q);
          if (NRLDPC_INBOUNDS(pos, p.lq_len, kBoundsLq)) lqi[pos] += (int32_t)(int16_t)(w4[q >> 1] >> (16 * (q & 1)));
        }
      }
    }
    for (; e < E; e += 8u * (uint32_t)p.Zc) {   // unaligned rows, and the tail of 8 LLRs
      for (uint32_t q = e; q < e + 8u && q < E; ++q) {
        const int pos = scatter_position(p, q);
        if (NRLDPC_INBOUNDS(pos, p.lq_len, kBoundsLq)) lqi[pos] += (int32_t)__ldg(in + q);
      }
    }
  }
  __syncthreads();
  if (active) {
    for (int i = zx; i < p.lq_len; i += p.Zc) {
      const int16_t a = (int16_t)lqi[i];
      if (hq) hq[i] = a;
      lq[i] = __fdiv_rn((float)a, 128.0f);
    }
  }
}

__device__ void emit_float_block(const DecodeParams& p, const float* lq, int zx, int cw, int status, int iters) {
  if (iters > 0 && p.bits) {
    const int nbytes = (p.B + 7) >> 3;
    uint8_t* out = p.bits + (int64_t)cw * p.bits_stride;
    for (int byte = zx; byte < nbytes; byte += p.Zc) {
      uint32_t v = 0u;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int i = byte * 8 + b;
        v = (v << 1) | ((i < p.B && lq[i] < 0.0f) ? 1u : 0u);
      }
      out[byte] = (uint8_t)v;
    }
  }
  if (p.app) {
    float* out = reinterpret_cast<float*>(p.app) + (int64_t)cw * p.app_stride;
    for (int i = zx; i < p.lq_len; i += p.Zc) out[i] = lq[i];
  }
  if (zx == 0) {
    if (p.status) p.status[cw] = status;
    if (p.iters) p.iters[cw] = iters;
  }
}

template <bool kBP>
__global__ void __launch_bounds__(kThreadsTarget, 2) float_kernel(const __grid_constant__ DecodeParams p) {
  extern __shared__ __align__(16) float s_lqf[];     // [G][lq_len]
  __shared__ uint32_t s_crc[kMaxGroups];
  for (int e = threadIdx.x; e < kMaxNnz; e += blockDim.x) s_fedge[e] = p.edge[e];   // read after the first barrier
  // BP: per row, the 16-byte-aligned part of the next row's message slice
  // (row 0 of the next iteration after the last row) as {byte offset from the
  // CTA's scratch, bytes}, for the bulk L2 prefetch in the row loop.
  __shared__ uint2 s_pf[kMaxRows];
  if (kBP) {
    for (int r = threadIdx.x; r < p.R; r += blockDim.x) {
      const int rn = r + 1 < p.R ? r + 1 : 0;
      const uintptr_t base = reinterpret_cast<uintptr_t>(p.scratch + (int64_t)blockIdx.x * p.scratch_words);
      const uintptr_t lo = base + 4u * (uintptr_t)p.lr_off[rn];
      const uintptr_t hi = lo + 4u * (uintptr_t)(p.row_off[rn + 1] - p.row_off[rn]) * (uintptr_t)p.nact;
      const uintptr_t a = (lo + 15u) & ~(uintptr_t)15u, b = hi & ~(uintptr_t)15u;
      s_pf[r] = b > a ? make_uint2((uint32_t)(a - base), (uint32_t)(b - a)) : make_uint2(0u, 0u);
    }
  }

  const int tid = threadIdx.x;
  const int g = tid / p.Zc;
  const int zx = tid - g * p.Zc;
  const bool active = g < p.G;
  float* lq = s_lqf + (active ? g : 0) * p.lq_len;
  uint32_t* scratch = p.scratch + (int64_t)blockIdx.x * p.scratch_words;
  const int NT = p.nact;
  // debug build: every message word of the CTA (planes of nact words, ending at
  // lr_off[R]) lies inside its scratch
  if (!NRLDPC_INBOUNDS(p.lr_off[p.R] - 1u, p.scratch_words, kBoundsScratch)) return;
  const int Bp = (p.B + 31) & ~31;
  const uint32_t bpm = bp_magic(Bp);

  // Work items: fixed (item += grid) or, with a queue cursor, taken from the
  // device queue so CTAs that run faster take more (see the fixed-point kernel).
  __shared__ int s_item;
  for (int item = blockIdx.x;;) {
    if (p.cursor) {
      if (tid == 0) s_item = atomicAdd(p.cursor, 1);
      __syncthreads();
      item = s_item;
    }
    if (item >= p.num_items) break;
    const int cw = item * p.G + g;
    const bool valid = active && cw < p.num_cw;
    if (p.rr_scatter) recover_scatter_f(p, lq, zx, active, valid, cw);
    if (active && !p.rr_scatter) {
      const int16_t* in = p.llr + (int64_t)(valid ? cw : 0) * p.llr_stride;
      int16_t* hq = (p.harq && valid) ? p.harq + (int64_t)cw * p.harq_stride : nullptr;
      for (int i = zx; i < p.lq_len; i += p.Zc) {
        int32_t a = (p.harq_on && hq) ? hq[i] : 0;
        a = valid ? recover_position(p, in, i, a) : 0;
        if (hq) hq[i] = (int16_t)a;
        // dequantize_int16_to_llr (c_lib/tx_rx_process.c:42-44): exact.
        lq[i] = __fdiv_rn((float)(int16_t)a, 128.0f);
      }
    }
    if (tid < kMaxGroups) s_crc[tid] = 0u;
    bool done = !valid;
    __syncthreads();

    int it = 0;
    for (; it < p.max_it; ++it) {
      for (int row = 0; row < p.R; ++row) {
        if (active) {
          const int e0 = p.row_off[row];
          const int deg = p.row_off[row + 1] - e0;
          uint32_t* lrp = scratch + p.lr_off[row] + tid;
          if constexpr (kBP) {
            // The per-edge messages of the blocks in flight exceed L2, so their
            // loads wait on DRAM: start moving the next row's (row 0 of the next
            // iteration after the last row) toward L2 while this row computes.
            // The row's messages are one contiguous slice of the CTA's scratch,
            // so one thread asks for all of it with a single bulk prefetch (the
            // 16-byte-aligned part; the slice lies inside the scratch).
            if (tid == 0) {
              const uint2 pf = s_pf[row];
              if (pf.y) bulk_prefetch_l2(reinterpret_cast<const char*>(scratch) + pf.x, pf.y);
            }
          }
          if (kBP) {
            bp_dispatch(deg, p, lq, (uint32_t)zx, e0, it == 0, lrp, NT);
          } else {
            fms_dispatch(deg, p, lq, (uint32_t)zx, e0, it == 0, lrp, NT);
          }
        }
        __syncthreads();
      }
      // Hard decisions (LQ < 0) + CRC remainder per slot.  With B a multiple of
      // 4, four positions per step (one 16-byte shared load of their beliefs,
      // one 16-byte load of T[B-4-i0 .. B-1-i0]) over Bq4 = roundup(B, 128) / 4
      // steps per slot; otherwise one position per step over roundup(B, 32).
      // Either way a warp's 32 steps share one slot: XOR per thread, reduce
      // once per slot.
      {
        const bool quad = (p.B & 3) == 0;
        const int span = quad ? ((p.B + 127) & ~127) >> 2 : Bp;
        const uint32_t smag = quad ? bp_magic(span) : bpm;
        uint32_t r = 0u;
        int cur = -1;
        for (int k = tid; k < p.G * span; k += blockDim.x) {
          const int gg = div_bp(k, smag);
          if (gg != cur) {
            if (cur >= 0) {
              r = __reduce_xor_sync(0xFFFFFFFFu, r);
              if ((tid & 31) == 0 && r) atomicXor(&s_crc[cur], r);
            }
            r = 0u;
            cur = gg;
          }
          if (quad) {
            const int i0 = 4 * (k - gg * span);
            if (i0 < p.B && NRLDPC_INBOUNDS(p.B - 1 - i0, kMaxB, kBoundsCrc)) {   // i0 + 4 <= B
              const float4 w = *reinterpret_cast<const float4*>(s_lqf + gg * p.lq_len + i0);
              const uint4 t = __ldg(reinterpret_cast<const uint4*>(p.crc_tab + (p.B - 4 - i0)));
              // position i0 + j pairs with T[B-1-i0-j]
              r ^= (w.x < 0.0f ? t.w : 0u) ^ (w.y < 0.0f ? t.z : 0u) ^ (w.z < 0.0f ? t.y : 0u) ^
                   (w.w < 0.0f ? t.x : 0u);
            }
          } else {
            const int i = k - gg * Bp;
            if (i < p.B && s_lqf[gg * p.lq_len + i] < 0.0f) r ^= crc_term(p, i);
          }
        }
        if (cur >= 0) {
          r = __reduce_xor_sync(0xFFFFFFFFu, r);
          if ((tid & 31) == 0 && r) atomicXor(&s_crc[cur], r);
        }
      }
      __syncthreads();
      if (active && !done && s_crc[g] == 0u) {
        emit_float_block(p, lq, zx, cw, 0, it + 1);
        done = true;
      }
      const bool all_done = __syncthreads_and(done);
      if (tid < kMaxGroups) s_crc[tid] = 0u;
      if (all_done) {
        ++it;
        break;
      }
    }
    if (active && !done) emit_float_block(p, lq, zx, cw, 1, it);
    __syncthreads();   // LQ, s_crc and s_item are reused by the next item
    if (!p.cursor) item += gridDim.x;
  }
  if (p.cursor && tid == 0) {
    // every take of this CTA is done: the last CTA to finish rewinds the queue
    __threadfence();
    if (atomicAdd(p.cursor + 1, 1) == (int)gridDim.x - 1) {
      atomicExch(p.cursor, 0);
      atomicExch(p.cursor + 1, 0);
    }
  }
}

template <typename K>
int launch_impl(K kernel, std::atomic<uint32_t>* attr_done, const DecodeParams& p, int grid, int block, int smem,
                void* stream) {
  const int err = raise_smem_limit_once(kernel, attr_done);
  if (err != 0) return err;
  kernel<<<grid, block, smem, reinterpret_cast<cudaStream_t>(stream)>>>(p);
  count_launch();
  return (int)cudaGetLastError();
}

template <typename K>
int occupancy_impl(K kernel, std::atomic<uint32_t>* attr_done, int block, int smem) {
  int n = 0;
  if (raise_smem_limit_once(kernel, attr_done) != 0) return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, smem);
  return n;
}

}  // namespace

static std::atomic<uint32_t> g_attr_minsum{0}, g_attr_bp{0};   // raise_smem_limit_once, per kernel

int launch_float_minsum(const DecodeParams& p, int grid, int block, int smem, void* stream) {
  return launch_impl(float_kernel<false>, &g_attr_minsum, p, grid, block, smem, stream);
}
int launch_float_bp(const DecodeParams& p, int grid, int block, int smem, void* stream) {
  return launch_impl(float_kernel<true>, &g_attr_bp, p, grid, block, smem, stream);
}
int bounds_read_float(uint32_t* out, bool reset) { return bounds_read_tu(out, reset); }

int occupancy_float_minsum(int block, int smem) { return occupancy_impl(float_kernel<false>, &g_attr_minsum, block, smem); }
int occupancy_float_bp(int block, int smem) { return occupancy_impl(float_kernel<true>, &g_attr_bp, block, smem); }

}  // namespace nrldpc
