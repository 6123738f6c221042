// nrldpc_mixed.cu — one persistent fixed-point decode kernel for batches that
// mix base graphs, lifting sizes, rates, modulations, redundancy versions and
// CRC types (algos 1, 2, 3).
//
// Same arithmetic as the uniform kernel (nrldpc_fixed_row.cuh, bit-exact with
// c_lib/fixedpoint_ldpc_decoder.c).  Differences:
//  * work items come from a device work queue (atomic counter, after each
//    CTA's first item, which is its own index); an item is a
//    CTA's claim on one (BG, Zc), whose tables (per-edge shared-memory offsets,
//    row offsets, scratch layout) are staged into shared memory;
//  * the CTA takes up to 2G blocks of that graph from the graph's block queue
//    (a second atomic cursor) and, whenever a block passes its CRC or reaches
//    max_iterations, emits it and refills that int16 half lane with the next
//    block of the queue: every block costs its own iterations, not the slowest
//    block's of its CTA.  The refilled half starts from zero messages (the
//    `fresh` mask) and its own iteration count, so each block decodes exactly
//    as it would alone;
//  * the two blocks of a lane pair share (BG, Zc) but may differ in every other
//    parameter: rate recovery, the CRC check and the outputs use each block's
//    own B, E, Qm, rv and CRC type.
#include <cuda_runtime.h>
#include <stdint.h>

#include "nrldpc_decode_common.cuh"
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
    const int64_t idx = (int64_t)sidx * c.Qm + b;
    if (NRLDPC_INBOUNDS(idx, c.E, kBoundsLlr)) s += __ldg(in + idx);
  }
  return s;
}

// The block descriptors are read from global memory where they are used
// rather than kept in registers through the decode loop.
__device__ void mixed_emit(const MixedParams& p, const uint32_t* lq, int zx, int Zc, int cw, int h, int status,
                           int iters) {
  const int shift = 16 * h;
  if (iters > 0 && p.bits) {
    const MixedCw& c = p.cws[cw];
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

// Next block of graph `key`'s queue, or -1 when it is empty.
__device__ __forceinline__ int take_block(const MixedParams& p, int key) {
  const int i = atomicAdd(p.key_cursor + key, 1);
  return i < p.key_count[key] ? p.cb_list[p.key_base[key] + i] : -1;
}

// Rate recovery of the refreshed halves (r_h) of a group's LQ words: half h gets
// block cw_h, zeros when cw_h < 0; the other half keeps its bits.  Blocks with
// E <= Nv (no LLR repeats) use the scatter form: (A) base values (filler, the
// stored soft buffer when combining, else 0), (B) each LLR, read with 16-byte
// loads where the row is aligned, added to its own position (int16 wrap-around),
// (C) the soft buffer stored.  Blocks with repetitions take the gather form in
// (A).  Called by every thread of the CTA (CTA barriers inside).
__device__ __noinline__ void recover_halves_mixed(const MixedParams& p, const MixedGraph& g, uint32_t* lq, int zx, bool active,
                                     const int* cw, bool r0, bool r1) {
  const bool rr[2] = {r0, r1};
  bool scat[2] = {false, false};
  if (active) {
    const uint32_t keep = (r0 ? 0u : 0x0000FFFFu) | (r1 ? 0u : 0xFFFF0000u);
    if (r0 || r1)
      for (int i = zx; i < g.lq_len; i += g.Zc) lq[i] &= keep;
    for (int h = 0; h < 2; ++h) {
      if (!rr[h] || cw[h] < 0) continue;
      const MixedCw c = p.cws[cw[h]];
      scat[h] = c.E <= c.Nv;
      int16_t* hq = (c.harq_mode && p.harq) ? p.harq + c.harq_off : nullptr;
      const int shift = 16 * h;
      if (scat[h]) {
        for (int i = zx; i < g.lq_len; i += g.Zc) {
          const int32_t a = (i >= c.B && i < g.K) ? p.fill : ((hq && (c.harq_mode & 1)) ? hq[i] : 0);
          lq[i] |= ((uint32_t)a & 0xFFFFu) << shift;
        }
      } else {
        const int16_t* in = p.llr + c.llr_off;
        for (int i = zx; i < g.lq_len; i += g.Zc) {
          const int32_t init = (hq && (c.harq_mode & 1)) ? hq[i] : 0;
          const int32_t a = mixed_recover(g, c, in, i, p.fill, init);
          if (hq && (c.harq_mode & 2)) hq[i] = (int16_t)a;
          lq[i] |= ((uint32_t)a & 0xFFFFu) << shift;
        }
      }
    }
  }
  __syncthreads();
  int16_t* lq16 = reinterpret_cast<int16_t*>(lq);
  const int twoZ = 2 * g.Zc;
  for (int h = 0; h < 2; ++h) {
    if (!scat[h]) continue;
    const MixedCw c = p.cws[cw[h]];
    const int16_t* in = p.llr + c.llr_off;
    const uint32_t magic = qm_magic(c.Qm);
    const uint32_t E = (uint32_t)c.E;
    auto add = [&](uint32_t e, int16_t x) {
      const uint32_t s = div_qm(e, (uint32_t)c.Qm, magic);
      int cc = c.c0 + (int)((e - s * (uint32_t)c.Qm) * (uint32_t)c.symbols + s);
      cc -= cc >= c.Nv ? c.Nv : 0;
      const int pos = (cc < c.B - twoZ ? cc : cc + c.F) + twoZ;
      if (NRLDPC_INBOUNDS(pos, g.lq_len, kBoundsLq)) lq16[2 * pos + h] = (int16_t)(lq16[2 * pos + h] + x);
    };
    uint32_t e = 8u * (uint32_t)zx;
    if ((reinterpret_cast<uintptr_t>(in) & 15u) == 0) {
      for (; e + 8u <= E; e += 8u * (uint32_t)g.Zc) {
        const int4 v = __ldg(reinterpret_cast<const int4*>(in + e));
        const uint32_t w4[4] = {(uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z, (uint32_t)v.w};
#pragma unroll
        for (int q = 0; q < 8; ++q) add(e + (uint32_t)q, (int16_t)(w4[q >> 1] >> (16 * (q & 1))));
      }
    }
    for (; e < E; e += 8u * (uint32_t)g.Zc)
      for (uint32_t q = e; q < e + 8u && q < E; ++q) add(q, __ldg(in + q));
  }
  __syncthreads();
  for (int h = 0; h < 2; ++h) {
    if (!scat[h]) continue;
    const MixedCw c = p.cws[cw[h]];
    if (!(c.harq_mode & 2) || !p.harq) continue;
    int16_t* hq = p.harq + c.harq_off;
    for (int i = zx; i < g.lq_len; i += g.Zc) hq[i] = (int16_t)(lq[i] >> (16 * h));
  }
}

// XOR of the warp's partial CRC remainders of slot gg into s_crc.
__device__ __forceinline__ void mixed_crc_flush(uint32_t* s_crc, int gg, uint32_t r0, uint32_t r1) {
  r0 = __reduce_xor_sync(0xFFFFFFFFu, r0);
  r1 = __reduce_xor_sync(0xFFFFFFFFu, r1);
  if ((threadIdx.x & 31) == 0) {
    if (r0) atomicXor(&s_crc[2 * gg], r0);
    if (r1) atomicXor(&s_crc[2 * gg + 1], r1);
  }
}

template <int kClip, int kThreads, int kCap, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) fixed_mixed_kernel(const __grid_constant__ MixedParams p) {
  constexpr int kGroups = kCap / 2;       // G = floor(kCap / Zc) <= kCap / 2 (Zc >= 2)
  extern __shared__ __align__(16) uint32_t s_lq[];
  __shared__ uint32_t s_crc[2 * kGroups];
  __shared__ MixedGraph s_g;
  __shared__ int4 s_grp[kGroups];         // per group: B of both halves (0 when idle), CRC table offsets
  __shared__ int s_cw[2 * kGroups];       // block in each half lane, -1 when idle (not held in registers:
                                          // the layer loop needs every register it can get)
  __shared__ uint4 s_rows[kMaxRows];      // per-layer descriptors of the claim's graph (row_descriptor layout)
  __shared__ int s_item;

  const int tid = threadIdx.x;
  uint32_t* scratch = p.scratch + (int64_t)blockIdx.x * p.scratch_words;
  const int num_items = p.num_items_dev ? *p.num_items_dev : p.num_items;
  // A CTA's first claim is its own index and later ones come from the queue:
  // CTAs are placed on the SMs breadth first, so a batch with fewer claims
  // than SMs gets one SM per claim instead of whichever CTAs reach the queue
  // first (two of them may share an SM), which shortens small batches.
  bool first = true;
  for (;;) {
    if (tid == 0) s_item = first ? (int)blockIdx.x : (int)gridDim.x + atomicAdd(p.counter, 1);
    first = false;
    __syncthreads();
    const int item = s_item;
    if (item >= num_items) break;
    const int key = p.items[item].graph;
    {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(p.graphs + key);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&s_g);
      for (int w = tid; w < (int)(sizeof(MixedGraph) / 4); w += blockDim.x) dst[w] = __ldg(src + w);
    }
    __syncthreads();
    const int Zc = s_g.Zc, G = s_g.G, lq_len = s_g.lq_len;
    // debug build: the graph's message planes fit the CTA's scratch (uniform over the CTA)
    if (!NRLDPC_INBOUNDS(s_g.lr_off[s_g.R] - 1u, p.scratch_words, kBoundsScratch)) break;
    const int g = tid / Zc;
    const int zx = tid - g * Zc;
    const bool active = g < G;
    uint32_t* lq = s_lq + (active ? g : 0) * lq_len;
    const int bi = s_g.bgn == 1 ? 0 : 1;
    for (int r = tid; r < s_g.R; r += blockDim.x) {
      const uint32_t e0 = s_g.row_off[r], dg = (uint32_t)s_g.row_off[r + 1] - e0;
      const uint32_t five = s_g.lr_off[r + 1] - s_g.lr_off[r] > 4u * kThreadsTarget ? 1u : 0u;
      s_rows[r] = make_uint4(s_g.lr_off[r], e0 | (dg << 16) | (five << 24), p.w_inline[bi][r], 0u);
    }
    if (tid < 2 * G) s_cw[tid] = take_block(p, key);
    __syncthreads();
    {
      const int cw[2] = {active ? s_cw[2 * g] : -1, active ? s_cw[2 * g + 1] : -1};
      if (__syncthreads_and(!active || (cw[0] < 0 && cw[1] < 0))) continue;   // the graph's queue is empty
      if (active) {
        if (zx == 0)
          s_grp[g] = make_int4(cw[0] >= 0 ? p.cws[cw[0]].B : 0, cw[1] >= 0 ? p.cws[cw[1]].B : 0,
                               cw[0] >= 0 ? p.cws[cw[0]].crctype * kMaxB : 0,
                               cw[1] >= 0 ? p.cws[cw[1]].crctype * kMaxB : 0);
      }
      recover_halves_mixed(p, s_g, lq, zx, active, cw, true, true);
    }
    uint32_t itv = 0u;   // iterations of half 0 in bits 0-15, half 1 in bits 16-31
    if (tid < 2 * kGroups) s_crc[tid] = 0u;
    uint32_t fresh = 0xFFFFFFFFu;   // both halves start their first iteration
    __syncthreads();
    // A group whose two half lanes hold no block skips the row work (it only
    // takes part in the barriers); such a group is never refilled.
    bool busy = active && (s_cw[2 * g] >= 0 || s_cw[2 * g + 1] >= 0);

    const uint32_t zx4 = 4u * (uint32_t)zx;
    const uint32_t zxm4 = zx4 - 4u * (uint32_t)Zc;
    const uint32_t gb4 = 4u * (uint32_t)((active ? g : 0) * lq_len);
    RowMsg nxt{};
    for (;;) {
      const bool run = p.max_it > 0;   // max_iterations == 0: rate recovery only, status 1
      for (int row = 0; run && row < s_g.R; ++row) {
        if (busy) {
          const RowMsg cur = nxt;
          const uint4 d = s_rows[row];
          const int rn = row + 1 < s_g.R ? row + 1 : 0;
          const uint2 dn = *reinterpret_cast<const uint2*>(&s_rows[rn]);
          nxt = load_row_msg(scratch + dn.x + tid, row_five(dn.y));
          uint32_t ab0, ab1;
          if (p.weights_T[bi] > 0) {
            ab0 = __ldg(p.weights[bi] + (min((int)(itv & 0xFFFFu), p.weights_T[bi] - 1) * s_g.R + row));
            ab1 = __ldg(p.weights[bi] + (min((int)(itv >> 16), p.weights_T[bi] - 1) * s_g.R + row));
          } else {
            ab0 = ab1 = d.z;
          }
          layer_dispatch<kClip, true, false>(row_deg(d.y), p, s_g.edges, reinterpret_cast<char*>(s_lq), zx4, zxm4, gb4,
                                           4u * (uint32_t)(G * lq_len), row_e0(d.y),
                                           (int32_t)(int16_t)(ab0 & 0xFFFFu), ((int32_t)ab0) >> 16,
                                           (int32_t)(int16_t)(ab1 & 0xFFFFu), ((int32_t)ab1) >> 16, cur, fresh,
                                           scratch + d.x + tid);
        }
        __syncthreads();
      }
      fresh = 0u;
      // Hard decisions + CRC of both halves of every group (each with its own B
      // and CRC type), four positions per step: one 16-byte shared load of
      // their LQ words and, for a half whose B is a multiple of 4 and which
      // covers all four, one 16-byte load of its table entries
      // T[B-4-i0 .. B-1-i0] (16-byte aligned), else one load per position.
      // A slot spans Bq4 = roundup(K, 128) / 4 steps (every block's B <= K),
      // a multiple of 32, so a warp's 32 steps share one slot: terms are XORed
      // per thread while the slot stays the same and the warp reduces once per
      // slot.
      {
        const int Bq4 = ((s_g.K + 127) & ~127) >> 2;
        const uint32_t bpm = bp_magic(Bq4);
        uint32_t r0 = 0u, r1 = 0u;
        int cur = -1;
        for (int k = tid; run && k < G * Bq4; k += blockDim.x) {
          const int gg = div_bp(k, bpm);
          if (gg != cur) {
            if (cur >= 0) mixed_crc_flush(s_crc, cur, r0, r1);
            r0 = r1 = 0u;
            cur = gg;
          }
          const int i0 = 4 * (k - gg * Bq4);
          const int4 gr = s_grp[gg];
          // i0 < B <= K for a half with work here, so i0 + 3 < lq_len
          if ((i0 < gr.x || i0 < gr.y) && NRLDPC_INBOUNDS(i0 + 3, lq_len, kBoundsLq)) {
            const uint4 w = *reinterpret_cast<const uint4*>(s_lq + gg * lq_len + i0);
            const uint32_t wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int B = h ? gr.y : gr.x;
              const uint32_t* tab = p.crc_tab + (h ? gr.w : gr.z);
              uint32_t acc = 0u;
              if (i0 + 4 <= B && (B & 3) == 0) {
                if (NRLDPC_INBOUNDS(B - 1 - i0, kMaxB, kBoundsCrc)) {
                  const uint4 t = __ldg(reinterpret_cast<const uint4*>(tab + (B - 4 - i0)));
                  const uint32_t tv[4] = {t.w, t.z, t.y, t.x};   // position i0 + j pairs with T[B-1-i0-j]
#pragma unroll
                  for (int j = 0; j < 4; ++j) acc ^= tv[j] & (h ? sign_of_byte3(wv[j]) : sign_of_byte1(wv[j]));
                }
              } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                  if (i0 + j < B && NRLDPC_INBOUNDS(B - 1 - i0 - j, kMaxB, kBoundsCrc))
                    acc ^= __ldg(tab + (B - 1 - i0 - j)) & (h ? sign_of_byte3(wv[j]) : sign_of_byte1(wv[j]));
                }
              }
              if (h) r1 ^= acc; else r0 ^= acc;
            }
          }
        }
        if (cur >= 0) mixed_crc_flush(s_crc, cur, r0, r1);
      }
      __syncthreads();
      bool refill[2] = {false, false};
      if (active) {
        for (int h = 0; h < 2; ++h) {
          const int c = s_cw[2 * g + h];
          if (c < 0) continue;
          if (run) itv += h ? 0x10000u : 1u;
          const int ith = (int)(h ? itv >> 16 : itv & 0xFFFFu);
          const bool pass = run && s_crc[2 * g + h] == 0u;
          if (pass || ith >= p.max_it) {
            mixed_emit(p, lq, zx, Zc, c, h, pass ? 0 : 1, ith);
            refill[h] = true;
          }
        }
      }
      // s_crc read and emits done before the lanes are refilled
      const bool any = __syncthreads_or(refill[0] || refill[1]);
      if (tid < 2 * kGroups) s_crc[tid] = 0u;
      if (!any) continue;   // nothing finished: the next iteration (the rows' barriers order s_crc)
      if (active && zx == 0)
        for (int h = 0; h < 2; ++h)
          if (refill[h]) s_cw[2 * g + h] = take_block(p, key);
      __syncthreads();
      const int cw[2] = {active ? s_cw[2 * g] : -1, active ? s_cw[2 * g + 1] : -1};
      if (active) {
        for (int h = 0; h < 2; ++h) {
          if (!refill[h]) continue;
          itv &= h ? 0x0000FFFFu : 0xFFFF0000u;
          if (cw[h] >= 0) fresh |= h ? 0xFFFF0000u : 0x0000FFFFu;
        }
        if (zx == 0 && (refill[0] || refill[1]))
          s_grp[g] = make_int4(cw[0] >= 0 ? p.cws[cw[0]].B : 0, cw[1] >= 0 ? p.cws[cw[1]].B : 0,
                               cw[0] >= 0 ? p.cws[cw[0]].crctype * kMaxB : 0,
                               cw[1] >= 0 ? p.cws[cw[1]].crctype * kMaxB : 0);
      }
      recover_halves_mixed(p, s_g, lq, zx, active, cw, refill[0], refill[1]);
      busy = active && (cw[0] >= 0 || cw[1] >= 0);
      if (__syncthreads_and(!busy)) break;
    }
  }
}

// Kernel instance of (check-node arithmetic variant, class).
template <int C>
struct MixedShape;
template <>
struct MixedShape<0> {
  static constexpr int kThreads = 384, kCap = 384, kMinBlocks = 2;
};
template <>
struct MixedShape<1> {
  static constexpr int kThreads = 256, kCap = 240, kMinBlocks = 3;
};

template <int D, int C>
constexpr auto mixed_fn() {
  return fixed_mixed_kernel<D, MixedShape<C>::kThreads, MixedShape<C>::kCap, MixedShape<C>::kMinBlocks>;
}

template <int D, int C>
int mixed_op(int op, const MixedParams* p, int grid, cudaStream_t s, int* occ) {
  const auto fn = mixed_fn<D, C>();
  const int smem = MixedShape<C>::kCap * kMaxCols * 4;   // largest G * (N + 2Zc) words of any of its graphs
  static std::atomic<uint32_t> attr_done{0};
  const int err = raise_smem_limit_once(fn, &attr_done, smem);
  if (err != 0) return err;
  if (op == 1) {
    fn<<<grid, MixedShape<C>::kThreads, smem, s>>>(*p);
    count_launch();
    return (int)cudaGetLastError();
  }
  if (op == 2) {
    *occ = 0;
    return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, fn, MixedShape<C>::kThreads, smem);
  }
  return 0;
}

template <int C>
int mixed_dispatch_c(int op, int clip_mode, const MixedParams* p, int grid, cudaStream_t s, int* occ) {
  switch (clip_mode) {
    case kClipDegen: return mixed_op<kClipDegen, C>(op, p, grid, s, occ);
    case kClipOpenMax: return mixed_op<kClipOpenMax, C>(op, p, grid, s, occ);
    default: return mixed_op<kClipClamp, C>(op, p, grid, s, occ);
  }
}

int mixed_dispatch(int op, int clip_mode, int cls, const MixedParams* p, int grid, void* stream, int* occ) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return cls == 1 ? mixed_dispatch_c<1>(op, clip_mode, p, grid, s, occ) : mixed_dispatch_c<0>(op, clip_mode, p, grid, s, occ);
}

}  // namespace

int bounds_read_mixed(uint32_t* out, bool reset) { return bounds_read_tu(out, reset); }

int mixed_class_capacity(int cls) { return cls == 1 ? MixedShape<1>::kCap : MixedShape<0>::kCap; }

int launch_mixed(const MixedParams& p, int grid, int clip_mode, void* stream, int cls) {
  return mixed_dispatch(1, clip_mode, cls, &p, grid, stream, nullptr);
}

int prepare_mixed(int clip_mode, int cls) { return mixed_dispatch(0, clip_mode, cls, nullptr, 0, nullptr, nullptr); }

int occupancy_mixed(int clip_mode, int cls) {
  int n = 0;
  mixed_dispatch(2, clip_mode, cls, nullptr, 0, nullptr, &n);
  return n;
}

}  // namespace nrldpc
