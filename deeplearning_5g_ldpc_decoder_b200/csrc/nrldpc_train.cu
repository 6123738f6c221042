// nrldpc_train.cu — differentiable unrolled layered float min-sum (forward and
// hand-written backward) for learning the normalisation alpha and offset beta.
//
// Forward semantics are those of the reference's PyTorch model
// (deep_learning/deeplearning_ldpc_model.py:315-410): per iteration t and
// base-graph row r, for every lifted check row
//   rel_j = LQ[c_j] - lr_old_j,  s_j = sign(rel_j) (+1 at 0),  a_j = |rel_j|
//   m1 = min a (first index idx), m2 = min over j != idx (first index idx2)
//   u_j = (j == idx) ? m2 : m1,  mag_j = alpha[t][r] * max(u_j - beta[t][r], 0)
//   lr_new_j = (prod s) * s_j * mag_j,  LQ[c_j] = clip(rel_j + lr_new_j)
// with the same float32 operations, so forward values match the model.
//
// Backward: the forward stores, at the start of every iteration, LQ and the
// check-to-variable messages (compressed: two magnitudes, one flip bit per edge,
// the minimum's position).  The backward walks iterations in reverse; for each
// it recomputes the iteration's forward from its checkpoint, keeping rel_j of
// every edge in a per-CTA tape, then back-propagates row by row:
//   g_v = g_LQ[c_j] * [|v| within clip],   g_lrt = g_carry_j + g_v
//   g_mag = (prod s) s_j g_lrt,            g_alpha += sum g_mag max(u - beta, 0)
//   g_u = g_mag alpha [u - beta >= 0],     g_beta -= sum g_u
//   g_a[idx] += sum_{j != idx} g_u_j,      g_a[idx2] += g_u_idx
//   g_rel = g_v + g_a sign0(rel)  (0 with detached check inputs)
//   g_LQ[c_j] = g_rel,  g_carry_j = -g_rel (for the previous iteration)
// which is what autograd computes for the model (torch.min routes the gradient
// to the returned index, abs to sign(x), clamp to its pass-through mask).
// Memory: O(iterations x state) for checkpoints, O(state) for tape and carry,
// instead of every intermediate tensor autograd would keep.
//
// Both kernels are templates over the real type: float is the training type;
// double exists so gradients can be checked against central finite differences
// without float32 rounding noise (the role float64 plays in torch's gradcheck).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

// Correctly rounded arithmetic in the kernel's real type (no FMA contraction,
// matching torch's separate elementwise ops).
__device__ __forceinline__ float r_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float r_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float r_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double r_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double r_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double r_mul(double a, double b) { return __dmul_rn(a, b); }
template <typename Real>
__device__ __forceinline__ Real r_inf() { return (Real)INFINITY; }

// Start moving a line toward L2 (the checkpoints, tape and carry are read row
// by row; issuing the next row's lines before the current row computes hides
// part of their DRAM latency).
__device__ __forceinline__ void prefetch_l2(const void* a) { asm volatile("prefetch.global.L2 [%0];" ::"l"(a)); }
// Ask L2 for the 16-byte-aligned interior of [lo, lo + bytes) with one
// cp.async.bulk.prefetch.L2 (a hint: nothing waits for it).
__device__ __forceinline__ void bulk_prefetch_l2(const void* lo, size_t bytes) {
  const uintptr_t a = (reinterpret_cast<uintptr_t>(lo) + 15u) & ~(uintptr_t)15u;
  const uintptr_t b = (reinterpret_cast<uintptr_t>(lo) + bytes) & ~(uintptr_t)15u;
  if (b > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(b - a)));
}

__device__ __forceinline__ uint32_t tr_addr(const TrainParams& p, int e, uint32_t zx) {
  const uint32_t ed = p.edge[e];
  uint32_t t = zx + (ed >> 16);
  t = min(t, t - (uint32_t)p.Zc);
  return (ed & 0xFFFFu) + t;
}

// Compressed messages of one lifted row block: Real m1[Zc], m2[Zc], then
// uint32 flips[Zc], first-minimum index[Zc].
template <typename Real>
struct MsgBlock {
  Real* mag;
  uint32_t* bits;
  __device__ MsgBlock(uint32_t* base, int row, int msg_words, int Zc) {
    uint32_t* b = base + (size_t)row * msg_words;
    mag = reinterpret_cast<Real*>(b);
    bits = b + 2 * Zc * (int)(sizeof(Real) / 4);
  }
};

// Forward of one lifted check row.  Old messages come from the checkpoint of
// iteration t (zero at t == 0); new messages go to the checkpoint of t+1.
template <int D, typename Real>
__device__ __forceinline__ void train_row_fwd(const TrainParams& p, Real* __restrict__ lq, uint32_t zx, int e0,
                                              int row, Real alpha, Real beta, uint32_t* old_msg,
                                              uint32_t* new_msg, Real* tape) {
  const int Zc = p.Zc;
  const Real clip = (Real)p.clip;
  Real n1 = 0, n2 = 0;
  uint32_t fl = 0u, ix = 0u;
  if (old_msg) {
    MsgBlock<Real> m(old_msg, row, p.msg_words, Zc);
    n1 = m.mag[zx];
    n2 = m.mag[Zc + zx];
    fl = m.bits[zx];
    ix = m.bits[Zc + zx];
  }
  Real rel[D];
  uint32_t addr[D];
  bool neg = false;
  Real m1 = r_inf<Real>(), m2 = r_inf<Real>();
  int idx = 0;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    addr[j] = tr_addr(p, e0 + j, zx);
    Real old = ((int)ix == j) ? n2 : n1;
    old = ((fl >> j) & 1u) ? -old : old;
    const Real r = r_sub(lq[addr[j]], old);
    rel[j] = r;
    if (tape) tape[(size_t)(e0 + j) * Zc + zx] = r;
    neg ^= (r < (Real)0);
    const Real a = fabs(r);
    if (a < m1) {
      m2 = m1;
      m1 = a;
      idx = j;
    } else if (a < m2) {
      m2 = a;
    }
  }
  const Real s1 = r_mul(alpha, fmax(r_sub(m1, beta), (Real)0));
  const Real s2 = r_mul(alpha, fmax(r_sub(m2, beta), (Real)0));
  uint32_t flips = 0u;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const bool flip = (rel[j] < (Real)0) != neg;
    const Real mag = (j == idx) ? s2 : s1;
    flips |= (flip ? 1u : 0u) << j;
    Real v = r_add(rel[j], flip ? -mag : mag);
    v = fmin(fmax(v, -clip), clip);
    lq[addr[j]] = v;
  }
  if (new_msg) {
    MsgBlock<Real> m(new_msg, row, p.msg_words, Zc);
    m.mag[zx] = s1;
    m.mag[Zc + zx] = s2;
    m.bits[zx] = flips;
    m.bits[Zc + zx] = (uint32_t)idx;
  }
}

// Backward of one lifted check row (see the file comment).
template <int D, typename Real>
__device__ __forceinline__ void train_row_bwd(const TrainParams& p, Real* __restrict__ glq, uint32_t zx, int e0,
                                              Real alpha, Real beta, const Real* tape, Real* carry, Real* ga,
                                              Real* gb) {
  const int Zc = p.Zc;
  const Real clip = (Real)p.clip;
  Real rel[D];
  uint32_t addr[D];
  bool neg = false;
  Real m1 = r_inf<Real>(), m2 = r_inf<Real>();
  int idx = 0, idx2 = -1;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    addr[j] = tr_addr(p, e0 + j, zx);
    rel[j] = tape[(size_t)(e0 + j) * Zc + zx];
    neg ^= (rel[j] < (Real)0);
    const Real a = fabs(rel[j]);
    if (a < m1) {
      m2 = m1;
      m1 = a;
      idx = j;
    } else if (a < m2) {
      m2 = a;
    }
  }
  // idx2 as torch.min over the entries other than idx: first strict minimum.
  {
    Real best = r_inf<Real>();
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const Real a = fabs(rel[j]);
      if (j != idx && a < best) {
        best = a;
        idx2 = j;
      }
    }
  }
  const Real o1 = r_sub(m1, beta), o2 = r_sub(m2, beta);
  const Real r1 = fmax(o1, (Real)0), r2 = fmax(o2, (Real)0);
  const Real k1 = o1 >= (Real)0 ? alpha : (Real)0;   // d mag / d u
  const Real k2 = o2 >= (Real)0 ? alpha : (Real)0;
  const Real s1 = r_mul(alpha, r1), s2 = r_mul(alpha, r2);
  Real g_a_idx = 0, g_a_idx2 = 0;
  Real g_mag_sum_r = 0, g_u_sum = 0;
  if constexpr (D > 10) {
    // Degree-19 rows keep only rel in registers: the edge addresses are
    // recomputed and the incoming gradient g_v is read again from shared
    // memory in the last pass (no other edge of the row writes that word),
    // so the BG1 kernel fits two CTAs per SM.  Same arithmetic as below.
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const uint32_t a = tr_addr(p, e0 + j, zx);
      const bool flip = (rel[j] < (Real)0) != neg;
      const Real mag = (j == idx) ? s2 : s1;
      const Real v = r_add(rel[j], flip ? -mag : mag);
      const Real gv = (v >= -clip && v <= clip) ? glq[a] : (Real)0;
      const Real g_lrt = carry[(size_t)(e0 + j) * Zc + zx] + gv;
      const Real g_mag = flip ? -g_lrt : g_lrt;
      g_mag_sum_r += g_mag * ((j == idx) ? r2 : r1);
      const Real g_u = g_mag * ((j == idx) ? k2 : k1);
      g_u_sum += g_u;
      if (j == idx) {
        g_a_idx2 += g_u;
      } else {
        g_a_idx += g_u;
      }
    }
    *ga += g_mag_sum_r;
    *gb -= g_u_sum;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const uint32_t a = tr_addr(p, e0 + j, zx);
      Real g_rel = 0;
      if (!p.detach) {
        const bool flip = (rel[j] < (Real)0) != neg;
        const Real mag = (j == idx) ? s2 : s1;
        const Real v = r_add(rel[j], flip ? -mag : mag);
        const Real gv = (v >= -clip && v <= clip) ? glq[a] : (Real)0;
        Real g_a = 0;
        if (j == idx) g_a += g_a_idx;
        if (j == idx2) g_a += g_a_idx2;
        const Real sg = rel[j] > (Real)0 ? (Real)1 : (rel[j] < (Real)0 ? (Real)-1 : (Real)0);
        g_rel = gv + g_a * sg;
      }
      glq[a] = g_rel;
      carry[(size_t)(e0 + j) * Zc + zx] = -g_rel;
    }
  } else {
    Real g_new[D];
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const bool flip = (rel[j] < (Real)0) != neg;
      const Real mag = (j == idx) ? s2 : s1;
      const Real v = r_add(rel[j], flip ? -mag : mag);
      const Real gv = (v >= -clip && v <= clip) ? glq[addr[j]] : (Real)0;
      g_new[j] = gv;
      Real* cr = carry + (size_t)(e0 + j) * Zc + zx;
      const Real g_lrt = *cr + gv;
      const Real g_mag = flip ? -g_lrt : g_lrt;
      g_mag_sum_r += g_mag * ((j == idx) ? r2 : r1);
      const Real g_u = g_mag * ((j == idx) ? k2 : k1);
      g_u_sum += g_u;
      if (j == idx) {
        g_a_idx2 += g_u;
      } else {
        g_a_idx += g_u;
      }
    }
    *ga += g_mag_sum_r;
    *gb -= g_u_sum;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      Real g_rel = 0;
      if (!p.detach) {
        Real g_a = 0;
        if (j == idx) g_a += g_a_idx;
        if (j == idx2) g_a += g_a_idx2;
        const Real sg = rel[j] > (Real)0 ? (Real)1 : (rel[j] < (Real)0 ? (Real)-1 : (Real)0);
        g_rel = g_new[j] + g_a * sg;
      }
      glq[addr[j]] = g_rel;
      carry[(size_t)(e0 + j) * Zc + zx] = -g_rel;
    }
  }
}

#define NRLDPC_TRAIN_DISPATCH(FN, R, deg, ...)   \
  switch (deg) {                                 \
    case 3: FN<3, R>(__VA_ARGS__); break;        \
    case 4: FN<4, R>(__VA_ARGS__); break;        \
    case 5: FN<5, R>(__VA_ARGS__); break;        \
    case 6: FN<6, R>(__VA_ARGS__); break;        \
    case 7: FN<7, R>(__VA_ARGS__); break;        \
    case 8: FN<8, R>(__VA_ARGS__); break;        \
    case 9: FN<9, R>(__VA_ARGS__); break;        \
    case 10: FN<10, R>(__VA_ARGS__); break;      \
    default: FN<(kMaxD > 10 ? 19 : 10), R>(__VA_ARGS__); break;      \
  }

// kMaxD: the largest row degree of the base graph (19 for BG1, 10 for BG2); a
// BG2 instantiation carries no degree-19 code and needs half the registers.
template <typename Real, int kMaxD>
__global__ void __launch_bounds__(kThreadsTarget) train_forward_kernel(const __grid_constant__ TrainParams p) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  Real* s_lq = reinterpret_cast<Real*>(s_raw);
  const Real* llr = static_cast<const Real*>(p.llr);
  const Real* alpha_t = static_cast<const Real*>(p.alpha);
  const Real* beta_t = static_cast<const Real*>(p.beta);
  Real* final_llr = static_cast<Real*>(p.final_llr);
  Real* iter_llr = static_cast<Real*>(p.iter_llr);
  Real* ck_lq = static_cast<Real*>(p.ck_lq);
  const Real clip = (Real)p.clip;
  const int tid = threadIdx.x;
  const int g = tid / p.Zc, zx = tid - g * p.Zc;
  const bool active = g < p.G;
  Real* lq = s_lq + (active ? g : 0) * p.n;
  const size_t cw_words = (size_t)p.R * p.msg_words;
  for (int item = blockIdx.x; item * p.G < p.batch; item += gridDim.x) {
    const int cw = item * p.G + g;
    const bool valid = active && cw < p.batch;
    if (valid)
      for (int i = zx; i < p.n; i += p.Zc) lq[i] = fmin(fmax(llr[(size_t)cw * p.n + i], -clip), clip);
    __syncthreads();
    for (int t = 0; t < p.T; ++t) {
      if (valid)
        for (int i = zx; i < p.n; i += p.Zc) ck_lq[((size_t)t * p.batch + cw) * p.n + i] = lq[i];
      uint32_t* old_msg = (t > 0 && valid) ? p.ck_lr + ((size_t)t * p.batch + cw) * cw_words : nullptr;
      uint32_t* new_msg = (t + 1 < p.T && valid) ? p.ck_lr + ((size_t)(t + 1) * p.batch + cw) * cw_words : nullptr;
      __syncthreads();
      for (int row = 0; row < p.R; ++row) {
        if (valid) {
          const int e0 = p.row_off[row], deg = p.row_off[row + 1] - e0;
          const Real alpha = alpha_t[t * p.R + row], beta = beta_t[t * p.R + row];
          NRLDPC_TRAIN_DISPATCH(train_row_fwd, Real, deg, p, lq, (uint32_t)zx, e0, row, alpha, beta, old_msg,
                                new_msg, nullptr)
        }
        __syncthreads();
      }
      if (valid && iter_llr)
        for (int i = zx; i < p.n; i += p.Zc) iter_llr[((size_t)t * p.batch + cw) * p.n + i] = lq[i];
    }
    if (valid)
      for (int i = zx; i < p.n; i += p.Zc) final_llr[(size_t)cw * p.n + i] = lq[i];
    __syncthreads();
  }
}

// Float: at most 85 registers, so two 384-thread CTAs fit an SM.
template <typename Real, int kMaxD, bool kAlias>
__global__ void __launch_bounds__(kThreadsTarget, sizeof(Real) > 4 ? 1 : 2)
    train_backward_kernel(const __grid_constant__ TrainParams p) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  __shared__ Real s_red[2][2][kThreadsTarget / 32];   // [row parity][alpha, beta][warp]
  Real* s_buf = reinterpret_cast<Real*>(s_raw);
  const Real* llr = static_cast<const Real*>(p.llr);
  const Real* alpha_t = static_cast<const Real*>(p.alpha);
  const Real* beta_t = static_cast<const Real*>(p.beta);
  const Real* ck_lq = static_cast<const Real*>(p.ck_lq);
  const Real* g_final = static_cast<const Real*>(p.g_final);
  const Real* g_iter = static_cast<const Real*>(p.g_iter);
  Real* g_llr = static_cast<Real*>(p.g_llr);
  Real* g_alpha = static_cast<Real*>(p.g_alpha);
  Real* g_beta = static_cast<Real*>(p.g_beta);
  const Real clip = (Real)p.clip;
  const int tid = threadIdx.x;
  const int g = tid / p.Zc, zx = tid - g * p.Zc;
  const bool active = g < p.G;
  // LQ and dLQ of each code block in shared memory.  With kAlias they share
  // one array (LQ while iteration t is recomputed, dLQ while it is
  // back-propagated; between iterations dLQ waits in the block's own row of
  // g_llr, which receives the final gradient at the end): half the shared
  // memory per block, for configurations where that puts more blocks on an SM.
  constexpr bool alias = kAlias;
  Real* lq = s_buf + (active ? g : 0) * p.n;
  Real* glq = alias ? lq : s_buf + (size_t)p.G * p.n + (active ? g : 0) * p.n;
  const size_t cw_words = (size_t)p.R * p.msg_words;
  const size_t edge_elems = (size_t)p.nnz * p.Zc;
  Real* tape = static_cast<Real*>(p.tape) + (size_t)blockIdx.x * p.scratch_per_cta + (size_t)(active ? g : 0) * edge_elems;
  Real* carry = static_cast<Real*>(p.carry) + (size_t)blockIdx.x * p.scratch_per_cta + (size_t)(active ? g : 0) * edge_elems;
  for (int item = blockIdx.x; item * p.G < p.batch; item += gridDim.x) {
    const int cw = item * p.G + g;
    const bool valid = active && cw < p.batch;
    Real* stash = g_llr + (size_t)(valid ? cw : 0) * p.n;
    Real* ginit = alias ? stash : glq;
    if (valid) {
      for (int i = zx; i < p.n; i += p.Zc) ginit[i] = g_final ? g_final[(size_t)cw * p.n + i] : (Real)0;
      for (size_t e = zx; e < edge_elems; e += p.Zc) carry[e] = 0;
    }
    __syncthreads();
    for (int t = p.T - 1; t >= 0; --t) {
      // every thread reads and writes only its own indices i = zx + k Zc here
      if (valid)
        for (int i = zx; i < p.n; i += p.Zc) {
          lq[i] = ck_lq[((size_t)t * p.batch + cw) * p.n + i];
          if (!alias && g_iter) glq[i] += g_iter[((size_t)t * p.batch + cw) * p.n + i];
        }
      uint32_t* old_msg = (t > 0 && valid) ? p.ck_lr + ((size_t)t * p.batch + cw) * cw_words : nullptr;
      __syncthreads();
      // Recompute iteration t, keeping every rel on the tape.
      for (int row = 0; row < p.R; ++row) {
        if (valid) {
          const int e0 = p.row_off[row], deg = p.row_off[row + 1] - e0;
          // The next row's checkpointed messages (all four planes).  Without
          // degree-19 rows (BG2) the group's first thread asks for the code
          // block's contiguous msg_words block with one bulk prefetch (BG2
          // Zc64 backward 6.33 -> 6.26 ms, no spills); the BG1 instantiation,
          // held at 80 registers, spills more with it (16.4 -> 16.9 ms) and
          // keeps one prefetch per plane and thread.
          if constexpr (kMaxD <= 10) {
            if (old_msg && row + 1 < p.R && zx == 0)
              bulk_prefetch_l2(old_msg + (size_t)(row + 1) * p.msg_words, (size_t)p.msg_words * 4u);
          } else if (old_msg && row + 1 < p.R) {
            MsgBlock<Real> m(old_msg, row + 1, p.msg_words, p.Zc);
            prefetch_l2(m.mag + zx);
            prefetch_l2(m.mag + p.Zc + zx);
            prefetch_l2(m.bits + zx);
            prefetch_l2(m.bits + p.Zc + zx);
          }
          const Real alpha = alpha_t[t * p.R + row], beta = beta_t[t * p.R + row];
          NRLDPC_TRAIN_DISPATCH(train_row_fwd, Real, deg, p, lq, (uint32_t)zx, e0, row, alpha, beta, old_msg,
                                nullptr, tape)
        }
        __syncthreads();
      }
      if constexpr (alias) {
        if (valid)
          for (int i = zx; i < p.n; i += p.Zc) {
            Real gq = stash[i];
            if (g_iter) gq += g_iter[((size_t)t * p.batch + cw) * p.n + i];
            glq[i] = gq;
          }
        __syncthreads();
      }
      // Back-propagate through the rows of iteration t.
      for (int row = p.R - 1; row >= 0; --row) {
        Real ga = 0, gb = 0;
        if (valid) {
          const int e0 = p.row_off[row], deg = p.row_off[row + 1] - e0;
          // tape and carry of the row back-propagated next (bulk, one slice
          // each, for the BG2 instantiation as above)
          if constexpr (kMaxD <= 10) {
            if (row > 0 && zx == 0) {
              const int ep = p.row_off[row - 1];
              const size_t bytes = (size_t)(e0 - ep) * (size_t)p.Zc * sizeof(Real);
              bulk_prefetch_l2(tape + (size_t)ep * p.Zc, bytes);
              bulk_prefetch_l2(carry + (size_t)ep * p.Zc, bytes);
            }
          } else if (row > 0) {
            const int ep = p.row_off[row - 1];
            for (int j = 0; j < e0 - ep; ++j) {
              prefetch_l2(tape + (size_t)(ep + j) * p.Zc + zx);
              prefetch_l2(carry + (size_t)(ep + j) * p.Zc + zx);
            }
          }
          const Real alpha = alpha_t[t * p.R + row], beta = beta_t[t * p.R + row];
          NRLDPC_TRAIN_DISPATCH(train_row_bwd, Real, deg, p, glq, (uint32_t)zx, e0, alpha, beta, tape, carry, &ga,
                                &gb)
        }
        // Block-level sum of this row's alpha/beta gradient, one atomic each.
        for (int o = 16; o > 0; o >>= 1) {
          ga += __shfl_xor_sync(0xFFFFFFFFu, ga, o);
          gb += __shfl_xor_sync(0xFFFFFFFFu, gb, o);
        }
        // Double-buffered by row parity: the next row's writes never meet this
        // row's read, which thread 0 finishes before the barrier after that row.
        if ((tid & 31) == 0) {
          s_red[row & 1][0][tid >> 5] = ga;
          s_red[row & 1][1][tid >> 5] = gb;
        }
        __syncthreads();
        if (tid == 0) {
          Real sa = 0, sb = 0;
          for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            sa += s_red[row & 1][0][w];
            sb += s_red[row & 1][1][w];
          }
          if (sa != (Real)0) atomicAdd(g_alpha + t * p.R + row, sa);
          if (sb != (Real)0) atomicAdd(g_beta + t * p.R + row, sb);
        }
      }
      if (alias && t > 0 && valid)
        for (int i = zx; i < p.n; i += p.Zc) stash[i] = glq[i];   // own indices: no barrier needed
    }
    if (valid)
      for (int i = zx; i < p.n; i += p.Zc) {
        const Real x = llr[(size_t)cw * p.n + i];
        g_llr[(size_t)cw * p.n + i] = (x >= -clip && x <= clip) ? glq[i] : (Real)0;
      }
    __syncthreads();
  }
}

template <typename K>
int launch_one(K kernel, const TrainParams& p, int grid, int block, int smem, void* stream) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return (int)e;
  kernel<<<grid, block, smem, reinterpret_cast<cudaStream_t>(stream)>>>(p);
  count_launch();
  return (int)cudaGetLastError();
}

template <typename K>
int occupancy_one(K kernel, int block, int smem) {
  int n = 0;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, smem);
  return n;
}

}  // namespace

// BG2 has 42 rows and degrees up to 10; BG1 46 rows and one row of degree 19.
int launch_train_forward(const TrainParams& p, bool f64, int grid, int block, int smem, void* stream) {
  const bool bg2 = p.R == 42;
  if (f64)
    return bg2 ? launch_one(train_forward_kernel<double, 10>, p, grid, block, smem, stream)
               : launch_one(train_forward_kernel<double, 19>, p, grid, block, smem, stream);
  return bg2 ? launch_one(train_forward_kernel<float, 10>, p, grid, block, smem, stream)
             : launch_one(train_forward_kernel<float, 19>, p, grid, block, smem, stream);
}

int launch_train_backward(const TrainParams& p, bool f64, int grid, int block, int smem, void* stream) {
  const bool bg2 = p.R == 42;
  if (f64) {
    if (p.alias)
      return bg2 ? launch_one(train_backward_kernel<double, 10, true>, p, grid, block, smem, stream)
                 : launch_one(train_backward_kernel<double, 19, true>, p, grid, block, smem, stream);
    return bg2 ? launch_one(train_backward_kernel<double, 10, false>, p, grid, block, smem, stream)
               : launch_one(train_backward_kernel<double, 19, false>, p, grid, block, smem, stream);
  }
  if (p.alias)
    return bg2 ? launch_one(train_backward_kernel<float, 10, true>, p, grid, block, smem, stream)
               : launch_one(train_backward_kernel<float, 19, true>, p, grid, block, smem, stream);
  return bg2 ? launch_one(train_backward_kernel<float, 10, false>, p, grid, block, smem, stream)
             : launch_one(train_backward_kernel<float, 19, false>, p, grid, block, smem, stream);
}

int occupancy_train(bool backward, bool f64, bool bg2, int block, int smem, bool alias) {
  if (backward) {
    if (f64) {
      if (alias)
        return bg2 ? occupancy_one(train_backward_kernel<double, 10, true>, block, smem)
                   : occupancy_one(train_backward_kernel<double, 19, true>, block, smem);
      return bg2 ? occupancy_one(train_backward_kernel<double, 10, false>, block, smem)
                 : occupancy_one(train_backward_kernel<double, 19, false>, block, smem);
    }
    if (alias)
      return bg2 ? occupancy_one(train_backward_kernel<float, 10, true>, block, smem)
                 : occupancy_one(train_backward_kernel<float, 19, true>, block, smem);
    return bg2 ? occupancy_one(train_backward_kernel<float, 10, false>, block, smem)
               : occupancy_one(train_backward_kernel<float, 19, false>, block, smem);
  }
  if (f64)
    return bg2 ? occupancy_one(train_forward_kernel<double, 10>, block, smem)
               : occupancy_one(train_forward_kernel<double, 19>, block, smem);
  return bg2 ? occupancy_one(train_forward_kernel<float, 10>, block, smem)
             : occupancy_one(train_forward_kernel<float, 19>, block, smem);
}

}  // namespace nrldpc
