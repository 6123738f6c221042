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
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "nrldpc_internal.h"

namespace nrldpc {
namespace {

__device__ __forceinline__ uint32_t tr_addr(const TrainParams& p, int e, uint32_t zx) {
  const uint32_t ed = p.edge[e];
  uint32_t t = zx + (ed >> 16);
  t = min(t, t - (uint32_t)p.Zc);
  return (ed & 0xFFFFu) + t;
}

// Forward of one lifted check row.  Old messages come from the checkpoint of
// iteration t (zero at t == 0); new messages go to the checkpoint of t+1.
template <int D>
__device__ __forceinline__ void train_row_fwd(const TrainParams& p, float* __restrict__ lq, uint32_t zx, int e0,
                                              int row, float alpha, float beta, const uint32_t* old_msg,
                                              uint32_t* new_msg, float* tape) {
  const int Zc = p.Zc;
  float n1 = 0.f, n2 = 0.f;
  uint32_t fl = 0u, ix = 0u;
  if (old_msg) {
    const uint32_t* m = old_msg + (size_t)row * 4 * Zc + zx;
    n1 = __uint_as_float(m[0]);
    n2 = __uint_as_float(m[Zc]);
    fl = m[2 * Zc];
    ix = m[3 * Zc];
  }
  float rel[D];
  uint32_t addr[D];
  bool neg = false;
  float m1 = INFINITY, m2 = INFINITY;
  int idx = 0;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    addr[j] = tr_addr(p, e0 + j, zx);
    float old = ((int)ix == j) ? n2 : n1;
    old = ((fl >> j) & 1u) ? -old : old;
    const float r = __fsub_rn(lq[addr[j]], old);
    rel[j] = r;
    if (tape) tape[(size_t)(e0 + j) * Zc + zx] = r;
    neg ^= (r < 0.0f);
    const float a = fabsf(r);
    if (a < m1) {
      m2 = m1;
      m1 = a;
      idx = j;
    } else if (a < m2) {
      m2 = a;
    }
  }
  const float s1 = __fmul_rn(alpha, fmaxf(__fsub_rn(m1, beta), 0.0f));
  const float s2 = __fmul_rn(alpha, fmaxf(__fsub_rn(m2, beta), 0.0f));
  uint32_t flips = 0u;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const bool flip = (rel[j] < 0.0f) != neg;
    const float mag = (j == idx) ? s2 : s1;
    const float lr = flip ? -mag : mag;
    flips |= (flip ? 1u : 0u) << j;
    float v = __fadd_rn(rel[j], lr);
    v = fminf(fmaxf(v, -p.clip), p.clip);
    lq[addr[j]] = v;
  }
  if (new_msg) {
    uint32_t* m = new_msg + (size_t)row * 4 * Zc + zx;
    m[0] = __float_as_uint(s1);
    m[Zc] = __float_as_uint(s2);
    m[2 * Zc] = flips;
    m[3 * Zc] = (uint32_t)idx;
  }
}

// Backward of one lifted check row (see the file comment).
template <int D>
__device__ __forceinline__ void train_row_bwd(const TrainParams& p, float* __restrict__ glq, uint32_t zx, int e0,
                                              float alpha, float beta, const float* tape, float* carry, float* ga,
                                              float* gb) {
  const int Zc = p.Zc;
  float rel[D];
  uint32_t addr[D];
  bool neg = false;
  float m1 = INFINITY, m2 = INFINITY;
  int idx = 0, idx2 = -1;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    addr[j] = tr_addr(p, e0 + j, zx);
    rel[j] = tape[(size_t)(e0 + j) * Zc + zx];
    neg ^= (rel[j] < 0.0f);
    const float a = fabsf(rel[j]);
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
    float best = INFINITY;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const float a = fabsf(rel[j]);
      if (j != idx && a < best) {
        best = a;
        idx2 = j;
      }
    }
  }
  const float o1 = __fsub_rn(m1, beta), o2 = __fsub_rn(m2, beta);
  const float r1 = fmaxf(o1, 0.0f), r2 = fmaxf(o2, 0.0f);
  const float k1 = o1 >= 0.0f ? alpha : 0.0f;   // d mag / d u
  const float k2 = o2 >= 0.0f ? alpha : 0.0f;
  const float s1 = __fmul_rn(alpha, r1), s2 = __fmul_rn(alpha, r2);
  float g_a_idx = 0.0f, g_a_idx2 = 0.0f;
  float g_new[D], g_mag_sum_r = 0.0f, g_u_sum = 0.0f;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const bool flip = (rel[j] < 0.0f) != neg;
    const float mag = (j == idx) ? s2 : s1;
    const float v = __fadd_rn(rel[j], flip ? -mag : mag);
    const float gv = (v >= -p.clip && v <= p.clip) ? glq[addr[j]] : 0.0f;
    g_new[j] = gv;
    float* cr = carry + (size_t)(e0 + j) * Zc + zx;
    const float g_lrt = *cr + gv;
    const float g_mag = flip ? -g_lrt : g_lrt;
    g_mag_sum_r += g_mag * ((j == idx) ? r2 : r1);
    const float g_u = g_mag * ((j == idx) ? k2 : k1);
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
    float g_rel = 0.0f;
    if (!p.detach) {
      float g_a = 0.0f;
      if (j == idx) g_a += g_a_idx;
      if (j == idx2) g_a += g_a_idx2;
      const float sg = rel[j] > 0.0f ? 1.0f : (rel[j] < 0.0f ? -1.0f : 0.0f);
      g_rel = g_new[j] + g_a * sg;
    }
    glq[addr[j]] = g_rel;
    carry[(size_t)(e0 + j) * Zc + zx] = -g_rel;
  }
}

#define NRLDPC_TRAIN_DISPATCH(FN, deg, ...)   \
  switch (deg) {                              \
    case 3: FN<3>(__VA_ARGS__); break;        \
    case 4: FN<4>(__VA_ARGS__); break;        \
    case 5: FN<5>(__VA_ARGS__); break;        \
    case 6: FN<6>(__VA_ARGS__); break;        \
    case 7: FN<7>(__VA_ARGS__); break;        \
    case 8: FN<8>(__VA_ARGS__); break;        \
    case 9: FN<9>(__VA_ARGS__); break;        \
    case 10: FN<10>(__VA_ARGS__); break;      \
    default: FN<19>(__VA_ARGS__); break;      \
  }

__global__ void __launch_bounds__(kThreadsTarget) train_forward_kernel(const __grid_constant__ TrainParams p) {
  extern __shared__ __align__(16) float s_lqf[];
  const int tid = threadIdx.x;
  const int g = tid / p.Zc, zx = tid - g * p.Zc;
  const bool active = g < p.G;
  float* lq = s_lqf + (active ? g : 0) * p.n;
  const size_t msg_words = (size_t)p.R * 4 * p.Zc;
  for (int item = blockIdx.x; item * p.G < p.batch; item += gridDim.x) {
    const int cw = item * p.G + g;
    const bool valid = active && cw < p.batch;
    if (valid)
      for (int i = zx; i < p.n; i += p.Zc) lq[i] = fminf(fmaxf(p.llr[(size_t)cw * p.n + i], -p.clip), p.clip);
    __syncthreads();
    for (int t = 0; t < p.T; ++t) {
      if (valid)
        for (int i = zx; i < p.n; i += p.Zc) p.ck_lq[((size_t)t * p.batch + cw) * p.n + i] = lq[i];
      const uint32_t* old_msg = (t > 0 && valid) ? p.ck_lr + ((size_t)t * p.batch + cw) * msg_words : nullptr;
      uint32_t* new_msg = (t + 1 < p.T && valid) ? p.ck_lr + ((size_t)(t + 1) * p.batch + cw) * msg_words : nullptr;
      __syncthreads();
      for (int row = 0; row < p.R; ++row) {
        if (valid) {
          const int e0 = p.row_off[row], deg = p.row_off[row + 1] - e0;
          const float alpha = p.alpha[t * p.R + row], beta = p.beta[t * p.R + row];
          NRLDPC_TRAIN_DISPATCH(train_row_fwd, deg, p, lq, (uint32_t)zx, e0, row, alpha, beta, old_msg, new_msg,
                                nullptr)
        }
        __syncthreads();
      }
      if (valid && p.iter_llr)
        for (int i = zx; i < p.n; i += p.Zc) p.iter_llr[((size_t)t * p.batch + cw) * p.n + i] = lq[i];
    }
    if (valid)
      for (int i = zx; i < p.n; i += p.Zc) p.final_llr[(size_t)cw * p.n + i] = lq[i];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreadsTarget) train_backward_kernel(const __grid_constant__ TrainParams p) {
  extern __shared__ __align__(16) float s_buf[];
  __shared__ float s_red[2][2][kThreadsTarget / 32];   // [row parity][alpha, beta][warp]
  const int tid = threadIdx.x;
  const int g = tid / p.Zc, zx = tid - g * p.Zc;
  const bool active = g < p.G;
  float* lq = s_buf + (active ? g : 0) * p.n;
  float* glq = s_buf + (size_t)p.G * p.n + (active ? g : 0) * p.n;
  const size_t msg_words = (size_t)p.R * 4 * p.Zc;
  const size_t edge_words = (size_t)p.nnz * p.Zc;
  float* tape = p.tape + (size_t)blockIdx.x * p.scratch_per_cta + (size_t)(active ? g : 0) * edge_words;
  float* carry = p.carry + (size_t)blockIdx.x * p.scratch_per_cta + (size_t)(active ? g : 0) * edge_words;
  for (int item = blockIdx.x; item * p.G < p.batch; item += gridDim.x) {
    const int cw = item * p.G + g;
    const bool valid = active && cw < p.batch;
    if (valid) {
      for (int i = zx; i < p.n; i += p.Zc) glq[i] = p.g_final ? p.g_final[(size_t)cw * p.n + i] : 0.0f;
      for (size_t e = zx; e < edge_words; e += p.Zc) carry[e] = 0.0f;
    }
    __syncthreads();
    for (int t = p.T - 1; t >= 0; --t) {
      if (valid) {
        for (int i = zx; i < p.n; i += p.Zc) {
          lq[i] = p.ck_lq[((size_t)t * p.batch + cw) * p.n + i];
          if (p.g_iter) glq[i] += p.g_iter[((size_t)t * p.batch + cw) * p.n + i];
        }
      }
      const uint32_t* old_msg = (t > 0 && valid) ? p.ck_lr + ((size_t)t * p.batch + cw) * msg_words : nullptr;
      __syncthreads();
      // Recompute iteration t, keeping every rel on the tape.
      for (int row = 0; row < p.R; ++row) {
        if (valid) {
          const int e0 = p.row_off[row], deg = p.row_off[row + 1] - e0;
          const float alpha = p.alpha[t * p.R + row], beta = p.beta[t * p.R + row];
          NRLDPC_TRAIN_DISPATCH(train_row_fwd, deg, p, lq, (uint32_t)zx, e0, row, alpha, beta, old_msg, nullptr,
                                tape)
        }
        __syncthreads();
      }
      // Back-propagate through the rows of iteration t.
      for (int row = p.R - 1; row >= 0; --row) {
        float ga = 0.0f, gb = 0.0f;
        if (valid) {
          const int e0 = p.row_off[row], deg = p.row_off[row + 1] - e0;
          const float alpha = p.alpha[t * p.R + row], beta = p.beta[t * p.R + row];
          NRLDPC_TRAIN_DISPATCH(train_row_bwd, deg, p, glq, (uint32_t)zx, e0, alpha, beta, tape, carry, &ga, &gb)
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
          float sa = 0.0f, sb = 0.0f;
          for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            sa += s_red[row & 1][0][w];
            sb += s_red[row & 1][1][w];
          }
          if (sa != 0.0f) atomicAdd(p.g_alpha + t * p.R + row, sa);
          if (sb != 0.0f) atomicAdd(p.g_beta + t * p.R + row, sb);
        }
      }
    }
    if (valid)
      for (int i = zx; i < p.n; i += p.Zc) {
        const float x = p.llr[(size_t)cw * p.n + i];
        p.g_llr[(size_t)cw * p.n + i] = (x >= -p.clip && x <= p.clip) ? glq[i] : 0.0f;
      }
    __syncthreads();
  }
}

}  // namespace

int launch_train_forward(const TrainParams& p, int grid, int block, int smem, void* stream) {
  cudaError_t e = cudaFuncSetAttribute(train_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return (int)e;
  train_forward_kernel<<<grid, block, smem, reinterpret_cast<cudaStream_t>(stream)>>>(p);
  count_launch();
  return (int)cudaGetLastError();
}

int launch_train_backward(const TrainParams& p, int grid, int block, int smem, void* stream) {
  cudaError_t e = cudaFuncSetAttribute(train_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return (int)e;
  train_backward_kernel<<<grid, block, smem, reinterpret_cast<cudaStream_t>(stream)>>>(p);
  count_launch();
  return (int)cudaGetLastError();
}

int occupancy_train(bool backward, int block, int smem) {
  int n = 0;
  if (backward) {
    cudaFuncSetAttribute(train_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, train_backward_kernel, block, smem);
  } else {
    cudaFuncSetAttribute(train_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, train_forward_kernel, block, smem);
  }
  return n;
}

}  // namespace nrldpc
