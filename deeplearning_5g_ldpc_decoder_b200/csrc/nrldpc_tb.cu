// nrldpc_tb.cu — transport blocks on the device: segmentation into code
// blocks, one mixed-size persistent decode of all code blocks of a batch, the
// transport-block CRC and payload gather; and the host serving loop that
// feeds batches to it (continuous batching, HBM-budget admission, bounded
// host-side waits only).
//
// Per batch, three launches on one stream, no host synchronisation:
//  1. tb_segment_kernel (one CTA): TS 38.212 5.2.2 segmentation of every
//     transport block, per-code-block rate-recovery parameters, then the code
//     blocks bucketed by (BG, Zc) into one block queue per graph, and one work
//     item per G lane pairs of each graph for the mixed kernel (largest
//     lifting sizes first);
//  2. fixed_mixed_kernel (nrldpc_mixed.cu), reading its item count from the
//     device;
//  3. tb_finish_kernel (one 512-thread CTA per transport block): code-block verdicts,
//     transport-block CRC as the XOR of per-code-block remainders shifted by
//     x^(bits after the block) mod g(x), and the payload bytes gathered.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <deque>
#include <thread>
#include <vector>

#include "nrldpc_internal.h"
#include "nrldpc_tb.cuh"

namespace nrldpc {
namespace {

constexpr int kCbBitsStride = kMaxB / 8;   // 1056 bytes of hard bits per code block
constexpr int kKeys = 128;                 // tb_graph_key range
constexpr int kSegThreads = 1024;

struct SegParams {
  MixedCw* cws;
  int32_t* cb_key;
  int32_t* tb_first;
  int32_t* tb_err;        // per TB: tb_segment error (0 = valid)
  MixedItem* items;
  int32_t* cb_list;       // [max_cbs] code blocks grouped by graph key
  int32_t* key_base;      // [kKeys] first cb_list entry of each key
  int32_t* key_count;     // [kKeys] code blocks of each key
  int32_t* key_cursor;    // [kKeys] queue cursors of the mixed kernel
  int32_t* num_items;     // [0] items of the batch, [1] batch error (1 = over capacity)
  int32_t* counter;       // work-queue head of the mixed kernel
  int32_t max_cbs, max_items;
  int32_t key_G[kKeys];           // pairs per work item of each (BG, Zc)
  int16_t key_by_rank[kKeys];     // keys in descending work per block; -1 past the end
};

__global__ void __launch_bounds__(kSegThreads) tb_segment_kernel(const nrldpc_tb_t* __restrict__ tbs, int n,
                                                                 const __grid_constant__ SegParams sp) {
  __shared__ int s_scan[kSegThreads];
  __shared__ int s_count[kKeys], s_cursor[kKeys], s_item_base[kKeys], s_cb_base[kKeys], s_items[kKeys];
  __shared__ int s_total, s_num_items, s_err;
  const int tid = threadIdx.x;
  if (tid < kKeys) {
    s_count[tid] = 0;
    s_cursor[tid] = 0;
    s_items[tid] = 0;
  }
  if (tid == 0) s_err = 0;
  // 1. code blocks per transport block, contiguous chunk of blocks per thread
  const int per = (n + kSegThreads - 1) / kSegThreads;
  const int t0 = min(n, tid * per), t1 = min(n, t0 + per);
  int local = 0;
  for (int t = t0; t < t1; ++t) {
    TbSeg s;
    int e = tb_segment(tbs[t].A, tbs[t].G, tbs[t].Qm, tbs[t].bgn, tbs[t].tbs_lbrm, &s);
    if (!e && tbs[t].rv > 3) e = kTbBadArg;
    sp.tb_err[t] = e;
    if (!e) local += s.C;
  }
  s_scan[tid] = local;
  __syncthreads();
  for (int off = 1; off < kSegThreads; off <<= 1) {   // inclusive Hillis-Steele scan
    const int v = tid >= off ? s_scan[tid - off] : 0;
    __syncthreads();
    s_scan[tid] += v;
    __syncthreads();
  }
  if (tid == kSegThreads - 1) s_total = s_scan[tid];
  __syncthreads();
  const int total = s_total;
  if (total > sp.max_cbs) {   // over capacity: nothing decodes, every block reports -4
    if (tid == 0) {
      sp.num_items[0] = 0;
      sp.num_items[1] = 1;
      *sp.counter = 0;
    }
    return;
  }
  // 2. code-block descriptors
  int cb = s_scan[tid] - local;
  for (int t = t0; t < t1; ++t) {
    sp.tb_first[t] = cb;
    if (sp.tb_err[t]) continue;
    TbSeg s;
    tb_segment(tbs[t].A, tbs[t].G, tbs[t].Qm, tbs[t].bgn, tbs[t].tbs_lbrm, &s);
    const int key = tb_graph_key(s.bgn, s.Zc, s.iLS);
    for (int r = 0; r < s.C; ++r, ++cb) {
      const int E = tb_cb_E(s, r);
      const CbDerived d = tb_cb_derive(s, E, tbs[t].rv, tbs[t].Qm);
      MixedCw c;
      c.B = d.B;
      c.E = E;
      c.Qm = tbs[t].Qm;
      c.symbols = d.symbols;
      c.c0 = d.c0;
      c.Nv = d.Nv;
      c.F = d.F;
      c.crctype = s.crc_cb;
      c.llr_off = tbs[t].llr_offset + tb_cb_llr_start(s, r);
      c.bits_off = (int64_t)cb * kCbBitsStride;
      c.ncb = d.Ncb;
      c.harq_mode = tbs[t].flags & (NRLDPC_TB_HARQ_COMBINE | NRLDPC_TB_HARQ_STORE);
      c.harq_off = tbs[t].harq_offset + (int64_t)r * (d.N + 2 * s.Zc);
      sp.cws[cb] = c;
      sp.cb_key[cb] = key;
      atomicAdd(&s_count[key], 1);
    }
  }
  __syncthreads();
  // 3. block queues and work items per (BG, Zc), largest lifting sizes first
  if (tid == 0) {
    int ib = 0, cbb = 0;
    for (int rank = 0; rank < kKeys; ++rank) {
      const int k = sp.key_by_rank[rank];
      if (k < 0) break;
      const int cnt = s_count[k];
      if (!cnt) continue;
      const int pairs = (cnt + 1) / 2, Gk = sp.key_G[k];
      const int items = (pairs + Gk - 1) / Gk;
      s_item_base[k] = ib;
      s_cb_base[k] = cbb;
      s_items[k] = items;
      ib += items;
      cbb += cnt;
    }
    s_num_items = ib;
    if (ib > sp.max_items) s_err = 1;
  }
  __syncthreads();
  if (s_err) {
    if (tid == 0) {
      sp.num_items[0] = 0;
      sp.num_items[1] = 1;
      *sp.counter = 0;
    }
    return;
  }
  if (tid < kKeys) {
    sp.key_base[tid] = s_count[tid] ? s_cb_base[tid] : 0;
    sp.key_count[tid] = s_count[tid];
    sp.key_cursor[tid] = 0;
  }
  // 4. scatter code blocks into their graph's queue (order inside a queue is
  //    free: a block's result does not depend on its lane partner)
  for (int c = tid; c < total; c += kSegThreads) {
    const int k = sp.cb_key[c];
    const int pos = atomicAdd(&s_cursor[k], 1);
    sp.cb_list[s_cb_base[k] + pos] = c;
  }
  // 5. item records: a claim on graph k's queue
  for (int i = tid; i < s_num_items; i += kSegThreads) {
    int k = -1;
    for (int rank = 0; rank < kKeys; ++rank) {
      const int kk = sp.key_by_rank[rank];
      if (kk < 0) break;
      if (s_items[kk] && i >= s_item_base[kk] && i < s_item_base[kk] + s_items[kk]) {
        k = kk;
        break;
      }
    }
    MixedItem m;
    m.graph = k;
    m.pad0 = m.pad1 = m.pad2 = 0;
    sp.items[i] = m;
  }
  if (tid == 0) {
    sp.num_items[0] = s_num_items;
    sp.num_items[1] = 0;
    *sp.counter = 0;
  }
}

// r(x) * b(x) mod g(x) for 24-bit remainders (g given without its x^24 term).
__device__ __forceinline__ uint32_t crc24_mulmod(uint32_t a, uint32_t b, uint32_t poly) {
  uint32_t r = 0;
  for (int i = 23; i >= 0; --i) {
    r <<= 1;
    if (r & 0x1000000u) r ^= 0x1000000u | poly;
    if ((b >> i) & 1u) r ^= a;
  }
  return r;
}

// x^k mod g(x).
__device__ __forceinline__ uint32_t crc24_xpow(uint64_t k, uint32_t poly) {
  uint32_t result = 1u, base = 2u;
  while (k) {
    if (k & 1u) result = crc24_mulmod(result, base, poly);
    base = crc24_mulmod(base, base, poly);
    k >>= 1;
  }
  return result;
}

struct FinishParams {
  const int32_t* tb_first;
  const int32_t* tb_err;
  const int32_t* batch_err;     // num_items[1]
  const uint8_t* cb_bits;
  const int32_t* cb_status;
  const int32_t* cb_iters;
  const uint32_t* crc24a_tab;   // T[d] = x^(d+24) mod g24A(x)
  uint8_t* out;
  int32_t* status;
  int32_t* iters;
};

__global__ void __launch_bounds__(512) tb_finish_kernel(const nrldpc_tb_t* __restrict__ tbs, int n,
                                                        const __grid_constant__ FinishParams fp) {
  const int tb = blockIdx.x;
  if (tb >= n) return;
  const int tid = threadIdx.x;
  __shared__ int s_fail, s_iters;
  __shared__ uint32_t s_rem;
  if (*fp.batch_err) {
    if (tid == 0) {
      fp.status[tb] = NRLDPC_ERR_ARG;
      if (fp.iters) fp.iters[tb] = 0;
    }
    return;
  }
  if (fp.tb_err[tb]) {
    if (tid == 0) {
      fp.status[tb] = NRLDPC_ERR_CONFIG;
      if (fp.iters) fp.iters[tb] = 0;
    }
    return;
  }
  TbSeg s;
  tb_segment(tbs[tb].A, tbs[tb].G, tbs[tb].Qm, tbs[tb].bgn, tbs[tb].tbs_lbrm, &s);
  const int first = fp.tb_first[tb];
  if (tid == 0) {
    s_fail = 0;
    s_iters = 0;
    s_rem = 0u;
  }
  __syncthreads();
  for (int r = tid; r < s.C; r += blockDim.x) {
    if (fp.cb_status[first + r] != 0) atomicOr(&s_fail, 1);
    atomicMax(&s_iters, fp.cb_iters[first + r]);
  }
  // payload bytes: code block r carries bytes [r*chunk, (r+1)*chunk) of the
  // transport block (its information part; C == 1: the whole payload)
  const int pay_bytes = tbs[tb].A / 8;
  const int chunk = s.C == 1 ? pay_bytes : s.A_cb / 8;
  uint8_t* out = fp.out + tbs[tb].out_offset;
  for (int i = tid; i < pay_bytes; i += blockDim.x) {
    const int r = i / chunk;
    out[i] = fp.cb_bits[(int64_t)(first + r) * kCbBitsStride + (i - r * chunk)];
  }
  if (s.C > 1) {
    // transport-block CRC24A over A + 24 bits spread over the code blocks
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int nbits = s.A_cb;
    for (int r = warp; r < s.C; r += nwarps) {
      const uint8_t* bits = fp.cb_bits + (int64_t)(first + r) * kCbBitsStride;
      uint32_t rem = 0u;
      for (int i = lane; i < nbits; i += 32)
        if ((bits[i >> 3] >> (7 - (i & 7))) & 1u) rem ^= __ldg(fp.crc24a_tab + (nbits - 1 - i));
      rem = __reduce_xor_sync(0xFFFFFFFFu, rem);
      if (lane == 0) {
        const uint64_t after = (uint64_t)s.B - (uint64_t)(r + 1) * nbits;
        atomicXor(&s_rem, crc24_mulmod(rem, crc24_xpow(after, 0x864CFBu), 0x864CFBu));
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    fp.status[tb] = (s_fail || s_rem != 0u) ? 1 : 0;
    if (fp.iters) fp.iters[tb] = s_iters;
  }
}

// Buffers and launch parameters of one batch in flight.  The engine has one
// lane per batch that may run concurrently (the serving loop's pipeline depth).
struct TbLane {
  MixedCw* d_cws = nullptr;
  int32_t* d_cb_key = nullptr;
  int32_t* d_tb_first = nullptr;
  int32_t* d_tb_err = nullptr;
  MixedItem* d_items = nullptr;
  int32_t* d_queue = nullptr;       // cb_list [max_cbs], key_base, key_count, key_cursor [kKeys each]
  int32_t* d_num_items = nullptr;   // [2]
  int32_t* d_counter = nullptr;
  uint8_t* d_cb_bits = nullptr;
  int32_t* d_cb_status = nullptr;
  int32_t* d_cb_iters = nullptr;
  uint32_t* d_scratch = nullptr;
  SegParams sp = {};
  MixedParams mp = {};
  FinishParams fp = {};
};

struct TbEngine {
  int device = 0, num_sms = 0;
  int max_tbs = 0, max_cbs = 0, max_items = 0;
  int clip = kClipClamp;   // check-node arithmetic variant (fixed_clip_mode)
  int grid = 1;
  MixedGraph* d_graphs = nullptr;
  const uint32_t* d_crc_tab = nullptr;
  SegParams sp = {};      // templates: key tables and decoder settings
  MixedParams mp = {};
  std::vector<TbLane*> lanes;
};

MixedGraph tb_make_graph(int bgn, int Zc, int iLS) {
  MixedGraph m;
  memset(&m, 0, sizeof(m));
  const BaseGraph& g = base_graph(bgn);
  m.bgn = bgn;
  m.Zc = Zc;
  m.R = g.rows;
  m.lq_len = g.cols * Zc;
  m.G = std::max(1, kThreadsTarget / Zc);
  m.K = (bgn == 1 ? 22 : 10) * Zc;
  m.N = (bgn == 1 ? 66 : 50) * Zc;
  uint32_t off = 0;
  for (int r = 0; r < g.rows; ++r) {
    m.lr_off[r] = off;
    off += (uint32_t)fixed_row_planes(g.degree[r]) * kThreadsTarget;
    m.row_off[r] = g.row_off[r];
  }
  m.lr_off[g.rows] = off;
  m.row_off[g.rows] = g.row_off[g.rows];
  for (int e = 0; e < g.nnz; ++e)
    m.edges[e] = make_uint2(4u * (uint32_t)g.col[e] * (uint32_t)Zc, 4u * (uint32_t)(g.vij[iLS][e] % Zc));
  return m;
}

void lane_free(TbLane* l) {
  cudaFree(l->d_cws);
  cudaFree(l->d_cb_key);
  cudaFree(l->d_tb_first);
  cudaFree(l->d_tb_err);
  cudaFree(l->d_items);
  cudaFree(l->d_queue);
  cudaFree(l->d_num_items);
  cudaFree(l->d_counter);
  cudaFree(l->d_cb_bits);
  cudaFree(l->d_cb_status);
  cudaFree(l->d_cb_iters);
  cudaFree(l->d_scratch);
  delete l;
}

void engine_free(TbEngine* e) {
  for (TbLane* l : e->lanes) lane_free(l);
  cudaFree(e->d_graphs);
  delete e;
}

// Allocate lanes until the engine has n of them.
int engine_lanes(TbEngine* e, int n) {
  while ((int)e->lanes.size() < n) {
    TbLane* l = new TbLane();
    const int max_cbs = e->max_cbs, max_tbs = e->max_tbs;
    const bool ok =
        cudaMalloc(&l->d_cws, (size_t)max_cbs * sizeof(MixedCw)) == cudaSuccess &&
        cudaMalloc(&l->d_cb_key, (size_t)max_cbs * sizeof(int32_t)) == cudaSuccess &&
        cudaMalloc(&l->d_tb_first, (size_t)max_tbs * sizeof(int32_t)) == cudaSuccess &&
        cudaMalloc(&l->d_tb_err, (size_t)max_tbs * sizeof(int32_t)) == cudaSuccess &&
        cudaMalloc(&l->d_items, (size_t)e->max_items * sizeof(MixedItem)) == cudaSuccess &&
        cudaMalloc(&l->d_queue, ((size_t)max_cbs + 3 * kKeys) * sizeof(int32_t)) == cudaSuccess &&
        cudaMalloc(&l->d_num_items, 2 * sizeof(int32_t)) == cudaSuccess &&
        cudaMalloc(&l->d_counter, sizeof(int32_t)) == cudaSuccess &&
        cudaMalloc(&l->d_cb_bits, (size_t)max_cbs * kCbBitsStride) == cudaSuccess &&
        cudaMalloc(&l->d_cb_status, (size_t)max_cbs * sizeof(int32_t)) == cudaSuccess &&
        cudaMalloc(&l->d_cb_iters, (size_t)max_cbs * sizeof(int32_t)) == cudaSuccess &&
        cudaMalloc(&l->d_scratch, (size_t)e->grid * mixed_scratch_words_per_cta() * sizeof(uint32_t)) == cudaSuccess &&
        cudaMemset(l->d_num_items, 0, 2 * sizeof(int32_t)) == cudaSuccess;
    if (!ok) {
      lane_free(l);
      return NRLDPC_ERR_CUDA;
    }
    SegParams& sp = l->sp;
    sp = e->sp;
    sp.cws = l->d_cws;
    sp.cb_key = l->d_cb_key;
    sp.tb_first = l->d_tb_first;
    sp.tb_err = l->d_tb_err;
    sp.items = l->d_items;
    sp.cb_list = l->d_queue;
    sp.key_base = l->d_queue + max_cbs;
    sp.key_count = l->d_queue + max_cbs + kKeys;
    sp.key_cursor = l->d_queue + max_cbs + 2 * kKeys;
    sp.num_items = l->d_num_items;
    sp.counter = l->d_counter;
    MixedParams& p = l->mp;
    p = e->mp;
    p.items = l->d_items;
    p.cb_list = sp.cb_list;
    p.key_base = sp.key_base;
    p.key_count = sp.key_count;
    p.key_cursor = sp.key_cursor;
    p.cws = l->d_cws;
    p.num_items_dev = l->d_num_items;
    p.counter = l->d_counter;
    p.bits = l->d_cb_bits;
    p.status = l->d_cb_status;
    p.iters = l->d_cb_iters;
    p.scratch = l->d_scratch;
    FinishParams& fp = l->fp;
    fp.tb_first = l->d_tb_first;
    fp.tb_err = l->d_tb_err;
    fp.batch_err = l->d_num_items + 1;
    fp.cb_bits = l->d_cb_bits;
    fp.cb_status = l->d_cb_status;
    fp.cb_iters = l->d_cb_iters;
    fp.crc24a_tab = e->d_crc_tab + (size_t)1 * kMaxB;
    e->lanes.push_back(l);
  }
  return NRLDPC_OK;
}

int engine_decode(TbEngine* e, int lane, const nrldpc_tb_t* d_tbs, int n, const int16_t* d_llr, uint8_t* d_out,
                  int32_t* d_status, int32_t* d_iters, int16_t* d_harq, cudaStream_t s) {
  if (n == 0) return NRLDPC_OK;
  TbLane* l = e->lanes[lane];
  tb_segment_kernel<<<1, kSegThreads, 0, s>>>(d_tbs, n, l->sp);
  count_launch();
  MixedParams mp = l->mp;
  mp.llr = d_llr;
  mp.harq = d_harq;
  if (launch_mixed(mp, e->grid, e->clip, s) != 0) return NRLDPC_ERR_CUDA;
  FinishParams fp = l->fp;
  fp.out = d_out;
  fp.status = d_status;
  fp.iters = d_iters;
  tb_finish_kernel<<<n, 512, 0, s>>>(d_tbs, n, fp);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? NRLDPC_OK : NRLDPC_ERR_CUDA;
}

// Serving's optional per-code-block record: the batch's code blocks sit in
// transport-block order in the lane (the segmentation kernel's scan), so
// member j's start is the sum of the C of the members before it.
int record_code_blocks(TbEngine* e, int lane, const nrldpc_serve_cfg_t* cfg, const std::vector<int>& members,
                       const std::vector<int>& ncb, cudaStream_t s) {
  const TbLane* l = e->lanes[lane];
  int first = 0;
  for (int i : members) {
    const int C = ncb[i];
    const int64_t dst = cfg->h_cb_first[i];
    if ((cfg->d_cb_status &&
         cudaMemcpyAsync(cfg->d_cb_status + dst, l->d_cb_status + first, (size_t)C * sizeof(int32_t),
                         cudaMemcpyDeviceToDevice, s) != cudaSuccess) ||
        (cfg->d_cb_iterations &&
         cudaMemcpyAsync(cfg->d_cb_iterations + dst, l->d_cb_iters + first, (size_t)C * sizeof(int32_t),
                         cudaMemcpyDeviceToDevice, s) != cudaSuccess) ||
        (cfg->d_cb_bits &&
         cudaMemcpyAsync(cfg->d_cb_bits + dst * kCbBitsStride, l->d_cb_bits + (int64_t)first * kCbBitsStride,
                         (size_t)C * kCbBitsStride, cudaMemcpyDeviceToDevice, s) != cudaSuccess))
      return NRLDPC_ERR_CUDA;
    first += C;
  }
  return NRLDPC_OK;
}

double now_s() {
  using clk = std::chrono::steady_clock;
  return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace nrldpc

using namespace nrldpc;

extern "C" {

int32_t nrldpc_tb_segment(const nrldpc_tb_t* tb, nrldpc_tb_info_t* info) {
  if (!tb || !info) return NRLDPC_ERR_ARG;
  memset(info, 0, sizeof(*info));
  TbSeg s;
  int e = tb_segment(tb->A, tb->G, tb->Qm, tb->bgn, tb->tbs_lbrm, &s);
  if (!e && tb->rv > 3) e = kTbBadArg;
  if (e) {
    static const char* why[] = {"", "bad A, G, Qm, rv or base graph", "does not split into equal byte-aligned code blocks",
                                "a code block's E exceeds 65535", "a code block gets no coded bits",
                                "the limited circular buffer is shorter than the systematic part"};
    fprintf(stderr, "nrldpc_tb_segment: invalid transport block (%s): A=%d G=%d Qm=%d rv=%d bgn=%d\n", why[e], tb->A,
            tb->G, tb->Qm, tb->rv, tb->bgn);
    return NRLDPC_ERR_CONFIG;
  }
  info->C = s.C;
  info->L_tb = s.L_tb;
  info->Kp = s.Kp;
  info->Zc = s.Zc;
  info->E_lo = s.E_lo;
  info->E_hi = s.E_hi;
  info->n_lo = s.n_lo;
  info->cb_cfg.bgn = (uint16_t)s.bgn;
  info->cb_cfg.A = (uint16_t)s.A_cb;
  info->cb_cfg.crctype = (uint16_t)s.crc_cb;
  info->cb_cfg.E = (uint16_t)s.E_lo;
  info->cb_cfg.rv = tb->rv;
  info->cb_cfg.Qm = tb->Qm;
  info->cb_cfg.HARQ_on = 0;
  const CbDerived d = tb_cb_derive(s, s.E_lo, tb->rv, tb->Qm);
  info->Ncb = d.Ncb;
  info->k0 = d.k0;
  info->harq_elems = (int64_t)s.C * (d.N + 2 * s.Zc);
  return NRLDPC_OK;
}

int32_t nrldpc_tb_select_bg(int32_t A, int32_t R_x1024) {
  if (A <= 292 || (A <= 3824 && R_x1024 <= 686) || R_x1024 <= 256) return 2;
  return 1;
}

int32_t nrldpc_tb_engine_create(int32_t max_tbs, int32_t max_cbs, const ldpc_decoder_cfg_t* dc, void** engine) {
  if (!engine || !dc || max_tbs <= 0 || max_cbs <= 0) return NRLDPC_ERR_ARG;
  *engine = nullptr;
  if (dc->algo < 1 || dc->algo > 3) {
    fprintf(stderr, "nrldpc_tb_engine_create: fixed-point algos 1-3 only (got %u)\n", dc->algo);
    return NRLDPC_ERR_ALGO;
  }
  TbEngine* e = new TbEngine();
  cudaGetDevice(&e->device);
  if (cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, e->device) != cudaSuccess) {
    delete e;
    return NRLDPC_ERR_CUDA;
  }
  e->max_tbs = max_tbs;
  e->max_cbs = max_cbs;
  // graph table for every (BG, Zc) key, and the key order (more work per block first)
  std::vector<MixedGraph> graphs(kKeys);
  memset(graphs.data(), 0, graphs.size() * sizeof(MixedGraph));
  std::vector<std::pair<long, int>> order;
  const int base[8] = {2, 3, 5, 7, 9, 11, 13, 15};
  for (int bgn = 1; bgn <= 2; ++bgn)
    for (int s = 0; s < 8; ++s)
      for (int j = 0; (base[s] << j) <= 384; ++j) {
        const int Zc = base[s] << j;
        const int key = tb_graph_key(bgn, Zc, s);
        graphs[key] = tb_make_graph(bgn, Zc, s);
        e->sp.key_G[key] = graphs[key].G;
        order.push_back(std::make_pair(-(long)base_graph(bgn).nnz * Zc, key));
      }
  std::sort(order.begin(), order.end());
  for (int r = 0; r < kKeys; ++r) e->sp.key_by_rank[r] = r < (int)order.size() ? (int16_t)order[r].second : -1;
  e->max_items = max_cbs + (int)order.size();
  int occ = occupancy_mixed(kClipClamp);   // every arithmetic variant has the same occupancy
  if (occ < 1) occ = 1;
  e->grid = std::max(1, std::min(2, occ) * e->num_sms);
  bool ok = cudaMalloc(&e->d_graphs, kKeys * sizeof(MixedGraph)) == cudaSuccess &&
            cudaMemcpy(e->d_graphs, graphs.data(), kKeys * sizeof(MixedGraph), cudaMemcpyHostToDevice) ==
                cudaSuccess &&
            device_crc_table(&e->d_crc_tab) == NRLDPC_OK;
  if (!ok) {
    engine_free(e);
    return NRLDPC_ERR_CUDA;
  }
  SegParams& sp = e->sp;
  sp.max_cbs = max_cbs;
  sp.max_items = e->max_items;
  MixedParams& p = e->mp;
  p.graphs = e->d_graphs;
  p.num_items = 0;
  p.crc_tab = e->d_crc_tab;
  p.scratch_words = mixed_scratch_words_per_cta();
  p.max_it = dc->max_iterations;
  p.fill = dc->filling_bit_value;
  p.max_llr = dc->max_llr;
  p.one = 1u;
  p.min_llr = dc->min_llr;
  for (int b = 0; b < 2; ++b) {
    const BaseGraph& g = base_graph(b + 1);
    for (int r = 0; r < g.rows; ++r) {
      const int16_t alpha = dc->algo == 3 ? current_degree_alpha(g.degree[r]) : (int16_t)dc->alpha;
      p.w_inline[b][r] = pack_ab(alpha, (int16_t)dc->beta);
    }
    p.weights_T[b] = 0;
    if (dc->algo == 2 && device_trained_table(b + 1, &p.weights[b], &p.weights_T[b]) != NRLDPC_OK) {
      engine_free(e);
      return NRLDPC_ERR_CUDA;
    }
  }
  // open-max arithmetic only when both base graphs' layers qualify
  e->clip = fixed_clip_mode(*dc, p.w_inline[0], base_graph(1).rows);
  if (e->clip == kClipOpenMax) e->clip = fixed_clip_mode(*dc, p.w_inline[1], base_graph(2).rows);
  if (engine_lanes(e, 1) != NRLDPC_OK) {
    engine_free(e);
    return NRLDPC_ERR_CUDA;
  }
  if (prepare_mixed(e->clip) != 0) {
    engine_free(e);
    return NRLDPC_ERR_CUDA;
  }
  *engine = e;
  return NRLDPC_OK;
}

int32_t nrldpc_tb_engine_destroy(void* engine) {
  if (!engine) return NRLDPC_ERR_ARG;
  cudaDeviceSynchronize();
  engine_free(static_cast<TbEngine*>(engine));
  return NRLDPC_OK;
}

int32_t nrldpc_tb_engine_decode(void* engine, const nrldpc_tb_t* d_tbs, int32_t num_tbs, const int16_t* d_llr,
                                uint8_t* d_out, int32_t* d_status, int32_t* d_iterations, int16_t* d_harq,
                                void* stream) {
  TbEngine* e = static_cast<TbEngine*>(engine);
  if (!e || num_tbs < 0 || num_tbs > e->max_tbs) return NRLDPC_ERR_ARG;
  if (num_tbs == 0) return NRLDPC_OK;
  if (!d_tbs || !d_llr || !d_out || !d_status) return NRLDPC_ERR_ARG;
  return engine_decode(e, 0, d_tbs, num_tbs, d_llr, d_out, d_status, d_iterations, d_harq,
                       reinterpret_cast<cudaStream_t>(stream));
}

int32_t nrldpc_tb_engine_views(void* engine, const uint8_t** d_cb_bits, const int32_t** d_cb_status,
                               const int32_t** d_cb_iterations, const int32_t** d_tb_first_cb) {
  TbEngine* e = static_cast<TbEngine*>(engine);
  if (!e) return NRLDPC_ERR_ARG;
  const TbLane* l = e->lanes[0];
  if (d_cb_bits) *d_cb_bits = l->d_cb_bits;
  if (d_cb_status) *d_cb_status = l->d_cb_status;
  if (d_cb_iterations) *d_cb_iterations = l->d_cb_iters;
  if (d_tb_first_cb) *d_tb_first_cb = l->d_tb_first;
  return NRLDPC_OK;
}

int32_t nrldpc_serve_run(void* engine, const nrldpc_serve_cfg_t* cfg, const nrldpc_tb_t* tbs, const double* arrival_s,
                         int32_t n, const int16_t* d_llr, uint8_t* d_out, int32_t* h_status, double* h_latency_s,
                         nrldpc_serve_stats_t* stats, void* stream) {
  TbEngine* e = static_cast<TbEngine*>(engine);
  if (!e || !cfg || n < 0 || (n > 0 && (!tbs || !arrival_s || !d_llr || !d_out || !h_status || !h_latency_s)))
    return NRLDPC_ERR_ARG;
  const int depth = std::max(1, std::min(16, cfg->pipeline_depth));
  const int max_tbs = std::max(1, std::min(cfg->max_batch_tbs, e->max_tbs));
  const int max_cbs = std::max(1, std::min(cfg->max_batch_cbs, e->max_cbs));
  for (int i = 1; i < n; ++i)
    if (arrival_s[i] < arrival_s[i - 1]) return NRLDPC_ERR_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // Per in-flight slot: its own stream and engine lane (so a new batch starts
  // while earlier ones still decode, on SMs they leave free), pinned
  // descriptors and verdicts, device descriptors, a completion event.
  struct Slot {
    nrldpc_tb_t* h_tbs = nullptr;
    int32_t* h_status = nullptr;
    nrldpc_tb_t* d_tbs = nullptr;
    int32_t* d_status = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    std::vector<int> members;
  };
  std::vector<Slot> slots(depth);
  int rc = engine_lanes(e, depth);
  cudaEvent_t start = nullptr;
  if (rc == NRLDPC_OK && (cudaEventCreateWithFlags(&start, cudaEventDisableTiming) != cudaSuccess ||
                          cudaEventRecord(start, s) != cudaSuccess))
    rc = NRLDPC_ERR_CUDA;
  for (Slot& sl : slots) {
    if (rc != NRLDPC_OK) break;
    if (cudaMallocHost(&sl.h_tbs, (size_t)max_tbs * sizeof(nrldpc_tb_t)) != cudaSuccess ||
        cudaMallocHost(&sl.h_status, (size_t)max_tbs * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&sl.d_tbs, (size_t)max_tbs * sizeof(nrldpc_tb_t)) != cudaSuccess ||
        cudaMalloc(&sl.d_status, (size_t)max_tbs * sizeof(int32_t)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamWaitEvent(sl.stream, start, 0) != cudaSuccess ||   // after the caller's queued work
        cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess)
      rc = NRLDPC_ERR_CUDA;
  }
  // code blocks per transport block (host copy of the segmentation, for batch sizing)
  std::vector<int> ncb(n, 0);
  for (int i = 0; i < n && rc == NRLDPC_OK; ++i) {
    TbSeg sg;
    const int err = tb_segment(tbs[i].A, tbs[i].G, tbs[i].Qm, tbs[i].bgn, tbs[i].tbs_lbrm, &sg);
    ncb[i] = (err || tbs[i].rv > 3) ? -1 : sg.C;
    if (ncb[i] > max_cbs) ncb[i] = -1;   // cannot fit any batch: rejected as a configuration error
  }
  nrldpc_serve_stats_t st;
  memset(&st, 0, sizeof(st));
  std::deque<int> ready;
  std::vector<int> inflight;   // slot indices
  std::vector<int> free_slots;
  for (int k = depth - 1; k >= 0; --k) free_slots.push_back(k);
  int64_t budget_used = 0;
  int next = 0;
  int64_t done = 0;
  double batch_tbs_sum = 0.0;
  const double t0 = now_s();
  double t_last = t0;
  while (rc == NRLDPC_OK && done < n) {
    const double t = now_s() - t0;
    if (t > cfg->timeout_s) {
      fprintf(stderr, "nrldpc_serve_run: timeout after %.3f s with %lld of %d blocks finished\n", t,
              (long long)done, n);
      rc = NRLDPC_ERR_CUDA;
      break;
    }
    bool progress = false;
    // completions (batches on different streams may finish in any order)
    for (size_t q_i = 0; q_i < inflight.size();) {
      Slot& sl = slots[inflight[q_i]];
      const cudaError_t q = cudaEventQuery(sl.ev);
      if (q == cudaErrorNotReady) {
        ++q_i;
        continue;
      }
      if (q != cudaSuccess) {
        rc = NRLDPC_ERR_CUDA;
        break;
      }
      const double tv = now_s();
      for (size_t j = 0; j < sl.members.size(); ++j) {
        const int i = sl.members[j];
        h_status[i] = sl.h_status[j];
        h_latency_s[i] = (tv - t0) - arrival_s[i];
        budget_used -= 2 * (int64_t)tbs[i].G;
        st.completed++;
        if (sl.h_status[j] != 0) st.failed++;
        done++;
      }
      t_last = tv;
      free_slots.push_back(inflight[q_i]);
      inflight.erase(inflight.begin() + q_i);
      progress = true;
    }
    if (rc != NRLDPC_OK) break;
    // admitted blocks past their wait bound leave the queue (it is in arrival order)
    while (cfg->max_wait_s > 0.0 && !ready.empty() && t - arrival_s[ready.front()] > cfg->max_wait_s) {
      const int i = ready.front();
      ready.pop_front();
      h_status[i] = NRLDPC_TB_EXPIRED;
      h_latency_s[i] = NAN;
      budget_used -= 2 * (int64_t)tbs[i].G;
      st.expired++;
      done++;
      progress = true;
    }
    // arrivals: admit into the LLR budget or drop
    while (next < n && arrival_s[next] <= t) {
      const int64_t bytes = 2 * (int64_t)tbs[next].G;
      if (ncb[next] < 0) {
        h_status[next] = NRLDPC_ERR_CONFIG;
        h_latency_s[next] = NAN;
        done++;
      } else if (budget_used + bytes <= cfg->llr_budget_bytes) {
        ready.push_back(next);
        budget_used += bytes;
        st.admitted++;
      } else {
        h_status[next] = NRLDPC_TB_DROPPED;
        h_latency_s[next] = NAN;
        st.dropped++;
        done++;
      }
      next++;
      progress = true;
    }
    // launch a batch of everything admitted, up to the batch limits
    if (!ready.empty() && !free_slots.empty()) {
      const int k = free_slots.back();
      free_slots.pop_back();
      Slot& sl = slots[k];
      sl.members.clear();
      int cbs = 0;
      while (!ready.empty() && (int)sl.members.size() < max_tbs && cbs + ncb[ready.front()] <= max_cbs) {
        const int i = ready.front();
        ready.pop_front();
        sl.h_tbs[sl.members.size()] = tbs[i];
        sl.members.push_back(i);
        cbs += ncb[i];
      }
      const int m = (int)sl.members.size();
      cudaStream_t ss = sl.stream;
      if (cudaMemcpyAsync(sl.d_tbs, sl.h_tbs, (size_t)m * sizeof(nrldpc_tb_t), cudaMemcpyHostToDevice, ss) !=
              cudaSuccess ||
          engine_decode(e, k, sl.d_tbs, m, d_llr, d_out, sl.d_status, nullptr, nullptr, ss) != NRLDPC_OK ||
          cudaMemcpyAsync(sl.h_status, sl.d_status, (size_t)m * sizeof(int32_t), cudaMemcpyDeviceToHost, ss) !=
              cudaSuccess ||
          (cfg->h_cb_first && record_code_blocks(e, k, cfg, sl.members, ncb, ss) != NRLDPC_OK) ||
          cudaEventRecord(sl.ev, ss) != cudaSuccess) {
        rc = NRLDPC_ERR_CUDA;
        break;
      }
      inflight.push_back(k);
      st.batches++;
      batch_tbs_sum += m;
      progress = true;
    }
    if (!progress) std::this_thread::yield();
  }
  // leave nothing in flight that references the slot buffers; later work on
  // the caller's stream comes after every batch
  for (Slot& sl : slots) {
    if (sl.stream) {
      cudaStreamSynchronize(sl.stream);
      if (sl.ev && cudaEventRecord(sl.ev, sl.stream) == cudaSuccess) cudaStreamWaitEvent(s, sl.ev, 0);
    }
  }
  for (Slot& sl : slots) {
    cudaFreeHost(sl.h_tbs);
    cudaFreeHost(sl.h_status);
    cudaFree(sl.d_tbs);
    cudaFree(sl.d_status);
    if (sl.ev) cudaEventDestroy(sl.ev);
    if (sl.stream) cudaStreamDestroy(sl.stream);
  }
  if (start) cudaEventDestroy(start);
  st.wall_s = t_last - t0 - (n > 0 ? arrival_s[0] : 0.0);
  st.mean_batch_tbs = st.batches ? batch_tbs_sum / (double)st.batches : 0.0;
  if (stats) *stats = st;
  return rc;
}

}  // extern "C"
